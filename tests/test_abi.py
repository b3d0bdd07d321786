"""The drop-in boundary on CPU: librocrand.so loads, exports every entry point that
include/rocrand/rocrand.h declares, and the host-side status logic matches the reference's
library/src/rocrand.cpp (no kernel is launched here)."""

import ctypes
import os
import re

import pytest

import rocrand_b200 as rb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in (os.path.join("rocrand", "rocrand.h"), "rocrand_b200.h"):
        with open(os.path.join(ROOT, "include", h)) as f:
            text = f.read()
        names |= set(re.findall(r"\b(rocrand_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(lib):
    decl = declared_functions()
    assert len(decl) >= 33
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing


def test_version(lib):
    assert rb.get_version() == 300200


def _create(lib, t):
    g = ctypes.c_void_p()
    st = lib.rocrand_create_generator(ctypes.byref(g), t)
    return st, g


def test_null_generator_is_not_created(lib):
    null = ctypes.c_void_p(0)
    assert lib.rocrand_generate(null, None, 0) == rb.ROCRAND_STATUS_NOT_CREATED
    assert lib.rocrand_generate_uniform(null, None, 0) == rb.ROCRAND_STATUS_NOT_CREATED
    assert lib.rocrand_set_seed(null, 1) == rb.ROCRAND_STATUS_NOT_CREATED
    assert lib.rocrand_set_offset(null, 1) == rb.ROCRAND_STATUS_NOT_CREATED
    assert lib.rocrand_set_ordering(null, 101) == rb.ROCRAND_STATUS_NOT_CREATED
    assert lib.rocrand_generate_poisson(null, None, 0, 1.0) == rb.ROCRAND_STATUS_NOT_CREATED
    assert lib.rocrand_initialize_generator(null) == rb.ROCRAND_STATUS_NOT_CREATED


def test_unknown_type_is_type_error(lib):
    st, _ = _create(lib, 12345)
    assert st == rb.ROCRAND_STATUS_TYPE_ERROR


def test_version_null_pointer(lib):
    assert lib.rocrand_get_version(None) == rb.ROCRAND_STATUS_OUT_OF_RANGE


@pytest.mark.parametrize("rng", [rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10])
def test_host_side_semantics(lib, rng):
    st, g = _create(lib, rng)
    assert st == 0
    try:
        # lambda <= 0 is rejected before any work (rocrand.cpp:371-374)
        assert lib.rocrand_generate_poisson(g, None, 10, 0.0) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        assert lib.rocrand_generate_poisson(g, None, 10, -1.0) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        # 64-bit output from a 32-bit engine (philox4x32_10.hpp:359-375)
        assert lib.rocrand_generate_long_long(g, None, 10) == rb.ROCRAND_STATUS_TYPE_ERROR
        # orderings: quasi ordering and SEEDED are refused by Philox
        assert lib.rocrand_set_ordering(g, rb.ROCRAND_ORDERING_QUASI_DEFAULT) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        assert lib.rocrand_set_ordering(g, rb.ROCRAND_ORDERING_PSEUDO_SEEDED) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        for o in (100, 101, 103, 104):
            assert lib.rocrand_set_ordering(g, o) == 0
        # pseudo generators have no dimensions and no uint4 seed
        assert lib.rocrand_set_quasi_random_generator_dimensions(g, 4) == rb.ROCRAND_STATUS_TYPE_ERROR
        assert lib.rocrand_set_seed_uint4(g, rb._Uint4(1, 2, 3, 4)) == rb.ROCRAND_STATUS_TYPE_ERROR
        # a NULL output pointer initialises and returns SUCCESS (philox4x32_10.hpp:323-326);
        # initialising allocates the Poisson tables on the device (philox4x32_10.hpp:298), so
        # on a machine without one both calls report that allocation failing, as the
        # reference's do
        import torch
        init = 0 if torch.cuda.is_available() else rb.ROCRAND_STATUS_ALLOCATION_FAILED
        assert lib.rocrand_set_seed(g, 5) == 0
        assert lib.rocrand_set_offset(g, 17) == 0
        assert lib.rocrand_generate_uniform(g, None, 100) == init
        assert lib.rocrand_initialize_generator(g) == init
    finally:
        assert lib.rocrand_destroy_generator(g) == 0


def test_discrete_null_arguments(lib):
    lib.rocrand_create_poisson_distribution.argtypes = [ctypes.c_double, ctypes.c_void_p]
    lib.rocrand_create_discrete_distribution.argtypes = [ctypes.c_void_p, ctypes.c_uint,
                                                        ctypes.c_uint, ctypes.c_void_p]
    lib.rocrand_destroy_discrete_distribution.argtypes = [ctypes.c_void_p]
    out = ctypes.c_void_p()
    assert lib.rocrand_create_poisson_distribution(1.0, None) == rb.ROCRAND_STATUS_OUT_OF_RANGE
    assert lib.rocrand_create_poisson_distribution(0.0, ctypes.byref(out)) == rb.ROCRAND_STATUS_OUT_OF_RANGE
    assert lib.rocrand_create_discrete_distribution(None, 0, 0, ctypes.byref(out)) == rb.ROCRAND_STATUS_OUT_OF_RANGE
    assert lib.rocrand_destroy_discrete_distribution(None) == rb.ROCRAND_STATUS_OUT_OF_RANGE


def test_host_generator_creation(lib):
    """rocrand_create_generator_host(_blocking) (rocrand.cpp:118-160): every type is created,
    setters keep their meaning, unknown types give TYPE_ERROR, NULL out-pointer OUT_OF_RANGE."""
    import ctypes
    for create in (lib.rocrand_create_generator_host, lib.rocrand_create_generator_host_blocking):
        for t in (400, 401, 402, 403, 404, 405, 406, 407, 408, 409, 410, 411, 500, 501, 502, 504, 505):
            g = ctypes.c_void_p()
            assert create(ctypes.byref(g), t) == 0, t
            try:
                if t < 500:
                    assert lib.rocrand_set_seed(g, 7) == 0
                    if t in (403, 407):
                        assert lib.rocrand_set_offset(g, 5) == rb.ROCRAND_STATUS_TYPE_ERROR
                    else:
                        assert lib.rocrand_set_offset(g, 5) == 0
                else:
                    assert lib.rocrand_set_quasi_random_generator_dimensions(g, 0) == rb.ROCRAND_STATUS_OUT_OF_RANGE
                    assert lib.rocrand_set_quasi_random_generator_dimensions(g, 4) == 0
            finally:
                assert lib.rocrand_destroy_generator(g) == 0
        g = ctypes.c_void_p()
        assert create(ctypes.byref(g), 123) == rb.ROCRAND_STATUS_TYPE_ERROR
        assert create(None, 400) == rb.ROCRAND_STATUS_OUT_OF_RANGE


def test_mtgp32_host_side_semantics(lib):
    """MTGP32 (mtgp32.hpp:389-416): no offset, the four pseudo orderings, no 64-bit output."""
    st, g = _create(lib, rb.ROCRAND_RNG_PSEUDO_MTGP32)
    assert st == 0
    try:
        assert lib.rocrand_set_offset(g, 5) == rb.ROCRAND_STATUS_TYPE_ERROR
        for o in (rb.ROCRAND_ORDERING_PSEUDO_SEEDED, rb.ROCRAND_ORDERING_QUASI_DEFAULT):
            assert lib.rocrand_set_ordering(g, o) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        for o in (100, 101, 103, 104):
            assert lib.rocrand_set_ordering(g, o) == 0
        assert lib.rocrand_generate_long_long(g, None, 10) == rb.ROCRAND_STATUS_TYPE_ERROR
    finally:
        assert lib.rocrand_destroy_generator(g) == 0


def test_mt19937_host_side_semantics(lib):
    """MT19937 (mt19937.hpp:758-780, 1044-1060): no offset, orderings DEFAULT/BEST/LEGACY
    only, no 64-bit output; all refused before any device work."""
    st, g = _create(lib, rb.ROCRAND_RNG_PSEUDO_MT19937)
    assert st == 0
    try:
        assert lib.rocrand_set_offset(g, 5) == rb.ROCRAND_STATUS_TYPE_ERROR
        assert lib.rocrand_set_offset(g, 0) == rb.ROCRAND_STATUS_TYPE_ERROR
        for o in (rb.ROCRAND_ORDERING_PSEUDO_DYNAMIC, rb.ROCRAND_ORDERING_PSEUDO_SEEDED,
                  rb.ROCRAND_ORDERING_QUASI_DEFAULT):
            assert lib.rocrand_set_ordering(g, o) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        for o in (100, 101, 103):
            assert lib.rocrand_set_ordering(g, o) == 0
        assert lib.rocrand_generate_long_long(g, None, 10) == rb.ROCRAND_STATUS_TYPE_ERROR
        assert lib.rocrand_set_seed(g, 0) == 0
        assert lib.rocrand_set_quasi_random_generator_dimensions(g, 2) == rb.ROCRAND_STATUS_TYPE_ERROR
    finally:
        assert lib.rocrand_destroy_generator(g) == 0


C_CALLER = r"""
#include <rocrand/rocrand.h>
#include <rocrand_b200.h>
#include <stdio.h>
int main(void)
{
    rocrand_generator g;
    int               v = 0;
    if(rocrand_get_version(&v) != ROCRAND_STATUS_SUCCESS)
        return 1;
    if(rocrand_create_generator(&g, ROCRAND_RNG_QUASI_SOBOL32) != ROCRAND_STATUS_SUCCESS)
        return 2;
    if(rocrand_set_quasi_random_generator_dimensions(g, 64) != ROCRAND_STATUS_SUCCESS)
        return 3;
    if(rocrand_set_offset(g, 4096) != ROCRAND_STATUS_SUCCESS)
        return 4;
    if(rocrand_destroy_generator(g) != ROCRAND_STATUS_SUCCESS)
        return 5;
    printf("%d\n", v);
    return 0;
}
"""


def test_headers_compile_as_c_and_link(tmp_path, lib):
    """A C caller (the reference's rocrand.h is a C header: rocrand.h:52-54) compiles with gcc
    -std=c99 -Werror against include/, links against librocrand.so and runs its host calls."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "app.c"
    src.write_text(C_CALLER)
    exe = str(tmp_path / "app")
    pkg = os.path.join(ROOT, "rocrand_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", "-o", exe, str(src), "-L", pkg, "-lrocrand",
                    "-Wl,-rpath," + pkg], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stderr)
    assert out.stdout.strip() == "300200"
