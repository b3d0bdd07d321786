"""Device API (include/rocrand/rocrand_kernel.h) against the reference's device API.

tests/devapi/harness.cu is compiled twice with the same flags: against this library's
headers (tests/devapi/libdevapi_b200.so) and against the reference's own device headers
(oracle/_ref/libdevapi_ref.so, built by oracle/Makefile.ref from the reference sources).
Both run on the B200 with the same inputs -- per thread a state initialised with seed,
subsequence t and offset 7t (Sobol: dimension vectors and offset 5t), then a run of calls of
one function -- and every result must be bit-identical: raw values, uniforms, normals and
log-normals (both evaluate the same expressions with the same device intrinsics), Poisson
(all three samplers: lambda below 64, up to 4000 and above) and discrete distributions,
skip-ahead by values, subsequences and sequences, and a mix that crosses the cached second
Box-Muller value.

Poisson lambda between 500 and 1000 is never run through the reference: its inversion sampler
(Sobol, ThreeFry, LFSR113) then searches until a 32-bit counter wraps (tens of seconds per
call); this library's sampler moves the segment bound and is checked on the CPU instead.
"""

import ctypes
import os
from ctypes import byref, c_double, c_int, c_size_t, c_uint, c_ulonglong, c_void_p, POINTER

import numpy as np
import pytest

import rocrand_b200 as rb

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OURS = os.path.join(HERE, "devapi", "libdevapi_b200.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libdevapi_ref.so")

ENGINES = {"philox": 0, "mrg32k3a": 1, "mrg31k3p": 2, "threefry2x32": 3, "threefry2x64": 4,
           "threefry4x32": 5, "threefry4x64": 6, "sobol32": 7, "scrambled_sobol32": 8, "sobol64": 9,
           "scrambled_sobol64": 10, "xorwow": 11, "lfsr113": 12}
FUNCS = {"rocrand": 0, "rocrand_block": 1, "uniform": 2, "uniform2": 3, "uniform4": 4, "uniform_double": 5,
         "uniform_double2": 6, "uniform_double4": 7, "normal": 8, "normal2": 9, "normal4": 10,
         "normal_double": 11, "normal_double2": 12, "normal_double4": 13, "log_normal": 14,
         "log_normal2": 15, "log_normal4": 16, "log_normal_double": 17, "log_normal_double2": 18,
         "log_normal_double4": 19, "poisson": 20, "poisson4": 21, "discrete": 22, "discrete4": 23,
         "skipahead": 24, "skipahead_subsequence": 25, "skipahead_sequence": 26, "mix": 27}
THREADS, CALLS = 256, 24


def _load(path):
    lib = ctypes.CDLL(path)
    lib.devapi_run.argtypes = [c_int, c_int, c_ulonglong, c_int, c_int, c_double, c_double, c_void_p,
                               c_ulonglong, c_void_p, c_void_p]
    lib.devapi_run.restype = c_int
    lib.devapi_run_mtgp32.argtypes = [c_int, c_ulonglong, c_int, c_int, c_double, c_double, c_void_p, c_void_p]
    lib.devapi_run_mtgp32.restype = c_int
    return lib


@pytest.fixture(scope="module")
def env(lib):
    import torch
    if not os.path.exists(REF):
        pytest.skip("reference device-API build (oracle/_ref/libdevapi_ref.so) absent")
    ours, ref = _load(OURS), _load(REF)
    lib.rocrand_get_direction_vectors32.argtypes = [POINTER(c_void_p), c_int]
    lib.rocrand_get_direction_vectors64.argtypes = [POINTER(c_void_p), c_int]
    lib.rocrand_get_scramble_constants32.argtypes = [POINTER(c_void_p)]
    lib.rocrand_get_scramble_constants64.argtypes = [POINTER(c_void_p)]
    lib.rocrand_create_poisson_distribution.argtypes = [c_double, POINTER(c_void_p)]
    lib.rocrand_destroy_discrete_distribution.argtypes = [c_void_p]
    dim = 3
    vec = {}
    for name, fn, words, t, sets in (("sobol32", lib.rocrand_get_direction_vectors32, 32, np.uint32, (101, 102)),
                                     ("sobol64", lib.rocrand_get_direction_vectors64, 64, np.uint64, (103, 104))):
        for scrambled, s in zip((False, True), sets):
            p = c_void_p()
            assert fn(byref(p), s) == 0
            host = np.ctypeslib.as_array(ctypes.cast(p, POINTER(ctypes.c_uint32 if words == 32 else ctypes.c_uint64)),
                                         shape=((dim + 1) * words,))[dim * words:(dim + 1) * words].copy()
            vec[(name, scrambled)] = torch.from_numpy(host.view(np.int32 if words == 32 else np.int64)).cuda()
    sc = {}
    for name, fn, t in (("sobol32", lib.rocrand_get_scramble_constants32, ctypes.c_uint32),
                        ("sobol64", lib.rocrand_get_scramble_constants64, ctypes.c_uint64)):
        p = c_void_p()
        assert fn(byref(p)) == 0
        sc[name] = int(ctypes.cast(p, POINTER(t))[dim])
    dist = c_void_p()
    assert lib.rocrand_create_poisson_distribution(c_double(40.5), byref(dist)) == 0
    yield ours, ref, vec, sc, dist
    lib.rocrand_destroy_discrete_distribution(dist)


def _run(env, engine, func, p0, p1, seed=0x1234567890ABCDEF):
    import torch
    ours, ref, vec, sc, dist = env
    e = ENGINES[engine]
    v, s = None, 0
    if e >= 7:
        fam = "sobol32" if e in (7, 8) else "sobol64"
        scrambled = e in (8, 10)
        v = vec[(fam, scrambled)].data_ptr()
        s = sc[fam] if scrambled else 0
    outs = []
    for lib in (ours, ref):
        out = torch.zeros(THREADS * CALLS * 32, dtype=torch.uint8, device="cuda")
        st = lib.devapi_run(e, FUNCS[func], seed, THREADS, CALLS, p0, p1, v, s, dist.value, out.data_ptr())
        outs.append((st, out.cpu().numpy()))
    return outs


CASES = [("rocrand", 0, 0), ("rocrand_block", 0, 0), ("uniform", 0, 0), ("uniform2", 0, 0), ("uniform4", 0, 0),
         ("uniform_double", 0, 0), ("uniform_double2", 0, 0), ("uniform_double4", 0, 0), ("normal", 0, 0),
         ("normal2", 0, 0), ("normal4", 0, 0), ("normal_double", 0, 0), ("normal_double2", 0, 0),
         ("normal_double4", 0, 0), ("log_normal", 0.3, 0.7), ("log_normal2", 0.3, 0.7), ("log_normal4", 0.3, 0.7),
         ("log_normal_double", -0.2, 1.5), ("log_normal_double2", -0.2, 1.5), ("log_normal_double4", -0.2, 1.5),
         ("poisson", 3.5, 0), ("poisson", 300.0, 0), ("poisson", 2500.0, 0), ("poisson", 5000.0, 0),
         ("poisson4", 20.0, 0), ("discrete", 0, 0), ("discrete4", 0, 0), ("skipahead", 1000003, 0),
         ("skipahead_subsequence", 5, 0), ("skipahead_sequence", 3, 0), ("mix", 0.1, 0.9)]


@pytest.mark.parametrize("func,p0,p1", CASES, ids=lambda x: str(x))
@pytest.mark.parametrize("engine", sorted(ENGINES))
def test_device_api_equals_reference(env, engine, func, p0, p1):
    (so, vo), (sr, vr) = _run(env, engine, func, float(p0), float(p1))
    assert so != 2 and sr != 2, (so, sr)
    if sr == 1:
        pytest.skip("the reference has no %s for %s" % (func, engine))
    assert so == 0, "the reference has %s for %s, this library does not" % (func, engine)
    assert np.array_equal(vo, vr), np.flatnonzero(vo != vr)[:8]


MTGP_BLOCKS = 37


@pytest.mark.parametrize("func,p0,p1", CASES + [("set_params", 0, 0)], ids=lambda x: str(x))
def test_mtgp32_block_api_equals_reference(env, func, p0, p1):
    """rocrand_state_mtgp32: states from rocrand_make_state_mtgp32 (published parameter sets),
    block-copied to shared memory, every thread of the block calling together."""
    import torch
    ours, ref, _, _, dist = env
    f = 28 if func == "set_params" else FUNCS[func]
    outs = []
    for lib in (ours, ref):
        out = torch.zeros(MTGP_BLOCKS * 256 * CALLS * 32, dtype=torch.uint8, device="cuda")
        st = lib.devapi_run_mtgp32(f, 0xC0FFEE1234, MTGP_BLOCKS, CALLS, float(p0), float(p1), dist.value,
                                   out.data_ptr())
        outs.append((st, out.cpu().numpy()))
    (so, vo), (sr, vr) = outs
    assert so != 2 and sr != 2, (so, sr)
    if sr == 1:
        pytest.skip("the reference has no %s for MTGP32" % func)
    assert so == 0
    assert np.array_equal(vo, vr), np.flatnonzero(vo != vr)[:8]
