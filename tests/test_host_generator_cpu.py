"""Host generators computed on the CPU (no GPU needed), against the oracle.

In a process without a CUDA device -- or with ROCRAND_B200_HOST_CPU=1, set here around each
test so that it also runs the CPU form on a machine with a GPU -- rocrand_create_generator_host
returns the generator in host execution: every generate call writes host memory through the
same engine, output-order and distribution code as the kernels, compiled for the host, with
the C library's fp32 transcendentals (the reference's host path takes the same ones).  Each
call of a random sequence of distributions, sizes and misalignments must equal the oracle's
-- bit for bit, fp32 normals included; fp64 normals within the parity tests' tolerance
(tests/gpu_util.compare_call).
"""

import ctypes
import os
import zlib

import numpy as np
import pytest

from oracle import pyorc
from tests import gpu_util as gu



@pytest.fixture(autouse=True)
def _host_cpu(monkeypatch):
    """Host execution for the generators these tests create (read at creation), and only
    for them: the variable is removed again after each test."""
    monkeypatch.setenv("ROCRAND_B200_HOST_CPU", "1")

CPU_FAMILIES = {"xorwow": 401, "mrg32k3a": 402, "mtgp32": 403, "philox": 404, "mrg31k3p": 405,
                "lfsr113": 406, "mt19937": 407, "threefry2x32": 408, "threefry2x64": 409,
                "threefry4x32": 410, "threefry4x64": 411}
NO_OFFSET = {403, 407}  # MTGP32 and MT19937 take no offset (mtgp32.hpp:389-393, mt19937.hpp:758-763)
DISTS = [("uint", []), ("char", []), ("short", []), ("uniform", []), ("uniform_double", []),
         ("uniform_half", []), ("normal", [0.0, 1.0]), ("normal", [1.5, 2.0]), ("normal_double", [0.0, 1.0]),
         ("normal_half", [0.0, 1.0]), ("log_normal", [0.0, 0.5]), ("log_normal_double", [0.0, 0.5]),
         ("poisson", [0.5]), ("poisson", [10.0]), ("poisson", [1000.0]), ("poisson", [4500.0]),
         ("ulonglong", [])]


@pytest.fixture(scope="module")
def orc():
    return pyorc.CLib("orc")


def host_generate(lib, g, dist, n, params, mis):
    """One call into host memory placed (mis * itemsize) bytes past a 64-byte boundary (the
    oracle's placement); (status, values)."""
    suffix, dt, _ = pyorc.DISTS[dist]
    isz = np.dtype(dt).itemsize
    buf = np.zeros(n + 64 // isz + 16, dtype=dt)
    base = (-buf.ctypes.data // isz) % (64 // isz)
    view = buf[base + mis:base + mis + n]
    st = getattr(lib, "rocrand_" + suffix)(g, ctypes.c_void_p(view.ctypes.data), ctypes.c_size_t(n),
                                           *pyorc.dist_args(dist, params))
    return st, view.copy()


def run_case(lib, orc, rng, seed, offset, calls, dims=None):
    g = ctypes.c_void_p()
    assert lib.rocrand_create_generator_host(ctypes.byref(g), rng) == 0
    try:
        if seed is not None:
            assert lib.rocrand_set_seed(g, seed) == 0
        if dims is not None:
            assert lib.rocrand_set_quasi_random_generator_dimensions(g, dims) == 0
        if offset is not None:
            assert lib.rocrand_set_offset(g, offset) == 0
        ref = pyorc.run_sequence(orc, rng, seed, offset, calls, dims=dims)
        for k, ((d, n, p, mis), (ost, ovals)) in enumerate(zip(calls, ref)):
            st, vals = host_generate(lib, g, d, n, p, mis)
            assert st == ost, (rng, d, st, ost)
            if st != 0:
                continue
            if d in gu.BIT_EXACT or d in ("normal", "normal_half", "log_normal"):
                # fp32 transforms take the C library's functions on the host: bit-exact
                assert np.array_equal(vals.view(np.uint8), ovals.view(np.uint8)), (rng, d, n, mis)
            else:
                gu.compare_call(orc, rng, seed, offset, dims, calls, k, vals, ovals)
    finally:
        lib.rocrand_destroy_generator(g)


@pytest.mark.parametrize("name", sorted(CPU_FAMILIES))
def test_cpu_host_generator_sequences(lib, orc, name):
    rng = CPU_FAMILIES[name]
    rs = np.random.default_rng(zlib.crc32(name.encode()))
    seed = int(rs.integers(0, 2**63))
    offset = int(rs.integers(0, 2**20)) if rs.random() < 0.5 and rng not in NO_OFFSET else None
    calls = []
    for k in range(24):
        d, p = DISTS[int(rs.integers(0, len(DISTS)))]
        n = int(rs.choice([int(rs.integers(1, 40)), int(rs.integers(1, 5000)), int(rs.integers(1, 300000))]))
        calls.append((d, n, p, int(rs.integers(0, 16))))
    run_case(lib, orc, rng, seed, offset, calls)


QUASI = {"sobol32": 501, "scrambled_sobol32": 502, "sobol64": 504, "scrambled_sobol64": 505}


@pytest.mark.parametrize("name", sorted(QUASI))
def test_cpu_quasi_host_generator_sequences(lib, orc, name):
    rng = QUASI[name]
    rs = np.random.default_rng(zlib.crc32(name.encode()))
    dims = int(rs.choice([1, 3, 64]))
    offset = int(rs.integers(0, 2**20))
    calls = []
    for k in range(16):
        d, p = DISTS[int(rs.integers(0, len(DISTS)))]
        n = dims * int(rs.choice([int(rs.integers(1, 40)), int(rs.integers(1, 3000)), int(rs.integers(1, 60000))]))
        calls.append((d, n, p, int(rs.integers(0, 16))))
    run_case(lib, orc, rng, None, offset, calls, dims=dims)


def test_cpu_host_generator_large_call(lib, orc):
    """2^22 values in one call (spread over the host's cores) equal the oracle."""
    run_case(lib, orc, 404, 0xdeadbeef, 0, [("uniform", (1 << 22) + 3, [], 1), ("poisson", 1 << 21, [7.5], 0)])


CPU_ONLY_SCRIPT = r"""
import ctypes, sys
import numpy as np
import rocrand_b200
from oracle import pyorc
lib = rocrand_b200.load_library()
orc = pyorc.CLib("orc")
for rng in (401, 403, 404, 407, 501):
    calls = [("uint", 1000, [], 0), ("uniform", 777, [], 3), ("poisson", 5000, [12.5], 1)]
    ref = pyorc.run_sequence(orc, rng, 42 if rng != 501 else None, None, calls)
    g = ctypes.c_void_p()
    assert lib.rocrand_create_generator_host(ctypes.byref(g), rng) == 0
    if rng != 501:
        assert lib.rocrand_set_seed(g, 42) == 0
    for (d, n, p, mis), (ost, ovals) in zip(calls, ref):
        suffix, dt, _ = pyorc.DISTS[d]
        buf = np.zeros(n + 32, dtype=dt)
        isz = np.dtype(dt).itemsize
        base = (-buf.ctypes.data // isz) % (64 // isz)
        view = buf[base + mis:base + mis + n]
        st = getattr(lib, "rocrand_" + suffix)(g, ctypes.c_void_p(view.ctypes.data), ctypes.c_size_t(n),
                                               *pyorc.dist_args(d, p))
        assert st == ost == 0, (rng, d, st, ost)
        assert np.array_equal(view, ovals), (rng, d)
    lib.rocrand_destroy_generator(g)
print("cpu-only ok")
"""


def test_cpu_only_process_without_env():
    """A process that sees no CUDA device (CUDA_VISIBLE_DEVICES empty, no host-CPU switch)
    gets host generators computed on the CPU, equal to the oracle."""
    import subprocess
    import sys
    env = dict(os.environ)
    env.pop("ROCRAND_B200_HOST_CPU", None)
    env["CUDA_VISIBLE_DEVICES"] = ""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", CPU_ONLY_SCRIPT], cwd=root, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpu-only ok" in r.stdout


OUTPUT = {"uint": 0, "uniform_double": 5, "normal": 7, "poisson": 13}
POSITIONED = {"xorwow": 401, "mrg32k3a": 402, "mrg31k3p": 405, "lfsr113": 406, "philox": 404,
              "threefry2x64": 409}


@pytest.mark.parametrize("name", sorted(POSITIONED))
@pytest.mark.parametrize("dist,params", [("uniform_double", []), ("normal", [0.0, 1.0]), ("uint", []),
                                         ("poisson", [10.0])])
def test_cpu_output_position_slices(lib, orc, name, dist, params):
    """rocrand_b200_set_output_position on the CPU form: a generator positioned at output
    r*n writes outputs [r*n, (r+1)*n) of the oracle's one long call, and continues it."""
    rng = POSITIONED[name]
    seed = 0xACE + rng
    n = 2 * 131072 + 6
    ranks = 3
    (ost, whole), = pyorc.run_sequence(orc, rng, seed, None, [(dist, ranks * n, params, 0)])
    assert ost == 0
    for r in range(ranks):
        g = ctypes.c_void_p()
        assert lib.rocrand_create_generator_host(ctypes.byref(g), rng) == 0
        try:
            assert lib.rocrand_set_seed(g, seed) == 0
            assert lib.rocrand_b200_set_output_position(g, OUTPUT[dist], r * n) == 0
            st, part = host_generate(lib, g, dist, n, params, 0)
            assert st == 0
            st, more = host_generate(lib, g, dist, 1000, params, 0)
            assert st == 0
        finally:
            lib.rocrand_destroy_generator(g)
        assert np.array_equal(part.view(np.uint8), whole[r * n:(r + 1) * n].view(np.uint8)), (name, dist, r)
        if r < ranks - 1:
            assert np.array_equal(more.view(np.uint8),
                                  whole[(r + 1) * n:(r + 1) * n + 1000].view(np.uint8)), (name, dist, r)


def test_cpu_mt19937_calls_across_rounds(lib, orc):
    """MT19937 on the CPU with calls longer than a round (65536 lanes x 78 slots) and one that
    starts mid-round and crosses the next twist, against the oracle."""
    run_case(lib, orc, 407, 0x600D, None, [("uint", 5200001, [], 0), ("uniform", 5500000, [], 1),
                                           ("normal", 1001, [0.0, 1.0], 3), ("uint", 77, [], 2)])
