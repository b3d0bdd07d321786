"""Batched fill (rocrand_b200_generate_batch and batch plans) against plain calls.

Each request of a batch must write exactly what one plain call of the same generator type,
seed, offset and distribution writes on a fresh generator: bit for bit (normals included:
the batch kernel evaluates the same functors).  The batches mix generator types, sizes from
a few values to more than one engine round, output alignments, and Poisson lambdas.
"""

import ctypes

import numpy as np
import pytest

import rocrand_b200 as rb
from oracle import pyorc
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu

DISTS = {0: ("uint", ()), 1: ("uniform", ()), 2: ("uniform_double", ()),
         3: ("normal", (0.5, 2.0)), 4: ("poisson", (4.0,))}
TYPES = [rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, rb.ROCRAND_RNG_PSEUDO_XORWOW,
         rb.ROCRAND_RNG_PSEUDO_MRG32K3A, rb.ROCRAND_RNG_QUASI_SOBOL32]


class Request(ctypes.Structure):
    _fields_ = [("rng_type", ctypes.c_int), ("distribution", ctypes.c_int),
                ("seed", ctypes.c_ulonglong), ("offset", ctypes.c_ulonglong),
                ("param0", ctypes.c_double), ("param1", ctypes.c_double),
                ("output", ctypes.c_void_p), ("n", ctypes.c_size_t)]


def _plain(lib, rng, seed, offset, dist, n, mis):
    g = ctypes.c_void_p()
    assert lib.rocrand_create_generator(ctypes.byref(g), rng) == 0
    try:
        if rng != rb.ROCRAND_RNG_QUASI_SOBOL32:
            assert lib.rocrand_set_seed(g, seed) == 0
        assert lib.rocrand_set_offset(g, offset) == 0
        name, params = DISTS[dist]
        st, vals = gu.device_generate(lib, g, name, n, params, mis)
        assert st == 0
        return vals
    finally:
        lib.rocrand_destroy_generator(g)


def _make(rng_rs, count, types=TYPES, dists=(0, 1, 2, 3, 4)):
    reqs = []
    for _ in range(count):
        t = types[int(rng_rs.integers(0, len(types)))]
        d = dists[int(rng_rs.integers(0, len(dists)))]
        n = int(rng_rs.choice([int(rng_rs.integers(1, 64)), int(rng_rs.integers(64, 20000)),
                               int(rng_rs.integers(20000, 400000))]))
        offset = int(rng_rs.integers(0, 1 << 20)) if rng_rs.random() < 0.3 else 0
        reqs.append((t, d, int(rng_rs.integers(0, 2**63)), offset, n, int(rng_rs.integers(0, 4))))
    return reqs


def _run_batch(lib, reqs, plan_mode=None):
    import torch
    bufs, arr = [], (Request * len(reqs))()
    for k, (t, d, seed, offset, n, mis) in enumerate(reqs):
        dt = gu.torch_dtype(DISTS[d][0])
        buf = torch.zeros(n + 16, dtype=dt, device="cuda")
        bufs.append(buf)
        p = DISTS[d][1]
        arr[k] = Request(t, d, seed, offset, p[0] if p else 0.0, p[1] if len(p) > 1 else 0.0,
                         buf[mis:].data_ptr(), n)
    stream = torch.cuda.current_stream().cuda_stream
    if plan_mode is None:
        assert lib.rocrand_b200_generate_batch(arr, len(reqs), ctypes.c_void_p(stream)) == 0
    else:
        plan = ctypes.c_void_p()
        assert lib.rocrand_b200_create_batch_plan(ctypes.byref(plan), arr, len(reqs),
                                                  ctypes.c_void_p(stream)) == 0
        for _ in range(2):  # the second execution of a graph plan is a replay
            for b in bufs:
                b.zero_()
            assert lib.rocrand_b200_execute_batch_plan(plan, plan_mode, ctypes.c_void_p(stream)) == 0
        assert lib.rocrand_b200_destroy_batch_plan(plan) == 0
    torch.cuda.synchronize()
    out = []
    for (t, d, seed, offset, n, mis), buf in zip(reqs, bufs):
        out.append(buf[mis:mis + n].cpu().numpy().view(pyorc.DISTS[DISTS[d][0]][1]))
    return out


def _check(lib, reqs, got):
    for (t, d, seed, offset, n, mis), vals in zip(reqs, got):
        want = _plain(lib, t, seed, offset, d, n, mis)
        assert np.array_equal(vals.view(np.uint8), want.view(np.uint8)), (t, d, seed, offset, n, mis)


@pytest.mark.parametrize("seed", [1, 2])
def test_batch_equals_plain_calls(lib, seed):
    _setup(lib)
    reqs = _make(np.random.default_rng(seed), 60)
    _check(lib, reqs, _run_batch(lib, reqs))


def test_batch_equals_oracle(lib, orc):
    """Each request of a batch against the oracle directly, not only through the plain call
    of the same generator: bit-exact classes identical, normals within the parity bound."""
    _setup(lib)
    reqs = _make(np.random.default_rng(77), 24)
    got = _run_batch(lib, reqs)
    for (t, d, seed, offset, n, mis), vals in zip(reqs, got):
        name, params = DISTS[d]
        calls = [(name, n, list(params), mis)]
        s = None if t == rb.ROCRAND_RNG_QUASI_SOBOL32 else seed
        (ost, ovals), = pyorc.run_sequence(orc, t, s, offset, calls)
        assert ost == 0
        if gu.bit_exact(t, name):
            assert np.array_equal(vals.view(np.uint8), ovals.view(np.uint8)), (t, d, seed, offset, n, mis)
        else:
            gu.compare_call(orc, t, s, offset, None, calls, 0, vals, ovals)


@pytest.mark.parametrize("use_graph", [0, 1])
def test_batch_plan_and_graph_replay(lib, use_graph):
    _setup(lib)
    reqs = _make(np.random.default_rng(10 + use_graph), 40)
    _check(lib, reqs, _run_batch(lib, reqs, plan_mode=use_graph))


def test_batch_large_stateful_requests(lib):
    """Requests longer than one engine round (131072 engines) and with offsets beyond it."""
    _setup(lib)
    reqs = [(rb.ROCRAND_RNG_PSEUDO_XORWOW, 1, 99, 0, 3 * 131072 + 77, 0),
            (rb.ROCRAND_RNG_PSEUDO_XORWOW, 3, 98, 131072 * 2 + 5, 262147, 1),
            (rb.ROCRAND_RNG_PSEUDO_MRG32K3A, 2, 97, 131073, 300001, 1),
            (rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, 3, 96, 7, 262144 * 4 * 2 + 9, 1),
            (rb.ROCRAND_RNG_QUASI_SOBOL32, 4, 0, 4096, 1 << 20, 0)]
    _check(lib, reqs, _run_batch(lib, reqs))


def test_batch_rejects_bad_requests(lib):
    import torch
    _setup(lib)
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    bad_type = (Request * 1)(Request(rb.ROCRAND_RNG_PSEUDO_MT19937, 1, 1, 0, 0.0, 0.0, buf.data_ptr(), 8))
    assert lib.rocrand_b200_generate_batch(bad_type, 1, None) == rb.ROCRAND_STATUS_TYPE_ERROR
    bad_lambda = (Request * 1)(Request(rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, 4, 1, 0, 0.0, 0.0,
                                       buf.data_ptr(), 8))
    assert lib.rocrand_b200_generate_batch(bad_lambda, 1, None) == rb.ROCRAND_STATUS_OUT_OF_RANGE


def test_autotune_keeps_outputs(lib):
    """Tile sizes change the tiling only: outputs after autotuning are unchanged."""
    _setup(lib)
    assert lib.rocrand_b200_autotune_batch(None) == 0
    units = ctypes.c_uint()
    for t in TYPES:
        for d in DISTS:
            assert lib.rocrand_b200_get_batch_tile(t, d, ctypes.byref(units)) == 0
            assert units.value > 0
    reqs = _make(np.random.default_rng(77), 30)
    _check(lib, reqs, _run_batch(lib, reqs))


def _setup(lib):
    lib.rocrand_b200_generate_batch.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.rocrand_b200_create_batch_plan.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                                   ctypes.c_void_p]
    lib.rocrand_b200_execute_batch_plan.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.rocrand_b200_destroy_batch_plan.argtypes = [ctypes.c_void_p]
    lib.rocrand_b200_autotune_batch.argtypes = [ctypes.c_void_p]
    lib.rocrand_b200_get_batch_tile.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
