"""Serving loop: requests on resident generator handles, batched while others run.

The property the serving path must keep: each result is the same alone and in the mix.
A random interleaving of requests on several handles (Philox, XORWOW, MRG32k3a, Sobol32;
uint / uniform fp32 / fp64 / normal fp32 / Poisson) is submitted to a server; every output
must equal, bit for bit, what a fresh generator of the handle's type and seed writes when it
makes the same calls alone, in the same order, through the plain C ABI.  Both server modes
(continuous batching, and the plain per-request baseline) are checked, with a pool small
enough that admission has to wait for memory.
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


class TraceItem(ctypes.Structure):
    _fields_ = [("arrival_seconds", ctypes.c_double), ("handle", ctypes.c_uint),
                ("distribution", ctypes.c_int), ("param0", ctypes.c_double),
                ("param1", ctypes.c_double), ("n", ctypes.c_size_t)]


def _setup(lib):
    lib.rocrand_b200_server_create.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint, ctypes.c_int]
    lib.rocrand_b200_server_destroy.argtypes = [ctypes.c_void_p]
    lib.rocrand_b200_server_add_generator.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_ulonglong,
                                                      ctypes.c_void_p]
    lib.rocrand_b200_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p]
    lib.rocrand_b200_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong, ctypes.c_void_p,
                                             ctypes.c_void_p]
    lib.rocrand_b200_server_release.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong]
    lib.rocrand_b200_server_run_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                                  ctypes.c_void_p, ctypes.c_void_p]


class _DeviceView:
    """A device pointer seen as a 1-D array by torch (no copy)."""

    def __init__(self, ptr, n, dtype):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": np.dtype(dtype).str,
                                         "data": (ptr, False), "version": 3}


def _copy_out(ptr, n, dtype):
    import torch
    return torch.as_tensor(_DeviceView(ptr, n, dtype), device="cuda").cpu().numpy().copy()


def _alone(lib, rng, seed, calls):
    """The same calls made alone on a fresh generator through the plain C ABI."""
    g = ctypes.c_void_p()
    assert lib.rocrand_create_generator(ctypes.byref(g), rng) == 0
    out = []
    try:
        assert lib.rocrand_set_seed(g, seed) == 0
        for d, n in calls:
            name, params = DISTS[d]
            st, vals = gu.device_generate(lib, g, name, n, params, 0)
            assert st == 0
            out.append(vals)
    finally:
        lib.rocrand_destroy_generator(g)
    return out


@pytest.mark.parametrize("plain", [0, 1])
def test_results_equal_alone_and_in_the_mix(lib, orc, plain):
    _setup(lib)
    rs = np.random.default_rng(123 + plain)
    server = ctypes.c_void_p()
    # 96 MiB pool: the mix below needs several times that, so admission waits for memory
    assert lib.rocrand_b200_server_create(ctypes.byref(server), 96 << 20, 3, plain) == 0
    try:
        handles = []
        for t in TYPES:
            for k in range(2):
                h = ctypes.c_uint()
                seed = int(rs.integers(0, 2**63))
                assert lib.rocrand_b200_server_add_generator(server, t, seed, ctypes.byref(h)) == 0
                handles.append((h.value, t, seed))
        submitted = []
        for _ in range(90):
            h, t, seed = handles[int(rs.integers(0, len(handles)))]
            d = int(rs.integers(0, 5))
            n = int(rs.choice([int(rs.integers(1, 300)), int(rs.integers(300, 70000)),
                               int(rs.integers(70000, 3000000))]))
            p = DISTS[d][1]
            ticket = ctypes.c_ulonglong()
            assert lib.rocrand_b200_server_submit(server, h, d, p[0] if p else 0.0,
                                                  p[1] if len(p) > 1 else 0.0, n,
                                                  ctypes.byref(ticket)) == 0
            submitted.append((ticket.value, h, d, n))
        results = {}
        for ticket, h, d, n in submitted:
            ptr, lat = ctypes.c_void_p(), ctypes.c_double()
            assert lib.rocrand_b200_server_wait(server, ticket, ctypes.byref(ptr), ctypes.byref(lat)) == 0
            assert lat.value >= 0.0
            results[ticket] = _copy_out(ptr.value, n, pyorc.DISTS[DISTS[d][0]][1])
            assert lib.rocrand_b200_server_release(server, ticket) == 0
        for h, t, seed in handles:
            mine = [(tk, d, n) for tk, hh, d, n in submitted if hh == h]
            want = _alone(lib, t, seed, [(d, n) for _, d, n in mine])
            for (tk, d, n), w in zip(mine, want):
                assert np.array_equal(results[tk].view(np.uint8), w.view(np.uint8)), (t, d, n)
        # one handle per generator type against the oracle itself, not only through the
        # plain calls: bit-exact classes identical, normals within the parity bound
        seen = set()
        for h, t, seed in handles:
            if t in seen:
                continue
            seen.add(t)
            mine = [(tk, d, n) for tk, hh, d, n in submitted if hh == h]
            calls = [(DISTS[d][0], n, list(DISTS[d][1]), 0) for _, d, n in mine]
            s = None if t == rb.ROCRAND_RNG_QUASI_SOBOL32 else seed
            for k, ((tk, d, n), (ost, ovals)) in enumerate(zip(mine, pyorc.run_sequence(orc, t, s, None, calls))):
                assert ost == 0
                if gu.bit_exact(t, DISTS[d][0]):
                    assert np.array_equal(results[tk].view(np.uint8), ovals.view(np.uint8)), (t, d, n)
                else:
                    gu.compare_call(orc, t, s, None, None, calls, k, results[tk], ovals)
    finally:
        assert lib.rocrand_b200_server_destroy(server) == 0


def test_trace_replay_and_errors(lib):
    _setup(lib)
    server = ctypes.c_void_p()
    assert lib.rocrand_b200_server_create(ctypes.byref(server), 64 << 20, 2, 0) == 0
    try:
        handles = []
        for t in TYPES:
            h = ctypes.c_uint()
            assert lib.rocrand_b200_server_add_generator(server, t, 42, ctypes.byref(h)) == 0
            handles.append(h.value)
        rs = np.random.default_rng(5)
        count = 400
        items = (TraceItem * count)()
        t = 0.0
        for i in range(count):
            t += float(rs.exponential(1.0 / 20000.0))
            items[i] = TraceItem(t, handles[i % 4], int(rs.integers(0, 3)), 0.0, 0.0,
                                 int(np.exp(rs.uniform(np.log(256), np.log(1 << 20)))))
        lat = (ctypes.c_double * count)()
        wall = ctypes.c_double()
        assert lib.rocrand_b200_server_run_trace(server, items, count, lat, ctypes.byref(wall)) == 0
        assert wall.value > 0.0 and all(x >= 0.0 for x in lat)
        ticket = ctypes.c_ulonglong()
        assert lib.rocrand_b200_server_submit(server, 999, 0, 0.0, 0.0, 10,
                                              ctypes.byref(ticket)) == rb.ROCRAND_STATUS_NOT_CREATED
        assert lib.rocrand_b200_server_submit(server, handles[0], 0, 0.0, 0.0, 1 << 30,
                                              ctypes.byref(ticket)) == rb.ROCRAND_STATUS_OUT_OF_RANGE
        mt = ctypes.c_uint()
        assert lib.rocrand_b200_server_add_generator(server, rb.ROCRAND_RNG_PSEUDO_MT19937, 1,
                                                     ctypes.byref(mt)) == rb.ROCRAND_STATUS_TYPE_ERROR
    finally:
        assert lib.rocrand_b200_server_destroy(server) == 0
