"""Generate calls recorded by a CUDA graph capture, as in the reference's
test/test_rocrand_hipgraphs.cpp: the generator is initialised (rocrand_initialize_generator)
and bound to a non-blocking stream, then each call -- sizes 1, 2 at a misaligned pointer and
12563; uniform, normal, log-normal, and Poisson with lambda 10, 500 and 5000 (each a new table
inside its capture) -- is captured alone (global capture mode), the graph launched, and the
result must equal the same call made directly on a twin generator.  A replay of a captured
Poisson call after the table changed must give the captured lambda's values again: the table
travels with the graph."""

import ctypes
from ctypes import c_double, c_float, c_size_t, c_void_p

import numpy as np
import pytest

import rocrand_b200 as rb

pytestmark = pytest.mark.gpu

TYPES = [rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, rb.ROCRAND_RNG_PSEUDO_XORWOW, rb.ROCRAND_RNG_PSEUDO_MRG32K3A,
         rb.ROCRAND_RNG_PSEUDO_MRG31K3P, rb.ROCRAND_RNG_PSEUDO_LFSR113, rb.ROCRAND_RNG_PSEUDO_MT19937,
         rb.ROCRAND_RNG_PSEUDO_MTGP32, rb.ROCRAND_RNG_PSEUDO_THREEFRY2_32_20,
         rb.ROCRAND_RNG_PSEUDO_THREEFRY4_64_20, rb.ROCRAND_RNG_QUASI_SOBOL32,
         rb.ROCRAND_RNG_QUASI_SCRAMBLED_SOBOL64]
SIZE = 12563


def _generator(lib, rng, stream):
    g = c_void_p()
    assert lib.rocrand_create_generator(ctypes.byref(g), rng) == 0
    assert lib.rocrand_set_stream(g, c_void_p(stream.cuda_stream)) == 0
    assert lib.rocrand_initialize_generator(g) == 0
    return g


def _calls(lib, kind):
    """(function, element dtype, extra arguments) of each call of the reference's test."""
    if kind == "uniform":
        return [(lib.rocrand_generate_uniform, "float32", ())] * 3
    if kind == "normal":
        return [(lib.rocrand_generate_normal, "float32", (c_float(5.0), c_float(2.0)))] * 3
    if kind == "log_normal":
        return [(lib.rocrand_generate_log_normal, "float32", (c_float(5.0), c_float(2.0)))] * 3
    return [(lib.rocrand_generate_poisson, "int32", (c_double(lam),)) for lam in (10.0, 500.0, 5000.0)]


@pytest.mark.parametrize("kind", ["uniform", "normal", "log_normal", "poisson"])
@pytest.mark.parametrize("rng", TYPES)
def test_captured_calls_equal_direct_calls(lib, rng, kind):
    import torch
    stream = torch.cuda.Stream()
    g = _generator(lib, rng, stream)
    twin = _generator(lib, rng, stream)
    dtype = getattr(torch, _calls(lib, kind)[0][1])
    out = torch.zeros(SIZE + 8, dtype=dtype, device="cuda")
    ref = torch.zeros(SIZE + 8, dtype=dtype, device="cuda")
    graphs = []
    try:
        for (fn, _, extra), (off, n) in zip(_calls(lib, kind), [(0, 1), (1, 2), (0, SIZE)]):
            # the direct call first (it also loads the kernel outside the capture)
            with torch.cuda.stream(stream):
                assert fn(twin, c_void_p(ref.data_ptr() + off * ref.element_size()), c_size_t(n), *extra) == 0
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=stream, capture_error_mode="global"):
                st = fn(g, c_void_p(out.data_ptr() + off * out.element_size()), c_size_t(n), *extra)
            assert st == 0, st
            graph.replay()
            stream.synchronize()
            a = out[off:off + n].cpu().numpy()
            b = ref[off:off + n].cpu().numpy()
            assert np.array_equal(a.view(np.uint32 if a.itemsize == 4 else np.uint64),
                                  b.view(np.uint32 if b.itemsize == 4 else np.uint64)), (off, n)
            graphs.append((graph, off, n, a.copy()))
        if kind == "poisson" and rng in (rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, rb.ROCRAND_RNG_QUASI_SOBOL32):
            # a counter-based or quasi generator replays the same positions: the first graph
            # (lambda 10) after the table moved on to lambda 500 gives its lambda-10 values again
            graph, off, n, first = graphs[0]
            graph.replay()
            stream.synchronize()
            assert np.array_equal(out[off:off + n].cpu().numpy(), first)
    finally:
        del graphs
        stream.synchronize()
        lib.rocrand_destroy_generator(g)
        lib.rocrand_destroy_generator(twin)
