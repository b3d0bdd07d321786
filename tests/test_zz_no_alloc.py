"""The Poisson entry point that allocates nothing, against the generator path and the oracle.

Callers that cannot call cudaMalloc (inside a graph capture or a driver callback, or with
device memory fully pre-partitioned) use rocrand_b200_generate_poisson_noalloc, whose alias
table lives in a fixed array of the library.  Its values must equal those of a Philox4x32-10
generator calling rocrand_generate_poisson with the same seed and offset -- bit for bit, the
Poisson tolerance of every other test -- on two calls in a row (the second continuing the
stream and switching lambda, so the shared array is rewritten).  Collected last so a run
stopping at the first failure has already run everything else; it also passes on its own in
a fresh process.
"""

import ctypes

import numpy as np
import pytest

import rocrand_b200 as rb

pytestmark = pytest.mark.gpu


def _entry(lib):
    f = lib.rocrand_b200_generate_poisson_noalloc
    f.argtypes = [ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.c_size_t,
                  ctypes.c_double, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_poisson_equals_generator_two_calls(lib):
    import torch
    noalloc = _entry(lib)
    seed, n0, n1 = 0x5EED1234, (1 << 20) + 3, 77777
    lambdas = (10.0, 1000.0)

    g = ctypes.c_void_p()
    assert lib.rocrand_create_generator(ctypes.byref(g), rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10) == 0
    assert lib.rocrand_set_seed(g, seed) == 0
    want = []
    for n, lam in zip((n0, n1), lambdas):
        buf = torch.empty(n, dtype=torch.int32, device="cuda")
        assert lib.rocrand_generate_poisson(g, ctypes.c_void_p(buf.data_ptr()), n, lam) == 0
        want.append(buf)
    torch.cuda.synchronize()
    assert lib.rocrand_destroy_generator(g) == 0

    stream = torch.cuda.current_stream().cuda_stream
    offset = 0
    for k, (n, lam) in enumerate(zip((n0, n1), lambdas)):
        got = torch.empty(n, dtype=torch.int32, device="cuda")
        st = noalloc(seed, offset, ctypes.c_void_p(got.data_ptr()), n, lam, ctypes.c_void_p(stream))
        assert st == 0
        torch.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy(), want[k].cpu().numpy()), "call %d" % k
        offset += n


def _generator_values(lib, seed, calls):
    """Values of one Philox4x32-10 generator making the given (n, lambda) calls in order."""
    import torch
    g = ctypes.c_void_p()
    assert lib.rocrand_create_generator(ctypes.byref(g), rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10) == 0
    assert lib.rocrand_set_seed(g, seed) == 0
    out = []
    for n, lam in calls:
        buf = torch.empty(n, dtype=torch.int32, device="cuda")
        assert lib.rocrand_generate_poisson(g, ctypes.c_void_p(buf.data_ptr()), n, lam) == 0
        out.append(buf)
    torch.cuda.synchronize()
    assert lib.rocrand_destroy_generator(g) == 0
    return [b.cpu().numpy() for b in out]


@pytest.mark.parametrize("mis", [1, 2, 3])
def test_noalloc_large_lambda_and_unaligned_output(lib, mis):
    """lambda above 4000 (no table: the normal approximation) followed by a table lambda,
    both written 1-3 elements past an aligned address (the head/tail path of the kernel)."""
    import torch
    noalloc = _entry(lib)
    seed = 0xC0FFEE + mis
    calls = [(100003, 4001.0), (65537, 4.0)]
    want = _generator_values(lib, seed, calls)
    stream = torch.cuda.current_stream().cuda_stream
    offset = 0
    for k, (n, lam) in enumerate(calls):
        buf = torch.empty(n + 8, dtype=torch.int32, device="cuda")
        view = buf[mis:mis + n]
        assert noalloc(seed, offset, ctypes.c_void_p(view.data_ptr()), n, lam, ctypes.c_void_p(stream)) == 0
        torch.cuda.synchronize()
        assert np.array_equal(view.cpu().numpy(), want[k]), "call %d" % k
        offset += n


def test_noalloc_equals_oracle(lib, orc):
    """The entry point against the oracle directly: a Philox4x32-10 stream at a seed and an
    offset, table and no-table lambdas, an aligned and a misaligned output."""
    import torch
    from oracle import pyorc
    noalloc = _entry(lib)
    stream = torch.cuda.current_stream().cuda_stream
    for seed, offset, n, lam, mis in ((0x1234, 0, 200001, 10.0, 0), (77, 12345, 99999, 1000.0, 3),
                                      (5, 7, 50003, 4500.0, 1)):
        (ost, ovals), = pyorc.run_sequence(orc, rb.ROCRAND_RNG_PSEUDO_PHILOX4_32_10, seed, offset,
                                           [("poisson", n, [lam], mis)])
        assert ost == 0
        buf = torch.empty(n + 8, dtype=torch.int32, device="cuda")
        view = buf[mis:mis + n]
        assert noalloc(seed, offset, ctypes.c_void_p(view.data_ptr()), n, lam, ctypes.c_void_p(stream)) == 0
        torch.cuda.synchronize()
        assert np.array_equal(view.cpu().numpy().view(np.uint32), ovals.view(np.uint32)), (seed, offset, lam)


def test_noalloc_inside_graph_capture(lib):
    """The call recorded by a CUDA graph capture: the launched graph equals the generator
    path, and still does after a direct call with another lambda has rewritten the shared
    array (the captured call carries its own table)."""
    import torch
    noalloc = _entry(lib)
    seed, n = 0xABCDEF, 50021
    want10 = _generator_values(lib, seed, [(n, 10.0)])[0]
    want500 = _generator_values(lib, seed, [(n, 500.0)])[0]
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    warm = torch.empty(16, dtype=torch.int32, device="cuda")
    # a first call on this device (looks up the array's address) before the capture
    assert noalloc(1, 0, ctypes.c_void_p(warm.data_ptr()), 16, 3.0,
                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        st = noalloc(seed, 0, ctypes.c_void_p(out.data_ptr()), n, 10.0,
                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want10)
    other = torch.empty(n, dtype=torch.int32, device="cuda")
    assert noalloc(seed, 0, ctypes.c_void_p(other.data_ptr()), n, 500.0,
                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)) == 0
    torch.cuda.synchronize()
    assert np.array_equal(other.cpu().numpy(), want500)
    out.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), want10)
    del graph


def test_noalloc_rejects_bad_lambda(lib):
    noalloc = _entry(lib)
    assert noalloc(1, 0, None, 10, 0.0, None) == rb.ROCRAND_STATUS_OUT_OF_RANGE
    assert noalloc(1, 0, None, 10, -3.0, None) == rb.ROCRAND_STATUS_OUT_OF_RANGE
    assert noalloc(1, 0, None, 10, float("nan"), None) == rb.ROCRAND_STATUS_OUT_OF_RANGE
