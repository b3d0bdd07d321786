"""Helpers of the GPU parity tests: device generation through the C ABI, comparison with
the oracle, ulp distances."""

import ctypes
import hashlib
from ctypes import c_size_t, c_void_p

import numpy as np

from oracle import pyorc

BIT_EXACT = {"uint", "ulonglong", "char", "short", "uniform", "uniform_double", "uniform_half",
             "poisson"}

# ulp tolerances of the floating-point distributions against the host oracle (glibc libm).
# They bound the error of the deviate the library computes, stddev * N, in ulps of that
# deviate: <= 4 ulp for fp32, <= 2 ulp for fp64, <= 1 ulp for half (rounded from fp32).
#  * normal = mean + stddev*N: allowed |got - exp| = tol * ulp(stddev*N) (+ 1 ulp of the
#    output for the final add when mean != 0, where cancellation makes output ulps
#    meaningless).  With mean 0 this is exactly "<= tol ulp of the output".
#  * log-normal = exp(z), z = mean + stddev*N: compared in the log domain,
#    |ln got - ln exp| <= tol * ulp(stddev*N) + ulp(z) + 2 ulp(1) (exp's own rounding),
#    because an ulp of z moves exp(z) by |z| output ulps.
ULP_TOL = {"normal": 4, "normal_double": 2, "normal_half": 1,
           "log_normal": 4, "log_normal_double": 2, "log_normal_half": 1}


def torch_dtype(dist):
    import torch
    dt = pyorc.DISTS[dist][1]
    return {np.uint32: torch.int32, np.uint64: torch.int64, np.uint8: torch.uint8,
            np.uint16: torch.int16, np.float32: torch.float32, np.float64: torch.float64,
            np.float16: torch.float16}[dt]


def device_generate(lib, g, dist, n, params=(), mis=0):
    """One generate call into device memory placed (mis * itemsize) bytes past a 512-byte
    boundary (the caching allocator's alignment), which matches the host placement of the
    oracle ((mis * itemsize) mod 64 past a 64-byte boundary) for mis * itemsize < 64;
    returns (status, numpy values)."""
    import torch
    suffix, dt, _ = pyorc.DISTS[dist]
    isz = np.dtype(dt).itemsize
    buf = torch.empty(n + 64 // isz + 16, dtype=torch_dtype(dist), device="cuda")
    view = buf[mis:mis + n]
    fn = getattr(lib, "rocrand_" + suffix)
    st = fn(g, c_void_p(view.data_ptr()), c_size_t(n), *pyorc.dist_args(dist, params))
    torch.cuda.synchronize()
    return st, view.cpu().numpy().view(dt)


def create(lib, rng, seed=None, offset=None, dims=None):
    g = c_void_p()
    st = lib.rocrand_create_generator(ctypes.byref(g), rng)
    assert st == 0, st
    if seed is not None:
        assert lib.rocrand_set_seed(g, seed) == 0
    if dims is not None:
        assert lib.rocrand_set_quasi_random_generator_dimensions(g, dims) == 0
    if offset is not None:
        assert lib.rocrand_set_offset(g, offset) == 0
    return g


def sha(vals):
    return hashlib.sha256(vals.view(np.uint8).tobytes()).hexdigest()


def _mono(a):
    bits = {2: np.int16, 4: np.int32, 8: np.int64}[a.itemsize]
    i = a.view(bits).astype(np.int64)
    mask = (1 << (8 * a.itemsize - 1)) - 1
    return np.where(i < 0, -(i & mask), i)


def ulp_diff(a, b):
    """Element-wise distance in units in the last place (same dtype arrays)."""
    return np.abs(_mono(a) - _mono(b))


def compare(dist, got, exp, params=()):
    """Asserts parity of one output; returns the max ulp distance (0 for bit-exact)."""
    assert got.shape == exp.shape
    if dist in BIT_EXACT:
        if not np.array_equal(got.view(np.uint8), exp.view(np.uint8)):
            bad = np.nonzero(got.view(exp.dtype) != exp)[0]
            raise AssertionError("%s: %d mismatches, first at %s: got %r want %r" % (
                dist, bad.size, bad[:5], got[bad[:5]], exp[bad[:5]]))
        return 0
    same_nonfinite = np.isfinite(got) == np.isfinite(exp)
    assert same_nonfinite.all(), "%s: finite/non-finite mismatch" % dist
    fin = np.isfinite(exp) & np.isfinite(got)
    g, e = got[fin], exp[fin]
    if not e.size:
        return 0
    tol = ULP_TOL[dist]
    mean = float(params[0]) if params else 0.0
    T = e.dtype.type

    def sp(x):  # ulp of |x| in the output precision, as float64
        return np.spacing(np.abs(x).astype(e.dtype)).astype(np.float64)

    if dist.startswith("log_normal"):
        pos = (e > 0) & (g > 0)
        assert pos.all() or np.array_equal(g[~pos], e[~pos]), "%s: sign/zero mismatch" % dist
        z = np.log(e[pos].astype(np.float64))
        err = np.abs(np.log(g[pos].astype(np.float64)) - z)
        lim = tol * sp(z - mean) + sp(z) + 2 * float(np.spacing(T(1)))
        ratio = err / lim
        worst_ulps = int(ulp_diff(g, e).max())
    else:
        err = np.abs(g.astype(np.float64) - e.astype(np.float64))
        lim = tol * sp(e.astype(np.float64) - mean) + (sp(e) if mean != 0.0 else 0.0)
        lim = np.maximum(lim, np.finfo(e.dtype).smallest_subnormal)
        ratio = err / lim
        worst_ulps = int(ulp_diff(g, e).max())
    if ratio.size and (ratio > 1.0).any():
        k = int(np.argmax(ratio))
        raise AssertionError("%s: error %.3g > limit %.3g at %d (got %r want %r); max output ulp %d" % (
            dist, err[k], lim[k], k, g[k], e[k], worst_ulps))
    return worst_ulps
