"""Helpers of the GPU parity tests: device generation through the C ABI, comparison with
the oracle, ulp distances."""

import ctypes
import hashlib
from ctypes import c_size_t, c_void_p

import numpy as np

from oracle import pyorc

BIT_EXACT = {"uint", "ulonglong", "char", "short", "uniform", "uniform_double", "uniform_half",
             "poisson"}

# Sobol's fp32 normal (and its half form) is bit-exact too: its only transcendental, logf, is
# the host C library's own result (logf_replay.cuh), and every other step is IEEE.
SOBOL_EXACT = {"normal", "normal_half"}


def bit_exact(rng, dist):
    return dist in BIT_EXACT or (rng in SOBOL and dist in SOBOL_EXACT)


# Elements of fp64 outputs that are outside the forward ulp bound and were accepted by the
# backward-error rule of compare_call, per (rng, dist): [accepted elements, elements compared].
FP64_EXCEPTIONS = {}
FP64_EXCEPTION_RATE = 1e-4

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


def generate_into(lib, g, dist, buf, params=()):
    """One generate call writing buf (a contiguous torch tensor on the device); the status."""
    suffix = pyorc.DISTS[dist][0]
    fn = getattr(lib, "rocrand_" + suffix)
    return fn(g, c_void_p(buf.data_ptr()), c_size_t(buf.numel()), *pyorc.dist_args(dist, params))


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


def _ratios(dist, got, exp, params):
    """Per-element error / allowed error of one output against one expectation (0 where
    both are the same non-finite value, inf where only one is finite)."""
    tol = ULP_TOL[dist]
    mean = float(params[0]) if params else 0.0
    T = exp.dtype.type
    ratio = np.full(exp.shape, np.inf)
    same = (got.view(np.uint8).reshape(exp.size, -1) == exp.view(np.uint8).reshape(exp.size, -1)).all(axis=1)
    ratio[same] = 0.0
    fin = np.isfinite(exp) & np.isfinite(got) & ~same
    g, e = got[fin], exp[fin]

    def sp(x):  # ulp of |x| in the output precision, as float64
        return np.spacing(np.abs(x).astype(exp.dtype)).astype(np.float64)

    if not e.size:
        return ratio
    if dist.startswith("log_normal"):
        pos = (e > 0) & (g > 0)
        r = np.full(e.shape, np.inf)
        z = np.log(e[pos].astype(np.float64))
        err = np.abs(np.log(g[pos].astype(np.float64)) - z)
        lim = tol * sp(z - mean) + sp(z) + 2 * float(np.spacing(T(1)))
        r[pos] = err / lim
    else:
        err = np.abs(g.astype(np.float64) - e.astype(np.float64))
        lim = tol * sp(e.astype(np.float64) - mean) + (sp(e) if mean != 0.0 else 0.0)
        lim = np.maximum(lim, np.finfo(exp.dtype).smallest_subnormal)
        r = err / lim
    ratio[fin] = r
    return ratio


SOBOL = {501, 502, 504, 505}


def compare(dist, got, exp, params=(), alts=()):
    """Asserts parity of one output; returns the max ulp distance (0 for bit-exact).
    Elements outside the tolerance of `exp` may instead be within it of one of `alts`."""
    assert got.shape == exp.shape
    if dist in BIT_EXACT:
        if not np.array_equal(got.view(np.uint8), exp.view(np.uint8)):
            bad = np.nonzero(got.view(exp.dtype) != exp)[0]
            raise AssertionError("%s: %d mismatches, first at %s: got %r want %r" % (
                dist, bad.size, bad[:5], got[bad[:5]], exp[bad[:5]]))
        return 0
    if not exp.size:
        return 0
    ratio = _ratios(dist, got, exp, params)
    for alt in alts:
        ratio = np.minimum(ratio, _ratios(dist, got, alt, params))
    fin = np.isfinite(exp) & np.isfinite(got)
    worst_ulps = int(ulp_diff(got[fin], exp[fin]).max()) if fin.any() else 0
    if (ratio > 1.0).any():
        k = int(np.argmax(ratio))
        raise AssertionError("%s: %d outside tolerance, worst %.3g x limit at %d (got %r want %r); "
                             "max output ulp %d" % (dist, int((ratio > 1.0).sum()), ratio[k], k,
                                                    got[k], exp[k], worst_ulps))
    return worst_ulps




def erfinv_normal(rng, dist):
    """Whether the reference computes this normal / log-normal by its inverse-erf formula
    (Sobol: normal.hpp:272-330; ThreeFry2x32 fp64: threefry.hpp:441-449)."""
    if dist not in ULP_TOL:
        return False
    return rng in SOBOL or (rng == 408 and dist in ("normal_double", "log_normal_double"))


def libm_shifts(rng, dist):
    """(log, sin/cos) ulp shifts of the host library's fp64 results under which a device
    output may instead match the reference formula: the fp64 inverse-erf normal (log only)
    and the fp64 Box-Muller transforms (log and sin/cos).  fp32 outputs have none: they must
    meet the forward bound (or be bit-exact)."""
    if dist not in ("normal_double", "log_normal_double"):
        return []
    if erfinv_normal(rng, dist):
        return [(1, 0), (-1, 0)]
    return [(a, b) for a in (-1, 0, 1) for b in (-1, 0, 1) if (a, b) != (0, 0)]


def compare_call(orc, rng, seed, offset, dims, calls, k, got, exp):
    """Parity of call k of a sequence.  Bit-exact classes must be identical; fp32 and half
    normals and log-normals must meet the forward ulp bound.  fp64 normals and log-normals
    must meet it too, except for elements where the host library's own log/sin/cos result is
    not correctly rounded and the reference formula amplifies that: the fp64 inverse-erf
    normal (sqrt(-tt1 + sqrt(tt1^2 - tt2)), tt1 and tt2 linear in log(x), cancels: tens of
    ulps) and the fp64 Box-Muller products (one ulp of sin can be two of the output).  Such
    an element is accepted only if it is within the bound of the reference formula evaluated
    with glibc's results moved by one ulp (the oracle rerun with those values; every other
    operation is IEEE and identical), and it is counted in FP64_EXCEPTIONS."""
    dist, _, params, _ = calls[k]
    if bit_exact(rng, dist):
        return compare("uint" if dist not in BIT_EXACT else dist, got, exp, params)
    try:
        return compare(dist, got, exp, params)
    except AssertionError:
        shifts = libm_shifts(rng, dist)
        if not shifts:
            raise
    alts = []
    for lg, tr in shifts:
        orc.set_libm_ulps(lg, tr)
        try:
            alts.append(pyorc.run_sequence(orc, rng, seed, offset, calls[:k + 1], dims=dims)[k][1])
        finally:
            orc.set_libm_ulps(0, 0)
    worst = compare(dist, got, exp, params, alts)
    outside = int((_ratios(dist, got, exp, params) > 1.0).sum())
    acc = FP64_EXCEPTIONS.setdefault((rng, dist), [0, 0])
    acc[0] += outside
    acc[1] += int(exp.size)
    # the stated rate of such elements: at most FP64_EXCEPTION_RATE of a call (measured:
    # about 4e-6 for Box-Muller, 2e-5 to 4e-5 for the inverse-erf normal)
    assert outside <= max(2, FP64_EXCEPTION_RATE * exp.size), (rng, dist, outside, exp.size)
    return worst
