"""The integer form of the Poisson alias-table test equals the reference's double form.

The kernels pick entry i = (size r) >> 32 and keep it when the low word of size r is below
ceil(prob[i] 2^32) (rocrand_b200/csrc/poisson.hpp alias_threshold); the reference computes
x = r 2^-32, nx = size x, i = floor(nx), y = nx - i and keeps i when y < prob[i]
(rocrand_discrete.h:38-63).  Checked here in IEEE double (numpy) on random and adversarial
inputs: thresholds at, just above and just below representable boundaries.
"""

import math

import numpy as np


def threshold(prob):
    return 1 << 32 if prob >= 1.0 else math.ceil(math.ldexp(prob, 32))


def test_integer_pick_equals_double_pick():
    rng = np.random.default_rng(7)
    inv32 = np.float64(2.3283064365386963e-10)
    for _ in range(20000):
        size = int(rng.integers(1, 4097))
        r = int(rng.integers(0, 2 ** 32))
        x = np.float64(r) * inv32
        nx = np.float64(size) * x
        fnx = np.floor(nx)
        y = nx - fnx
        i = int(fnx)
        # thresholds of several kinds: random, exactly at y, one ulp either side, 0 and 1
        cands = [float(rng.random()), float(y), float(np.nextafter(y, 2.0)), float(np.nextafter(y, -1.0)),
                 0.0, 1.0]
        p = (size * r)
        assert i == p >> 32
        lo = p & 0xFFFFFFFF
        for prob in cands:
            if not (0.0 <= prob <= 1.0):
                continue
            assert (y < prob) == (lo < threshold(prob)), (size, r, prob)
