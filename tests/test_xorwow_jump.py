"""The XORWOW jump polynomials of the seeding kernels, checked on the CPU.

Engine e of a fresh XORWOW generator is the base state moved by e subsequences of 2^67 steps
(xorwow.hpp:45-61).  The library seeds it as window sums of the base's word sequence over
the set coefficients of a build-time polynomial p_e (rocrand_b200/data/make_xorwow_jump.c).
Here p_e is applied to random states and compared with J^e computed independently: the
160 x 160 GF(2) matrix of one step, squared 67 times, raised to e by squaring (numpy).
"""

import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TABLE = os.path.join(ROOT, "_build", "data", "xorwow_jump.bin")
ENGINES = 131072


def _step(x):
    x = [int(v) for v in x]
    t = x[0] ^ (x[0] >> 2)
    return x[1:] + [((x[4] ^ (x[4] << 4)) ^ (t ^ (t << 1))) & 0xFFFFFFFF]


def _bits(x):
    return np.array([(x[i // 32] >> (i % 32)) & 1 for i in range(160)], dtype=np.uint8)


def _words(b):
    return [int(sum(int(b[32 * w + i]) << i for i in range(32))) for w in range(5)]


def _matrix():
    """Column i = image of input bit i under one xorshift step."""
    m = np.zeros((160, 160), dtype=np.uint8)
    for i in range(160):
        x = [0] * 5
        x[i // 32] = 1 << (i % 32)
        m[:, i] = _bits(_step(x))
    return m


def _mul(a, b):
    return (a.astype(np.int64) @ b.astype(np.int64) % 2).astype(np.uint8)


@pytest.fixture(scope="module")
def table():
    if not os.path.exists(TABLE):
        subprocess.run(["make", "-C", os.path.join(ROOT, "rocrand_b200", "csrc"), "../../_build/data/xorwow_jump.bin"],
                       check=True, capture_output=True)
    t = np.fromfile(TABLE, dtype=np.uint32)
    assert t.size == 5 * ENGINES
    return t.reshape(5, ENGINES)


def test_polynomials_equal_matrix_jumps(table):
    j = _matrix()
    for _ in range(67):
        j = _mul(j, j)
    rng = np.random.default_rng(2024)
    for e in [0, 1, 2, 63, 64, 4097, 99991, ENGINES - 1]:
        s = [int(v) for v in rng.integers(0, 2**32, 5)]
        # J^e s
        want, p, k = _bits(s), j, e
        while k:
            if k & 1:
                want = (p.astype(np.int64) @ want.astype(np.int64) % 2).astype(np.uint8)
            k >>= 1
            if k:
                p = _mul(p, p)
        # window sums of the word sequence over the set coefficients of p_e
        seq, x = list(s), list(s)
        while len(seq) < 164:
            x = _step(x)
            seq.append(x[4])
        coeff = [(int(table[k // 32, e]) >> (k % 32)) & 1 for k in range(160)]
        got = [0] * 5
        for k in range(160):
            if coeff[k]:
                for w in range(5):
                    got[w] ^= seq[k + w]
        assert got == _words(want), e
