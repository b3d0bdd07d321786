"""The C oracle (liborc.so) against the golden fixtures recorded from the reference's own
host generators (tests/golden/make_golden.py).  CPU only."""

import glob
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import pyorc

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "golden_*.json")))


def _cases():
    for path in FIXTURES:
        name = os.path.basename(path)[len("golden_"):-len(".json")]
        with open(path) as f:
            for i, case in enumerate(json.load(f)):
                yield pytest.param(case, id="%s-%d" % (name, i))


@pytest.mark.parametrize("case", list(_cases()))
def test_oracle_matches_reference_fixture(orc, case):
    outs = pyorc.run_sequence(orc, case["rng"], case.get("seed"), case.get("offset"),
                              [tuple(c) for c in case["calls"]], dims=case.get("dims"))
    for k, ((st, vals), exp) in enumerate(zip(outs, case["results"])):
        assert st == exp["status"], "call %d status" % k
        bits = vals.view({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[vals.itemsize])
        assert [int(x) for x in bits[:len(exp["prefix_bits"])]] == exp["prefix_bits"], "call %d prefix" % k
        assert hashlib.sha256(vals.view(np.uint8).tobytes()).hexdigest() == exp["sha256"], "call %d" % k


def test_fixtures_present():
    assert any("golden_philox" in p for p in FIXTURES)


def test_half_conversion_matches_numpy():
    """orc_float_to_half must round to nearest even like numpy's float16 cast."""
    import ctypes
    lib = pyorc.CLib("orc").lib
    lib.orc_float_to_half.argtypes = [ctypes.c_float]
    lib.orc_float_to_half.restype = ctypes.c_uint16
    rng = np.random.default_rng(5)
    vals = np.concatenate([
        rng.standard_normal(2000).astype(np.float32) * 10,
        (rng.random(2000) * 1e-4).astype(np.float32),  # subnormal halves
        np.array([65504, 65519, 65520, 1e6, -0.0, 0.0, 2 ** -24, 2 ** -25, 3 * 2 ** -26], np.float32),
    ])
    got = np.array([lib.orc_float_to_half(float(v)) for v in vals], dtype=np.uint16)
    exp = vals.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, exp)


def test_reference_constants_are_powers_of_two():
    """The uniform conversions are exact only because these literals round to 2^-k."""
    assert np.float32(2.3283064e-10) == np.float32(2.0 ** -32)
    assert np.float32(1.5258789e-05) == np.float32(2.0 ** -16)
    assert np.float64(1.1102230246251565e-16) == 2.0 ** -53
    assert np.float64(2.3283064365386963e-10) == 2.0 ** -32


def test_poisson_table_is_distribution(orc):
    import ctypes
    lib = orc.lib
    lib.orc_poisson_table.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_uint)]
    lib.orc_poisson_table.restype = ctypes.c_uint
    lib.orc_poisson_capacity.argtypes = [ctypes.c_double]
    lib.orc_poisson_capacity.restype = ctypes.c_uint
    for lam in (0.5, 4.0, 10.0, 1000.0, 4000.0):
        cap = lib.orc_poisson_capacity(lam)
        prob = np.zeros(cap)
        alias = np.zeros(cap, np.uint32)
        off = ctypes.c_uint(0)
        size = lib.orc_poisson_table(lam, prob.ctypes.data, alias.ctypes.data, ctypes.byref(off))
        assert 0 < size <= cap
        # the alias table reproduces the probabilities: P(k) = (prob_k + sum_{alias_j=k}(1-prob_j))/size
        p = prob[:size].copy()
        for j in range(size):
            if prob[j] < 1.0:
                p[alias[j]] += 1.0 - prob[j]
        p /= size
        k = np.arange(size) + off.value
        mean = float((p * k).sum())
        assert abs(mean - lam) < 1e-6 * max(1.0, lam)
