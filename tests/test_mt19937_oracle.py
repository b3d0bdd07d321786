"""MT19937 pins that do not depend on the reference's host code (CPU only).

* The jump polynomials derived at build time (rocrand_b200/data/make_mt19937_jump.c) equal the
  list the reference ships (tools/mt19937_precomputed_source.zip, extracted by
  oracle/Makefile.ref into oracle/_ref/gen), when that extraction is present.
* Generator 0 of the oracle is the unjumped seed state, so its eight lanes must reproduce the
  textbook MT19937 sequence of the Knuth-initialised state of (seed >> 32) ^ seed, word by
  word in the octo-lane order of mt19937_octo_engine.hpp -- an independent check of the
  twist and of the output order, written here in plain Python.
"""

import os

import numpy as np
import pytest

from oracle import pyorc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRIDE = 65536
SINGLE = [0, 113, 170, 283, 340, 397, 510, 567]
GROUP = [1, 57, 114, 171, 227, 284, 341, 398, 454, 511, 568]


def _slot_word(lane, slot):
    if slot == 0:
        return SINGLE[lane]
    i, j = divmod(slot - 1, 7)
    return GROUP[i] + 7 * lane + j


def _textbook_states(seed, rounds):
    mt = [0] * 624
    mt[0] = ((seed >> 32) ^ seed) & 0xFFFFFFFF
    for i in range(1, 624):
        mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
    out = []
    for _ in range(rounds):
        for i in range(624):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
            mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
        out.append(list(mt))
    return out


def _temper(y):
    y ^= y >> 11
    y ^= (y << 7) & 0x9D2C5680
    y ^= (y << 15) & 0xEFC60000
    y ^= y >> 18
    return y


def test_generator0_is_textbook_mt19937(orc):
    seed, rounds = 0x1234567890ABCDEF, 3
    n = STRIDE * 78 * rounds
    st, vals = pyorc.run_sequence(orc, 407, seed, None, [("uint", n, (), 0)])[0]
    assert st == 0
    states = _textbook_states(seed, rounds)
    for r in range(rounds):
        for slot in range(78):
            base = r * STRIDE * 78 + slot * STRIDE
            got = [int(v) for v in vals[base:base + 8]]
            want = [_temper(states[r][_slot_word(lane, slot)]) for lane in range(8)]
            assert got == want, (r, slot)


def test_lane_slots_cover_the_state_once():
    words = sorted(_slot_word(lane, slot) for lane in range(8) for slot in range(78))
    assert words == list(range(624))


def test_jump_polynomials_equal_reference_list():
    clist = os.path.join(ROOT, "oracle", "_ref", "gen", "clist_mt19937.txt")
    table = os.path.join(ROOT, "_build", "data", "mt19937_jump.bin")
    if not (os.path.exists(clist) and os.path.exists(table)):
        pytest.skip("reference polynomial list or build output not present")
    mexp = 19937
    with open(clist) as f:
        text = f.read().strip()
    mine = np.fromfile(table, dtype="<u4").reshape(-1, 624)
    assert mine.shape[0] == 255 + 31
    for digit, count in ((0, 255), (1, 31)):
        for i in range(1, count + 1):
            s = text[(digit * 255 + i - 1) * mexp:(digit * 255 + i) * mexp]
            coef = np.frombuffer(s.encode(), dtype=np.uint8)[::-1] - 48  # char k = x^(mexp-1-k)
            bits = np.zeros(624 * 32, dtype=np.uint8)
            bits[:mexp] = coef
            words = np.packbits(bits.reshape(-1, 32)[:, ::-1], axis=1).view(">u4").ravel()
            row = mine[i - 1] if digit == 0 else mine[255 + i - 1]
            assert np.array_equal(words, row), (digit, i)
