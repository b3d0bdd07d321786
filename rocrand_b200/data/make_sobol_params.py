"""Recovers the Sobol direction-number parameters and writes sobol_params.bin.

The library computes every Sobol direction-vector table (32/64-bit, plain/scrambled) from
the Joe-Kuo parameters of each dimension: the degree s and coefficients a of its primitive
polynomial and the initial direction numbers m_1..m_s.  Those parameters are the published
"new-joe-kuo-6.21201" set (S. Joe and F. Y. Kuo, 2008); the reference ships them only
expanded, as the 32-bit table library/src/rocrand_sobol32_precomputed.bin.  This script
inverts that table once:

  * dimension 0 is the identity table (v_j = 2^(31-j));
  * dimension d >= 1 uses the next primitive polynomial in (s, a) order, so candidates are
    scanned forward from the previous dimension's (s, a); m_j = v_j >> (31 - j) for j < s,
    and a candidate is accepted when the Joe-Kuo recurrence
        v_j = v_{j-s} ^ (v_{j-s} >> s) ^ XOR_{k=1..s-1} a_k v_{j-k}
    regenerates all 32 vectors of the dimension;
  * the whole 32-bit table is then regenerated from the recovered parameters and compared
    byte for byte with the reference file before anything is written.

Output format (little-endian bit stream, LSB first): magic "RBSOBOL1", uint32 dimension count
(20000, dimension 0 included with s = 0), then per dimension d >= 1: s (5 bits), a (s-1 bits),
m_j (j+1 bits each, j = 0..s-1).

Usage (in a checkout that has the reference sources):
    python rocrand_b200/data/make_sobol_params.py <reference>/library/src/rocrand_sobol32_precomputed.bin
"""

import os
import struct
import sys

import numpy as np

DIMS = 20000
HERE = os.path.dirname(os.path.abspath(__file__))


def vectors32(s, a, m):
    v = [0] * 32
    for j in range(s):
        v[j] = m[j] << (31 - j)
    for j in range(s, 32):
        x = v[j - s] ^ (v[j - s] >> s)
        for k in range(1, s):
            if (a >> (s - 1 - k)) & 1:
                x ^= v[j - k]
        v[j] = x & 0xFFFFFFFF
    return v


def matches(s, a, want):
    m = [want[j] >> (31 - j) for j in range(s)]
    if any((mj & 1) == 0 or mj >= (1 << (j + 1)) for j, mj in enumerate(m)):
        return None
    for j in range(s):
        if (m[j] << (31 - j)) != want[j]:
            return None
    v = list(want[:s])
    for j in range(s, 32):
        x = v[j - s] ^ (v[j - s] >> s)
        for k in range(1, s):
            if (a >> (s - 1 - k)) & 1:
                x ^= v[j - k]
        if x != want[j]:
            return None
        v.append(x)
    return m


def recover(table):
    params = [None]
    s, a = 1, -1
    for d in range(1, DIMS):
        want = [int(x) for x in table[d * 32:(d + 1) * 32]]
        while True:
            a += 1
            if a >= (1 << (s - 1)):
                s += 1
                a = 0
                if s > 18:
                    raise SystemExit("no parameters found for dimension %d" % d)
            m = matches(s, a, want)
            if m is not None:
                params.append((s, a, m))
                break
    return params


class BitWriter:
    def __init__(self):
        self.bits = []

    def put(self, value, n):
        for i in range(n):
            self.bits.append((value >> i) & 1)

    def bytes(self):
        out = bytearray((len(self.bits) + 7) // 8)
        for i, b in enumerate(self.bits):
            if b:
                out[i // 8] |= 1 << (i % 8)
        return bytes(out)


def main(argv):
    if len(argv) != 1:
        raise SystemExit(__doc__)
    table = np.fromfile(argv[0], dtype="<u4")
    assert table.size == DIMS * 32, table.size
    params = recover(table)
    regen = np.zeros(DIMS * 32, dtype=np.uint32)
    regen[:32] = [1 << (31 - j) for j in range(32)]
    for d in range(1, DIMS):
        regen[d * 32:(d + 1) * 32] = vectors32(*params[d])
    if not np.array_equal(regen, table):
        raise SystemExit("regenerated 32-bit table differs from the reference")
    w = BitWriter()
    for d in range(1, DIMS):
        s, a, m = params[d]
        w.put(s, 5)
        w.put(a, s - 1)
        for j, mj in enumerate(m):
            w.put(mj, j + 1)
    blob = b"RBSOBOL1" + struct.pack("<I", DIMS) + w.bytes()
    out = os.path.join(HERE, "sobol_params.bin")
    with open(out, "wb") as f:
        f.write(blob)
    print("wrote %s (%d bytes); max degree %d" % (out, len(blob), max(p[0] for p in params[1:])))


if __name__ == "__main__":
    main(sys.argv[1:])
