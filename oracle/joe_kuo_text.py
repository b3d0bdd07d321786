"""Writes the recovered Sobol parameters (rocrand_b200/data/sobol_params.bin) in the Joe-Kuo
text format ("d s a m_1 .. m_s", one header line) that the reference's own table tools read
(tools/sobol_utils.hpp:55-70).  Used by Makefile.ref to rebuild the reference's missing
Sobol64 tables for oracle/_ref.  TEST INFRASTRUCTURE ONLY."""

import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(out_path):
    blob = open(os.path.join(HERE, "..", "rocrand_b200", "data", "sobol_params.bin"), "rb").read()
    assert blob[:8] == b"RBSOBOL1"
    dims = struct.unpack("<I", blob[8:12])[0]
    data = blob[12:]
    pos = 0

    def get(n):
        nonlocal pos
        v = 0
        for i in range(n):
            v |= ((data[pos // 8] >> (pos % 8)) & 1) << i
            pos += 1
        return v

    lines = ["d       s       a       m_i"]
    for d in range(1, dims):
        s = get(5)
        a = get(s - 1)
        m = [get(j + 1) for j in range(s)]
        lines.append(" ".join(str(x) for x in [d + 1, s, a] + m))
    # the tools read SOBOL_DIM entries; one spare line keeps the stream in a good state
    lines.append(" ".join(["0", "1", "0", "1"]))
    with open(out_path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
