"""Writes mtgp32_params.bin: the MTGP32 parameter sets of the 512 generators.

MTGP32 (M. Saito and M. Matsumoto, "Variants of Mersenne Twister Suitable for Graphic
Processors", 2013) gives every block its own recurrence, found by the MTGP dynamic creator.
The 512 sets for Mersenne exponent 11213 are published with the MTGP distribution
(mtgp32dc-param-11213) and vendored by the reference as the initialiser
mtgp32dc_params_fast_11213 in library/include/rocrand/rocrand_mtgp32_11213.h.  They define
the streams, so the library needs them verbatim; this script reads the numbers out of that
header once and stores them in binary form, checking on the way that each set is what the
recurrence needs (mexp 11213, the 16-entry tables spanned by their entries 1, 2, 4 and 8,
one common state mask).

Output (little-endian uint32): magic "RBMTGP01" (8 bytes), count (512), then per set:
pos, sh1, sh2, tbl[16], tmp_tbl[16], mask -- 36 words.  (The float tempering table is not
used by the host API's integer path.)

Usage (in a checkout that has the reference sources):
    python rocrand_b200/data/make_mtgp32_params.py \\
        /root/reference/library/include/rocrand/rocrand_mtgp32_11213.h
"""

import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
COUNT = 512


def parse(text):
    body = text[text.index("mtgp32dc_params_fast_11213[]"):]
    body = body[body.index("{") + 1:]
    body = re.sub(r"/\*.*?\*/", " ", body, flags=re.S)  # drop comments ("No.0 delta:...")
    # every set: mexp, pos, sh1, sh2, {16}, {16}, {16}, mask, {21 bytes}
    sets = []
    tok = re.findall(r"UINT32_C\((0x[0-9a-fA-F]+)\)|(0x[0-9a-fA-F]+|\d+)|([{}])", body)
    depth, cur, group, groups = 0, [], None, []
    for u32, num, brace in tok:
        if brace == "{":
            depth += 1
            if depth == 2:
                group = []
            continue
        if brace == "}":
            if depth == 2:
                cur.append(group)
                group = None
            elif depth == 1:
                sets.append(cur)
                cur = []
                if len(sets) == COUNT:
                    break
            depth -= 1
            if depth < 0:
                break
            continue
        value = int(u32 or num, 0)
        if depth == 1:
            cur.append(value)
        elif depth == 2:
            group.append(value)
    return sets


def main(argv):
    src = argv[0] if argv else "/root/reference/library/include/rocrand/rocrand_mtgp32_11213.h"
    with open(src) as f:
        sets = parse(f.read())
    assert len(sets) == COUNT, len(sets)
    out = bytearray(b"RBMTGP01") + struct.pack("<I", COUNT)
    mask0 = None
    for k, s in enumerate(sets):
        mexp, pos, sh1, sh2, tbl, tmp_tbl, flt_tbl, mask, sha = s
        assert mexp == 11213 and len(tbl) == len(tmp_tbl) == 16 and len(sha) == 21, k
        for t in (tbl, tmp_tbl):
            for i in range(16):
                acc = 0
                for b in range(4):
                    if i >> b & 1:
                        acc ^= t[1 << b]
                assert acc == t[i], (k, i)
        mask0 = mask if mask0 is None else mask0
        assert mask == mask0, k
        out += struct.pack("<3I", pos, sh1, sh2)
        out += struct.pack("<16I", *tbl) + struct.pack("<16I", *tmp_tbl) + struct.pack("<I", mask)
    dst = os.path.join(HERE, "mtgp32_params.bin")
    with open(dst, "wb") as f:
        f.write(out)
    print("wrote", dst, len(out), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:])
