"""Generates the golden fixtures of tests/golden/ from the reference's OWN host generators.

Run in the build container (needs oracle/_ref/librocrand_ref.so, which oracle/Makefile.ref
compiles from the reference sources):

    make -C oracle -f Makefile.ref && python tests/golden/make_golden.py [rng ...]

For every case (generator, seed, offset, call sequence) it records each call's status, the
SHA-256 of its output bytes and the first values, in golden_<rng>.json.  The tests replay
the same sequences through the C oracle (liborc.so) and require identical hashes: that pins
the oracle to the reference.  The GPU tests then compare the CUDA library with the oracle.
"""

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import pyorc  # noqa: E402
from tests.golden.cases import CASES  # noqa: E402

PREFIX_VALUES = 16


def record(lib, case):
    outs = pyorc.run_sequence(lib, case["rng"], case.get("seed"), case.get("offset"),
                              [tuple(c) for c in case["calls"]], dims=case.get("dims"))
    res = []
    for st, vals in outs:
        raw = vals.view(np.uint8).tobytes()
        res.append({
            "status": int(st),
            "sha256": hashlib.sha256(raw).hexdigest(),
            "prefix_bits": [int(x) for x in vals.view(_uint_of(vals.dtype))[:PREFIX_VALUES]],
        })
    return res


def _uint_of(dt):
    return {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[np.dtype(dt).itemsize]


def main(argv):
    ref = pyorc.CLib("ref")
    names = argv or sorted(CASES)
    for name in names:
        out = []
        for case in CASES[name]:
            c = dict(case)
            c["results"] = record(ref, case)
            out.append(c)
        path = os.path.join(HERE, "golden_%s.json" % name)
        with open(path, "w") as f:
            json.dump(out, f, indent=0, sort_keys=True)
        print("wrote", path, len(out), "cases")


if __name__ == "__main__":
    main(sys.argv[1:])
