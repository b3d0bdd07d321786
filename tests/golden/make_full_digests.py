"""Records SHA-256 digests of full-size outputs of the reference's OWN host generators, for
the full-size GPU parity tests (tests/test_parity_gpu.py), in full_digests.json.

Run in the build container (needs oracle/_ref/librocrand_ref.so, which oracle/Makefile.ref
compiles from the reference sources):

    make -C oracle -f Makefile.ref && python tests/golden/make_full_digests.py

Each entry is one call on a fresh generator: the pseudo-random generators at 2^28 values
(seed 0xdeadbeef, offset 0 where the generator has offsets) and the quasi-random workload
(Sobol32 and scrambled Sobol64, 1, 64 and 1000 dimensions x 2^20 points at offset 4096).
Every digest is recorded from the reference and checked against the C oracle (liborc.so)
before it is written, so the file also pins the oracle at these sizes.
"""

import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import pyorc  # noqa: E402

PSEUDO = {"philox": 404, "threefry2x32": 408, "threefry2x64": 409, "threefry4x32": 410,
          "threefry4x64": 411, "xorwow": 401, "mrg32k3a": 402, "mrg31k3p": 405, "lfsr113": 406,
          "mt19937": 407, "mtgp32": 403}
NO_OFFSET = {"mt19937", "mtgp32"}
QUASI = {"sobol32": 501, "scrambled_sobol64": 505}
FULL_N = 1 << 28
QUASI_POINTS = 1 << 20
QUASI_OFFSET = 4096


def cases():
    # the small reference case: Philox4x32-10, seed 1234, uniform fp32, 2^24 values
    yield {"key": "philox/uniform/seed1234/2^24", "rng": PSEUDO["philox"], "seed": 1234, "offset": None,
           "dims": None, "call": ["uniform", 1 << 24, [], 0]}
    for name in sorted(PSEUDO):
        for dist in ("uniform", "uint"):
            yield {"key": "%s/%s/2^28" % (name, dist), "rng": PSEUDO[name], "seed": 0xdeadbeef,
                   "offset": None if name in NO_OFFSET else 0, "dims": None,
                   "call": [dist, FULL_N, [], 0]}
    for name in sorted(QUASI):
        for dims in (1, 64, 1000):
            for dist, params in (("uniform_double", []), ("normal", [0.0, 1.0])):
                yield {"key": "%s/%s/dims%d" % (name, dist, dims), "rng": QUASI[name], "seed": None,
                       "offset": QUASI_OFFSET, "dims": dims,
                       "call": [dist, dims * QUASI_POINTS, params, 0]}


def digest(lib, c):
    (st, vals), = pyorc.run_sequence(lib, c["rng"], c["seed"], c["offset"], [tuple(c["call"])],
                                     dims=c["dims"])
    assert st == 0, (c["key"], st)
    return hashlib.sha256(vals.view("u1").data).hexdigest()


def main(argv):
    ref = pyorc.CLib("ref")
    orc = pyorc.CLib("orc")
    path = os.path.join(HERE, "full_digests.json")
    out = {}
    if os.path.exists(path):
        with open(path) as f:
            out = json.load(f)
    for c in cases():
        if argv and not any(a in c["key"] for a in argv):
            continue
        d = digest(ref, c)
        # the C oracle must agree (it calls the same host libm for the normal transforms)
        assert digest(orc, c) == d, ("oracle differs from the reference", c["key"])
        entry = dict(c)
        entry["sha256"] = d
        out[c["key"]] = entry
        print(c["key"], d, flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
