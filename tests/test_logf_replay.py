"""The host-logf replay table of the inverse-erf normal (rocrand_b200/csrc/logf_replay.cuh).

The build's generator (rocrand_b200/data/make_logf_replay.cpp) enumerates every argument
the Sobol fp32 normal can pass to logf, compares the host C library's logf with the
kernels' rounding of the accurate logarithm, and replays every argument through the
kernels' lookup code compiled for the host.  Rerunning it must report no mismatch and
write exactly the table embedded in librocrand.so.
"""

import os
import re
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "_build", "data")


def test_replay_table_reproduces_host_logf():
    gen = os.path.join(DATA, "make_logf_replay")
    built = os.path.join(DATA, "logf_replay.bin")
    if not os.path.exists(gen):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "rocrand_b200", "csrc")])
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "logf_replay.bin")
        res = subprocess.run([gen, out], capture_output=True, text=True, check=True)
        m = re.search(r"(\d+) reachable arguments, (\d+) differ .* ([\d.]+)% looked up.* (\d+) mismatches",
                      res.stdout)
        assert m, res.stdout
        reachable, differ, looked, mismatches = int(m.group(1)), int(m.group(2)), float(m.group(3)), int(m.group(4))
        assert mismatches == 0
        assert reachable > 10_000_000 and 0 < differ < reachable // 50
        assert looked < 10.0
        with open(out, "rb") as a, open(built, "rb") as b:
            assert a.read() == b.read(), "the embedded table differs from a fresh run"
