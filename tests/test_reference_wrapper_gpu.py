"""The reference's C++ wrapper (rocrand.hpp) driving this library on the GPU.

oracle/Makefile.ref wrapper builds tests/wrapper/cpp_wrapper_check.cu against the
reference's own rocrand.hpp (read in place where the reference is mounted; the binary is test
infrastructure under oracle/_ref).  Every engine x distribution object of the wrapper fills
device memory, and the same call made directly through this library's C ABI, on a generator
seeded as the wrapper seeds it, must give the same bytes (the 64-bit quasi-random engines may
refuse 32-bit integers with ROCRAND_STATUS_TYPE_ERROR, as the reference's do).
"""

import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "wrapper", "cpp_wrapper_check")
ENGINES = ["philox4x32_10", "xorwow", "mrg31k3p", "mrg32k3a", "mtgp32", "lfsr113", "mt19937",
           "threefry2x32", "threefry2x64", "threefry4x32", "threefry4x64", "sobol32",
           "scrambled_sobol32"]
DISTS = ["uint", "uniform_float", "uniform_double", "normal_float", "log_normal_double", "poisson"]


@pytest.mark.skipif(not os.path.exists(EXE), reason="the wrapper check was not built (needs the reference)")
def test_cpp_wrapper_equals_c_abi(lib):
    env = dict(os.environ, LD_LIBRARY_PATH=os.path.join(ROOT, "rocrand_b200"))
    p = subprocess.run([EXE], capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    lines = p.stdout.splitlines()
    assert not [ln for ln in lines if "MISMATCH" in ln or "C-ABI-ERROR" in ln or "failed" in ln], lines
    ok = {tuple(ln.split()[:2]) for ln in lines if ln.endswith(" OK")}
    for e in ENGINES:
        for d in DISTS:
            assert (e, d) in ok, (e, d)
    # the 64-bit quasi-random engines: each distribution byte-equal to the C ABI, or the
    # wrapper's error for 32-bit integers from a 64-bit engine (TYPE_ERROR, as in the reference)
    for e in ("sobol64", "scrambled_sobol64"):
        mine = [ln for ln in lines if ln.startswith(e + " ")]
        assert mine, lines
        assert all(ln.endswith(" OK") or ln.startswith(e + " error 103") for ln in mine), mine
