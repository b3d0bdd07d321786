"""The reference's own Python binding against this library.

The binding (python/rocrand/rocrand/rocrand.py) loads librocrand.so by ctypes from
ROCRAND_PATH and the CUDA runtime from CUDA_PATH (python/rocrand/rocrand/hip.py:66-92), so
pointing ROCRAND_PATH at this package makes it drive this library unchanged.  The host-side
cases of the reference's Python suite (python/rocrand/tests/rocrand_test.py:36-185: version,
constructors of every generator type, seed / offset / ndim setters and the errors they must
raise, e.g. an offset on MT19937 or MTGP32) run here as written.  Its generate cases allocate
device memory and are not run on a machine without a GPU; the binding exists only where the
reference tree does, so the whole module is skipped without it.
"""

import json
import os
import subprocess
import sys

import pytest

REFERENCE = os.environ.get("ROCRAND_REFERENCE", "/root/reference")
BINDING = os.path.join(REFERENCE, "python", "rocrand")
SUITE = os.path.join(BINDING, "tests", "rocrand_test.py")
PACKAGE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rocrand_b200")

RUNNER = r"""
import importlib.util, json, sys, unittest
sys.path.insert(0, sys.argv[1])
spec = importlib.util.spec_from_file_location("rocrand_test", sys.argv[2])
m = importlib.util.module_from_spec(spec)
spec.loader.exec_module(m)
import rocrand.rocrand as binding
suite = unittest.TestSuite()
for name in sorted(dir(m)):
    obj = getattr(m, name)
    if isinstance(obj, type) and issubclass(obj, unittest.TestCase) and not name.startswith("TestGenerate"):
        suite.addTests(unittest.TestLoader().loadTestsFromTestCase(obj))
r = unittest.TextTestRunner(stream=sys.stderr, verbosity=0).run(suite)
print(json.dumps({"ran": r.testsRun, "skipped": len(r.skipped),
                  "failed": [str(t) for t, _ in r.failures + r.errors],
                  "library": binding.rocrand._name}))
"""


@pytest.mark.skipif(not os.path.exists(SUITE), reason="the reference's Python binding is not present")
def test_reference_python_suite_host_cases(lib):
    env = dict(os.environ, ROCRAND_PATH=PACKAGE, CUDA_PATH=os.environ.get("CUDA_PATH", "/usr/local/cuda"))
    p = subprocess.run([sys.executable, "-c", RUNNER, BINDING, SUITE], env=env, capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    # the binding loaded this library, not another librocrand.so
    assert os.path.realpath(res["library"]) == os.path.realpath(os.path.join(PACKAGE, "librocrand.so"))
    assert not res["failed"], res["failed"]
    # the version case, the invalid-type case, and 17 generator types (10 PRNG, 2 MT, 5 QRNG)
    # each in a constructor class and a parameter class
    assert res["ran"] - res["skipped"] >= 1 + 1 + 2 * (10 + 2 + 5)


CPP_CHECK = os.path.join(os.path.dirname(os.path.abspath(__file__)), "wrapper", "cpp_wrapper_check.cu")
CPP_WRAPPER = os.path.join(REFERENCE, "library", "include", "rocrand", "rocrand.hpp")


@pytest.mark.skipif(not os.path.exists(CPP_WRAPPER), reason="the reference's C++ wrapper is not present")
def test_reference_cpp_wrapper_builds_against_this_library(tmp_path, lib):
    """Every engine and distribution class of the reference's C++ wrapper compiles on this
    library's rocrand.h / rocrand_kernel.h and links against librocrand.so with no undefined
    symbol (library/include/rocrand/rocrand.hpp:139-3738)."""
    include = os.path.join(os.path.dirname(PACKAGE), "include")
    exe = str(tmp_path / "cpp_wrapper_check")
    cmd = ["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", include, "-I", os.path.join(REFERENCE, "library", "include"), "-Xcompiler", "-H",
           "-o", exe, CPP_CHECK, "-L", PACKAGE, "-lrocrand", "-Xlinker", "--no-undefined"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    assert os.path.exists(exe)
    # the wrapper came from the reference, every rocrand header it pulls in from this library
    included = [ln.lstrip(". ").strip() for ln in p.stderr.splitlines() if ln.startswith(".")]
    ours = [h for h in included if "rocrand" in os.path.basename(h) and not h.endswith("rocrand.hpp")]
    assert ours and all(os.path.realpath(h).startswith(os.path.realpath(include)) for h in ours), ours
