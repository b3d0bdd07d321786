"""Accuracy of the fp64 log / sincos used by the normal and log-normal transforms.

rocrand_b200/csrc/precise_math.cuh is compiled for the host (the same IEEE operations as on
the device) and measured against binary128 on 3*10^5 inputs of each kind: the Box-Muller
logarithm inputs (k+1) 2^-53, general normal numbers, and angles w*pi for w = k 2^-52.  The
results must be correctly rounded except in rare near-halfway cases (error <= 0.5 ulp plus
the internal 2^-66 error; glibc's functions, measured beside them, miss correct rounding
about a hundred times more often), and the special values must match the C library.
"""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def report(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    inc = os.path.join(ROOT, "_build", "data", "precise_tables.inc")
    if not os.path.exists(inc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "rocrand_b200", "csrc"), "../../_build/data/precise_tables.inc"],
                       check=True, capture_output=True)
    exe = str(tmp_path_factory.mktemp("pm") / "check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                    "-I", os.path.join(ROOT, "rocrand_b200", "csrc"), "-I", os.path.join(ROOT, "_build", "data"),
                    os.path.join(HERE, "precise_math_check.cpp"), "-o", exe, "-lquadmath"], check=True)
    out = subprocess.run([exe, "300000"], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.splitlines():
        k, *v = line.split()
        rows.setdefault(k, []).append(v)
    return rows


def test_log_sin_cos_nearly_correctly_rounded(report):
    for name, allowed in (("log", 3), ("log_near", 3), ("sin", 30), ("cos", 30), ("logf", 3)):
        err, miss, n = report[name][0]
        assert float(err) <= 0.5 + 2.0 ** -10, (name, err)
        assert int(miss) <= allowed, (name, miss, n)
    # the C library's own functions for comparison: far more often off correct rounding
    assert int(report["glibc_log"][0][1]) > int(report["log"][0][1])
    assert int(report["glibc_sin"][0][1]) > int(report["sin"][0][1])


def test_special_values(report):
    assert all(v[1] == "1" for v in report["special"]), report["special"]
