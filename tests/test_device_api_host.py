"""Device API functions evaluated on the host (nvcc-compiled host code, no GPU).

rocrand_kernel.h's functions are __host__ __device__.  The inversion Poisson sampler of the
quasi-random, ThreeFry and LFSR113 states is run here over lambdas that need one, two and
three rescaled segments (and the normal approximation above 1000): sample mean and variance
must match lambda.  (Between 500 and 1000 the reference's sampler does not terminate in
reasonable time, so this range is checked by statistics rather than against it.)
"""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_inversion_poisson_moments(tmp_path):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc absent")
    exe = str(tmp_path / "host_check")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "devapi", "host_check.cu"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    n = 200000
    for line in out.splitlines():
        lam, mean, var = map(float, line.split())
        # mean within 5 standard errors, variance within 3 %
        assert abs(mean - lam) < 5 * (lam / n) ** 0.5, (lam, mean)
        assert abs(var / lam - 1.0) < 0.03, (lam, var)
