"""The serving loop's host-side policies, run on the host: admission
(rocrand_b200/csrc/admission.hpp) and the output pool's allocator
(rocrand_b200/csrc/pool_allocator.hpp).

tests/admission_check.cpp drives random queues of requests on stateful and stateless
handles through the policy, with random batch limits and output budgets, and compares every
admission with a plain scan of the whole queue (the same rules: arrival order, no overtaking
of a request that does not fit, a stateful handle at most once per batch).
"""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_admission_matches_full_scan(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "admission_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", os.path.join(HERE, "admission_check.cpp"),
                    "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split()[0] == "ok" and int(out.stdout.split()[1]) >= 40000


def test_pool_allocator_first_fit_and_coalescing(tmp_path):
    """tests/pool_allocator_check.cpp: random allocations and releases on the serving pool's
    allocator (rocrand_b200/csrc/pool_allocator.hpp) against the list of live ranges --
    in bounds, no overlap, first fit, failure only when nothing fits, free list coalesced."""
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "pool_allocator_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Werror", os.path.join(HERE, "pool_allocator_check.cpp"),
                    "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.split()[0] == "ok" and int(out.stdout.split()[1]) >= 100000
