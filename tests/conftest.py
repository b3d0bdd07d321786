import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def orc():
    from oracle import pyorc
    return pyorc.CLib("orc")


@pytest.fixture(scope="session")
def lib():
    import rocrand_b200
    return rocrand_b200.load_library()
