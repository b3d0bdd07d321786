import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_addoption(parser):
    parser.addoption("--runslow", action="store_true", default=False,
                     help="also run the tests marked slow (full-size comparisons with the "
                          "single-core oracle)")


def pytest_collection_modifyitems(config, items):
    if config.getoption("--runslow") or os.environ.get("RB_RUN_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow: run with --runslow")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)


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


def pytest_terminal_summary(terminalreporter):
    """Reports the fp64 elements accepted by the backward-error rule of
    tests/gpu_util.compare_call (outside the forward ulp bound), per generator and
    distribution."""
    gu = sys.modules.get("tests.gpu_util")
    stats = getattr(gu, "FP64_EXCEPTIONS", None) if gu else None
    if not stats:
        return
    terminalreporter.write_line("fp64 elements outside the forward ulp bound, accepted by the "
                                "backward-error rule:")
    for (rng, dist), (bad, total) in sorted(stats.items()):
        terminalreporter.write_line("  rng %d %s: %d of %d (%.3g)" % (rng, dist, bad, total,
                                                                      bad / max(total, 1)))
