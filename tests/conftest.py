import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libreplay")
    config.addinivalue_line("markers", "montecarlo: statistical comparison with the reference's "
                            "unseeded Monte Carlo; runs after every bit-exact test")


def pytest_collection_modifyitems(session, config, items):
    """Bit-exact tests first, then the statistical ones (marked montecarlo),
    then the allocation-free entry point's test file, which stays last: a run
    that stops at its first failure has then run every bit-exact test."""
    def rank(item):
        if os.path.basename(str(item.fspath)) == "test_zz_no_alloc.py":
            return 2
        return 1 if item.get_closest_marker("montecarlo") else 0
    items.sort(key=rank)


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def oracle():
    from oracle import orc
    orc.lib()
    return orc


@pytest.fixture(scope="session")
def refshim():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference not built here (oracle/_ref)")
    return ref
