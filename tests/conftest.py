import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def pytest_collection_modifyitems(config, items):
    # GPU tests fail loudly when CUDA is missing rather than silently passing.
    pass


@pytest.fixture(scope="session")
def lib():
    import nutrlan_b200
    return nutrlan_b200.load()


@pytest.fixture(scope="session")
def reflib():
    from oracle import ref
    if not ref.available():
        pytest.skip("reference oracle library not built (make -C oracle)")
    return ref.load()
