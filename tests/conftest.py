import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def lib():
    from skirt7_b200 import build as _b  # noqa: F401
    from skirt7_b200 import _abi
    if not os.path.exists(_abi.LIB_PATH):
        from skirt7_b200.build import build
        build()
    return _abi.load()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    oracle.lib()
    return oracle
