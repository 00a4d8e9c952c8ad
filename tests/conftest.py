import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and runs the CUDA kernels")


@pytest.fixture(scope="session")
def lib():
    from sovereign_b200 import _lib
    return _lib.load()
