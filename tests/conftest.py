import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """The CUDA library and the restated oracle, built in-tree if missing."""
    from defmm_b200 import build as B
    if not os.path.exists(B.LIB):
        B.build()
    from oracle import oracle as O
    O.lib()
    return B.LIB


@pytest.fixture(scope="session")
def gpu():
    from defmm_b200 import api
    if api.device_count() < 1:
        pytest.skip("no CUDA device")
    return True
