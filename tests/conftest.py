import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device")


@pytest.fixture(scope="session")
def ctx():
    """One library context on cuda:0 for the GPU tests."""
    import abt_b200
    c = abt_b200.Context(0)
    yield c
    c.close()
