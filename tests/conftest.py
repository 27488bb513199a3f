import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU and the built libfastpls_b200.so")


@pytest.fixture(scope="session")
def lib():
    """The C-ABI library; GPU tests fail loudly when it or the device is missing."""
    from fastpls_b200 import _lib
    _lib.load()
    assert _lib.has_cuda(), "no usable B200 device for the GPU tests"
    return _lib
