import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the CUDA kernels through libxmp.so)")


@pytest.fixture(scope="session")
def golden():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def handle():
    """One libxmp handle for the GPU tests; fails loudly when the library or the device is missing."""
    import xmp_b200 as xmp
    h = xmp.Handle()
    yield h
    h.destroy()
