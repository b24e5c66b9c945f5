import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the libdftcuda kernels)")


@pytest.fixture(scope="session")
def dz():
    """The dft-zig_b200 package (host mirror over libdftcuda.so)."""
    import dftzig_loader

    return dftzig_loader.load()
