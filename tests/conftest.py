"""Shared pytest configuration.

`-m gpu` tests need a CUDA device and call the product library (libfysics_b200.so)
through its C-ABI; everything else runs on CPU: the oracle against the reference's own
known-answer tests and golden vectors, host logic, and the ABI/export surface.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a kernels)")


def has_cuda() -> bool:
    """A CUDA device is usable by the product library (fy_gpu_init != FY_ENODEV)."""
    import fysics_b200
    return fysics_b200.load().fy_gpu_init(int(os.environ.get("FY_DEVICE", "0"))) == 0


@pytest.fixture(scope="session")
def fy():
    """The product library (ctypes); fails loudly if it was not built."""
    import fysics_b200
    fysics_b200.load()
    return fysics_b200


@pytest.fixture(scope="session")
def gpu(fy):
    if not has_cuda():
        pytest.skip("no CUDA device: " + fy.load().fy_gpu_last_error().decode())
    return fy
