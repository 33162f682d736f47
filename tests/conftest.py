import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a) and libgenesis_gpu.so")


def _gpu_available() -> bool:
    try:
        import torch  # noqa: F401  (only to ask the CUDA driver for a device; the product does not use torch)
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Loads the CUDA library; a GPU test fails loudly when it is missing."""
    if not _gpu_available():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    from genesis_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.load()
    return oracle
