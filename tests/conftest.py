import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libmc.so")
    config.addinivalue_line("markers", "slow: full-size workloads")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    """Device fixture for -m gpu tests: requires CUDA and the in-tree libmc.so."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    from motioncorr1exp_b200 import _lib
    _lib.lib()  # raises ImportError when libmc.so is missing
    return 0
