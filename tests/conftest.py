import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running (full-size workloads)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    """libgpq.so on a machine with a GPU; fails loudly (never skips) when -m gpu is run
    without the library."""
    if not has_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    import gpupq_b200
    return gpupq_b200.lib()
