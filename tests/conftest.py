import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device; GPU tests fail (not skip) when the native library is missing."""
    if not _has_gpu():
        pytest.skip("no CUDA device")
    import torch
    from alpaca_b200 import native
    native.lib()  # raises if libalpaca_b200.so is absent
    return torch.device("cuda:0")
