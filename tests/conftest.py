import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libm3lb.so")
    config.addinivalue_line("markers", "slow: long-running known-answer check")


@pytest.fixture(scope="session")
def cuda_device():
    """The GPU tests run only where CUDA is present; the library itself must
    then load (no fallback)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from m3lb_b200 import capi
    capi.lib()
    torch.cuda.init()
    return torch.device("cuda:0")
