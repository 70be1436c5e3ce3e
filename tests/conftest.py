import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden():
    return GOLDEN


def cuda_available() -> bool:
    try:
        import ctypes

        cudart = ctypes.CDLL("libcudart.so.12")
    except OSError:
        try:
            import torch

            return torch.cuda.is_available()
        except Exception:
            return False
    count = ctypes.c_int(0)
    return cudart.cudaGetDeviceCount(ctypes.byref(count)) == 0 and count.value > 0
