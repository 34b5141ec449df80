import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def cuda_ok():
    """True when an sm_100 device is present (the -m gpu tests require it)."""
    import ctypes
    try:
        rt = ctypes.CDLL("libcudart.so.12")
    except OSError:
        return False
    n = ctypes.c_int(0)
    if rt.cudaGetDeviceCount(ctypes.byref(n)) != 0 or n.value < 1:
        return False
    return True
