import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200); runs the CUDA path through the C ABI")


def has_gpu() -> bool:
    try:
        import ctypes
        from gregpackagescpp_b200 import _lib
        L = _lib.load()
        n = ctypes.c_int()
        return L.gtd_device_count(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "reference_golden.npz"))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("a -m gpu test ran without a CUDA device or without libgtd_b200.so")
    return True
