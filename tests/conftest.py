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


@pytest.fixture(scope="session")
def hooks(tmp_path_factory):
    """tests/cpp/device_hooks.cu (device callbacks written against gtd_b200.h) compiled with nvcc
    into a scratch library."""
    import ctypes as C
    import subprocess
    out = str(tmp_path_factory.mktemp("hooks") / "device_hooks.so")
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-shared", "-Xcompiler", "-fPIC",
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "device_hooks.cu"),
                        "-o", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    lib = C.CDLL(out)
    lib.make_scale_args.restype = C.c_void_p
    lib.make_scale_args.argtypes = [C.c_double]
    lib.make_count_args.restype = C.c_void_p
    lib.make_count_args.argtypes = [C.c_uint64]
    lib.reset_count_args.argtypes = [C.c_void_p]
    lib.free_args.argtypes = [C.c_void_p, C.c_int]
    lib.addr = lambda name: C.cast(getattr(lib, name), C.c_void_p).value
    return lib
