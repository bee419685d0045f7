"""gtd_direct_accelerations_noalloc: direct-sum accelerations for callers that cannot let the
library allocate device memory (their memory is owned by a pool such as PyTorch's caching
allocator, or they cannot afford the device-wide synchronisation of cudaMalloc/cudaFree inside a
running loop).  The caller's torch tensors are the input and output; the entry point's only scratch
is a fixed array inside the library.

Checked through the C ABI against the existing allocating entry point (gtd_system_accelerations)
at the FP64 parity tolerance, on two calls in a row with different body counts (the second call
must not see the first call's leftovers), plus the size limit.  This file is collected last on
purpose."""
import ctypes as C

import numpy as np
import pytest

from gregpackagescpp_b200 import System, _lib
from gregpackagescpp_b200.ics import UNITS_G6674, plummer

pytestmark = pytest.mark.gpu
G = 6.674e-11


def _noalloc(pm4, acc3, precision=_lib.PREC_F64):
    import torch
    L = _lib.load()
    L.gtd_direct_accelerations_noalloc.argtypes = [C.c_int64, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                                                   C.c_void_p]
    L.gtd_direct_accelerations_noalloc.restype = C.c_int
    stream = torch.cuda.current_stream().cuda_stream
    return L.gtd_direct_accelerations_noalloc(pm4.shape[0], pm4.data_ptr(), G, precision, acc3.data_ptr(), stream)


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    import torch
    dev = torch.device("cuda:0")
    for n, seed in ((5000, 91), (3001, 92)):  # two calls in a row; the second has fewer bodies
        m, x, v = plummer(n, seed)
        pm4 = torch.tensor(np.concatenate([x, m[:, None]], 1), dtype=torch.float64, device=dev)
        acc3 = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
        _lib.check(_noalloc(pm4, acc3))
        torch.cuda.synchronize()
        got = acc3.cpu().numpy()
        want = System(m, x, v, units_format=UNITS_G6674).accelerations()
        rel = np.abs(got - want).max() / np.abs(want).max()
        assert rel < 1e-12, (n, rel)


def test_noalloc_mixed_precision_close_to_fp64(gpu):
    import torch
    m, x, v = plummer(8192, 93)
    pm4 = torch.tensor(np.concatenate([x, m[:, None]], 1), dtype=torch.float64, device="cuda:0")
    acc3 = torch.empty((8192, 3), dtype=torch.float64, device="cuda:0")
    _lib.check(_noalloc(pm4, acc3, _lib.PREC_MIXED))
    torch.cuda.synchronize()
    want = System(m, x, v, units_format=UNITS_G6674).accelerations()
    rel = np.linalg.norm(acc3.cpu().numpy() - want, axis=1) / np.linalg.norm(want, axis=1)
    assert np.sqrt((rel ** 2).mean()) < 1e-6, float(np.sqrt((rel ** 2).mean()))


def test_noalloc_rejects_more_bodies_than_its_scratch_holds(gpu):
    import torch
    pm4 = torch.zeros((65537, 4), dtype=torch.float64, device="cuda:0")
    acc3 = torch.zeros((65537, 3), dtype=torch.float64, device="cuda:0")
    rc = _noalloc(pm4, acc3)
    assert rc == _lib.ERR_CAPACITY
    assert b"65536" in _lib.load().gtd_last_error()


def test_noalloc_rejects_host_memory(gpu):
    """A host array where device memory is expected is turned into an error before any launch."""
    import torch
    L = _lib.load()
    L.gtd_direct_accelerations_noalloc.argtypes = [C.c_int64, C.c_void_p, C.c_double, C.c_int, C.c_void_p,
                                                   C.c_void_p]
    L.gtd_direct_accelerations_noalloc.restype = C.c_int
    host_pm4 = np.zeros((64, 4))
    acc3 = torch.zeros((64, 3), dtype=torch.float64, device="cuda:0")
    rc = L.gtd_direct_accelerations_noalloc(64, host_pm4.ctypes.data, G, _lib.PREC_F64, acc3.data_ptr(), None)
    assert rc == _lib.ERR_INVALID_ARGUMENT
    assert b"device" in L.gtd_last_error()


@pytest.mark.parametrize("precision", [_lib.PREC_F64, _lib.PREC_MIXED])
def test_noalloc_call_is_capturable(gpu, precision):
    """What the entry point exists for: once a first call has looked up the scratch address, a call
    allocates nothing and does not synchronise, so it can be captured in a CUDA graph (a cudaMalloc
    or a synchronisation inside the capture would make it fail).  The replay gives the eager call's
    result bit for bit."""
    import torch
    n = 4000
    m, x, _ = plummer(n, 94)
    pm4 = torch.tensor(np.concatenate([x, m[:, None]], 1), dtype=torch.float64, device="cuda:0")
    eager = torch.empty((n, 3), dtype=torch.float64, device="cuda:0")
    _lib.check(_noalloc(pm4, eager, precision))
    torch.cuda.synchronize()
    out = torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda:0")
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        rc = _noalloc(pm4, out, precision)
    assert rc == 0, _lib.load().gtd_last_error()
    assert torch.isnan(out).all()  # captured, not run
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, eager)
