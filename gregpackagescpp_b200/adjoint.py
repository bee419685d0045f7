"""Gradients of a loss on the final state of an FP64 leapfrog-KDK direct-summation run
(gtd::system::evolve(leapfrog_kdk), gregsys.hpp:2946-2990) with respect to the initial positions,
velocities and masses: the hand-written adjoint kernels of libgtd_b200.so behind a
torch.autograd.Function.  torch only carries the device buffers and the stream; every kernel is
the library's.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check


def _bind(L):
    vp, i64, u64, ip = C.c_void_p, C.c_int64, C.c_uint64, C.c_int
    if getattr(L, "_adj_bound", False):
        return
    L.gtd_adjoint_create.argtypes = [C.POINTER(vp), ip, i64, u64, u64, C.c_double, C.c_double]
    L.gtd_adjoint_destroy.argtypes = [vp]
    L.gtd_adjoint_forward.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.gtd_adjoint_backward.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.gtd_adjoint_launch_count.argtypes = [vp, C.POINTER(u64)]
    L._adj_bound = True


class AdjointRun:
    """One forward run kept for its reverse sweep (checkpoints every ``checkpoint_every`` steps)."""

    def __init__(self, n: int, steps: int, checkpoint_every: int, G: float, dt: float, device: int):
        L = _lib.load()
        _bind(L)
        self._L = L
        h = C.c_void_p()
        check(L.gtd_adjoint_create(C.byref(h), device, n, steps, checkpoint_every, G, dt))
        self._h = h

    def launches(self) -> int:
        c = C.c_uint64()
        check(self._L.gtd_adjoint_launch_count(self._h, C.byref(c)))
        return c.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._L.gtd_adjoint_destroy(self._h)
                self._h = None
        except Exception:
            pass


def leapfrog_final_state(x0, v0, m, G: float, dt: float, steps: int, checkpoint_every: int | None = None):
    """(x_T, v_T) of `steps` KDK steps from (x0, v0) with masses m (CUDA float64 tensors, shapes
    (n,3), (n,3), (n,)), differentiable with respect to x0, v0 and m."""
    import math

    import torch

    class _LeapfrogAdjoint(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x0_, v0_, m_):
            for t in (x0_, v0_, m_):
                if not (t.is_cuda and t.dtype == torch.float64):
                    raise TypeError("x0, v0, m must be CUDA float64 tensors")
            x0c, v0c, mc = x0_.contiguous(), v0_.contiguous(), m_.contiguous()
            n = mc.numel()
            every = checkpoint_every or max(1, int(round(math.sqrt(steps))))
            run = AdjointRun(n, steps, every, G, dt, x0c.device.index or 0)
            xT = torch.empty_like(x0c)
            vT = torch.empty_like(v0c)
            stream = torch.cuda.current_stream(x0c.device).cuda_stream
            check(run._L.gtd_adjoint_forward(run._h, x0c.data_ptr(), v0c.data_ptr(), mc.data_ptr(), xT.data_ptr(),
                                             vT.data_ptr(), stream))
            ctx.run = run
            ctx.shapes = (x0c.shape, mc.shape)
            return xT, vT

        @staticmethod
        def backward(ctx, gxT, gvT):
            run = ctx.run
            dev = gxT.device if gxT is not None else gvT.device
            xs, ms = ctx.shapes
            gx = (gxT if gxT is not None else torch.zeros(xs, dtype=torch.float64, device=dev)).contiguous()
            gv = gvT.contiguous() if gvT is not None else None
            gx0 = torch.empty(xs, dtype=torch.float64, device=dev)
            gv0 = torch.empty(xs, dtype=torch.float64, device=dev)
            gm = torch.empty(ms, dtype=torch.float64, device=dev)
            stream = torch.cuda.current_stream(dev).cuda_stream
            check(run._L.gtd_adjoint_backward(run._h, gx.data_ptr(), gv.data_ptr() if gv is not None else None,
                                              gx0.data_ptr(), gv0.data_ptr(), gm.data_ptr(), stream))
            return gx0, gv0, gm

    return _LeapfrogAdjoint.apply(x0, v0, m)
