"""Batched ensemble of independent gtd::system instances on the device (the drivers' one-system-
per-std::thread pattern, bdsim.cpp:82-113, as one persistent launch per step for all systems)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr


class Ensemble:
    """Systems s = 0..S-1 with bodies [offsets[s], offsets[s+1]); leapfrog KDK with FP64 state and
    FP32 pair forces; overlap merges after every step when ``merge`` is set."""

    def __init__(self, offsets, m, x, v=None, r=None, rest=None, G: float = 6.674e-11, dt: float = 600.0,
                 merge: bool = True, device: int = 0):
        L = _lib.load()
        self._L = L
        self.offsets = np.ascontiguousarray(np.asarray(offsets, np.int64))
        nb = int(self.offsets[-1])
        self.m = np.ascontiguousarray(np.asarray(m, np.float64))
        self.x = np.ascontiguousarray(np.asarray(x, np.float64).reshape(nb, 3))
        self.v = np.ascontiguousarray(np.zeros((nb, 3)) if v is None else np.asarray(v, np.float64).reshape(nb, 3))
        self.r = np.ascontiguousarray(np.zeros(nb) if r is None else np.asarray(r, np.float64))
        self.rest = np.ascontiguousarray(np.ones(nb) if rest is None else np.asarray(rest, np.float64))
        h = C.c_void_p()
        check(L.gtd_ensemble_create(C.byref(h), device))
        self._h = h
        check(L.gtd_ensemble_set_params(h, G, dt, 1 if merge else 0))
        check(L.gtd_ensemble_upload(h, len(self.offsets) - 1, ptr(self.offsets), ptr(self.m), ptr(self.r),
                                    ptr(self.rest), ptr(self.x), ptr(self.v)))

    @property
    def n_systems(self) -> int:
        return len(self.offsets) - 1

    def evolve(self, steps: int) -> int:
        ns = C.c_int64()
        check(self._L.gtd_ensemble_evolve(self._h, int(steps), C.byref(ns)))
        return ns.value

    def autotune(self):
        t, ms = C.c_int(), C.c_double()
        check(self._L.gtd_ensemble_autotune(self._h, C.byref(t), C.byref(ms)))
        return t.value, ms.value

    def set_threads(self, threads: int) -> None:
        check(self._L.gtd_ensemble_set_threads(self._h, int(threads)))

    def set_bodies_per_thread(self, bodies: int) -> None:
        check(self._L.gtd_ensemble_set_bodies_per_thread(self._h, int(bodies)))

    def config(self) -> tuple:
        """(CTA threads, bodies per thread) of the step kernel."""
        t, b = C.c_int(), C.c_int()
        check(self._L.gtd_ensemble_config(self._h, C.byref(t), C.byref(b)))
        return t.value, b.value

    def counts(self):
        c = np.zeros(self.n_systems, np.int64)
        merges, launches = C.c_uint64(), C.c_uint64()
        check(self._L.gtd_ensemble_counts(self._h, ptr(c), C.byref(merges), C.byref(launches)))
        return c, merges.value, launches.value

    def state(self):
        """Per-system survivors: list of dicts with m, r, rest, x, v, a (upload order)."""
        nb = int(self.offsets[-1])
        m, r, rest = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        x, v, a = np.zeros((nb, 3)), np.zeros((nb, 3)), np.zeros((nb, 3))
        check(self._L.gtd_ensemble_download(self._h, ptr(m), ptr(r), ptr(rest), ptr(x), ptr(v), ptr(a)))
        c, _, _ = self.counts()
        out = []
        for s in range(self.n_systems):
            b = int(self.offsets[s])
            k = int(c[s])
            out.append(dict(m=m[b:b + k], r=r[b:b + k], rest=rest[b:b + k], x=x[b:b + k], v=v[b:b + k],
                            a=a[b:b + k]))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gtd_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
