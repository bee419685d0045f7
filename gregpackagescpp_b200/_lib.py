"""ctypes binding of libgtd_b200.so (the C ABI declared in include/gtd_b200.h).

There is no fallback: if the library is missing or no CUDA device answers, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgtd_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "gtd_b200.h")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_OVERLAPPING_BODIES = 4
ERR_INVALID_BODY_PLACEMENT = 5
ERR_INDISTINGUISHABLE = 6
ERR_NONFINITE = 7
ERR_TIMEOUT = 8
ERR_TWO_BODY = 9
ERR_NO_DEVICE = 10
ERR_CAPACITY = 11
ERR_UNSUPPORTED = 12

PREC_F64 = 0
PREC_MIXED = 1
NO_COLL, OVERLAP_COLL, MERGE_COLL = 0, 3, 4


ERR_NSYS_LOAD = 13
ERR_NSYS_FORMAT = 14
ERR_CALLBACK = 15

# gtd_step_hook: int (*)(void *user)
STEP_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p)


class GtdError(RuntimeError):
    """A non-zero status from the C ABI; ``code`` is the GTD_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[gtd status {code}] {msg}")
        self.code = code


class NbodyError(GtdError):
    """gtd::nbody_error family (gregbod.hpp:19-90)."""


class OverlappingBodiesError(NbodyError):
    """gtd::overlapping_bodies_error (gregbod.hpp:24-43)."""


class TwoBodyError(NbodyError):
    """gtd::two_body_error (gregbod.hpp:62-67)."""


class BarnesHutError(NbodyError):
    """gtd::barnes_hut_error (greg8tree.hpp:11-16)."""


class InvalidBodyPlacement(BarnesHutError):
    """gtd::invalid_body_placement (greg8tree.hpp:17-31)."""


class IndistinguishableBodies(BarnesHutError):
    """gtd::indistinguishable_bodies (greg8tree.hpp:32-46)."""


class NsysLoadError(NbodyError):
    """gtd::nsys_load_error (gregsys.hpp:125-129)."""


class NsysFormatError(NsysLoadError):
    """gtd::nsys_format_error (gregsys.hpp:130-134)."""


class CallbackError(GtdError):
    """An evolve callback (host step hook or device hook) reported a failure."""


_EXC = {
    ERR_INVALID_ARGUMENT: ValueError,
    ERR_OVERLAPPING_BODIES: OverlappingBodiesError,
    ERR_TWO_BODY: TwoBodyError,
    ERR_INVALID_BODY_PLACEMENT: InvalidBodyPlacement,
    ERR_INDISTINGUISHABLE: IndistinguishableBodies,
    ERR_NSYS_LOAD: NsysLoadError,
    ERR_NSYS_FORMAT: NsysFormatError,
    ERR_CALLBACK: CallbackError,
}

_lib = None


def exported_symbols():
    """Names declared with GTD_API in include/gtd_b200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"GTD_API\s+[\w\s\*]+?\b(gtd_\w+)\s*\(", txt)))


def load():
    """Loads the library once; raises if it is absent (never falls back to host code)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with python -m gregpackagescpp_b200.build")
    L = C.CDLL(LIB_PATH)
    vp, i64, u64, dp, ip = C.c_void_p, C.c_int64, C.c_uint64, C.c_void_p, C.c_int
    L.gtd_last_error.restype = C.c_char_p
    L.gtd_abi_version.restype = ip
    L.gtd_device_count.argtypes = [C.POINTER(C.c_int)]
    L.gtd_system_create.argtypes = [C.POINTER(vp), ip, ip]
    L.gtd_system_destroy.argtypes = [vp]
    L.gtd_system_set_params.argtypes = [vp, C.c_double, C.c_double, u64, C.c_double, C.c_double]
    L.gtd_system_set_collisions.argtypes = [vp, ip]
    L.gtd_system_upload.argtypes = [vp, i64, dp, dp, dp, dp, dp]
    L.gtd_system_check_overlap.argtypes = [vp, ip, dp]
    L.gtd_system_download.argtypes = [vp, C.POINTER(i64), dp, dp, dp, dp, dp, dp]
    L.gtd_system_num_bodies.argtypes = [vp, C.POINTER(i64)]
    L.gtd_system_evolve.argtypes = [vp, ip, C.POINTER(i64)]
    L.gtd_system_evolve_begin.argtypes = [vp, ip]
    L.gtd_system_evolve_steps.argtypes = [vp, u64]
    L.gtd_system_accelerations.argtypes = [vp, ip, dp]
    L.gtd_system_energy.argtypes = [vp, dp, dp, dp, dp]
    L.gtd_system_launch_count.argtypes = [vp, C.POINTER(u64)]
    L.gtd_system_stream.argtypes = [vp, C.POINTER(vp)]
    L.gtd_system_time_force_kernels.argtypes = [vp, ip]
    L.gtd_system_force_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(u64), ip]
    L.gtd_measure_fma_peak.argtypes = [ip, ip, C.POINTER(C.c_double)]
    L.gtd_ensemble_create.argtypes = [C.POINTER(vp), ip]
    L.gtd_ensemble_destroy.argtypes = [vp]
    L.gtd_ensemble_set_params.argtypes = [vp, C.c_double, C.c_double, ip]
    L.gtd_ensemble_upload.argtypes = [vp, i64, dp, dp, dp, dp, dp, dp]
    L.gtd_ensemble_evolve.argtypes = [vp, u64, C.POINTER(i64)]
    L.gtd_ensemble_counts.argtypes = [vp, dp, C.POINTER(u64), C.POINTER(u64)]
    L.gtd_ensemble_download.argtypes = [vp, dp, dp, dp, dp, dp, dp]
    L.gtd_ensemble_set_threads.argtypes = [vp, ip]
    L.gtd_ensemble_set_bodies_per_thread.argtypes = [vp, ip]
    L.gtd_ensemble_config.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.gtd_ensemble_autotune.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.gtd_direct_variant_count.argtypes = [ip, C.POINTER(C.c_int)]
    L.gtd_direct_variant_info.argtypes = [ip, ip, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.gtd_system_set_direct_variant.argtypes = [vp, ip]
    L.gtd_system_autotune_direct.argtypes = [vp, ip, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.gtd_system_set_mixed_near_factor.argtypes = [vp, C.c_double]
    L.gtd_system_direct_plan_info.argtypes = [vp, C.POINTER(i64), C.POINTER(i64)]
    L.gtd_bh_build.argtypes = [vp, ip]
    L.gtd_bh_set_tree_float.argtypes = [vp, ip]
    L.gtd_bh_set_walk_variant.argtypes = [vp, ip]
    L.gtd_bh_tree_size.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), dp]
    L.gtd_bh_tree_download.argtypes = [vp] + [dp] * 10
    L.gtd_bh_accelerations.argtypes = [vp, dp, dp]
    L.gtd_nsys_chunk_size.argtypes = [ip, ip, ip, C.POINTER(C.c_int)]
    L.gtd_system_set_recording.argtypes = [vp, u64]
    L.gtd_system_recording.argtypes = [vp, C.POINTER(i64), C.POINTER(i64), dp, dp]
    L.gtd_system_to_nsys.argtypes = [vp, C.c_char_p, C.c_double, C.c_double, dp, ip, ip, ip, C.POINTER(i64)]
    L.gtd_system_to_nsys_async.argtypes = [vp, C.c_char_p, C.c_double, C.c_double, dp, ip, ip, ip]
    L.gtd_system_nsys_wait.argtypes = [vp, C.POINTER(i64)]
    L.gtd_system_load_nsys.argtypes = [vp, C.c_char_p, ip, ip, ip, ip, C.POINTER(C.c_double),
                                       C.POINTER(C.c_double), dp, C.POINTER(C.c_double)]
    L.gtd_system_set_step_hook.argtypes = [vp, vp, vp]
    L.gtd_system_update_bodies.argtypes = [vp, dp, dp, dp, dp, dp]
    L.gtd_system_set_device_callbacks.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    L.gtd_system_set_rest_from_com.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, dp, ip]
    L.gtd_system_rest_from_com_centre.argtypes = [vp, dp]
    L.gtd_system_set_continue_while_rest_below.argtypes = [vp, C.c_double, u64]
    L.gtd_system_evolve_callbacks.argtypes = [vp, ip, u64, C.POINTER(u64), C.POINTER(i64)]
    L.gtd_system_callback_stats.argtypes = [vp, C.POINTER(u64), C.POINTER(C.c_int)]
    for name in exported_symbols():
        if name != "gtd_last_error":
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    """Raises the exception that matches a non-zero status (the reference's exception family)."""
    if rc == OK:
        return
    msg = _lib.gtd_last_error().decode(errors="replace") if _lib else "library not loaded"
    cls = _EXC.get(rc)
    if cls is ValueError:
        raise ValueError(msg)
    raise (cls or GtdError)(rc, msg)


def ptr(a: np.ndarray | None):
    """Address of a C-contiguous array, or None for NULL."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data
