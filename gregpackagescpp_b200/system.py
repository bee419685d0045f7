"""Python mirror of gtd::system / gtd::body (gregsys.hpp:135-3612, gregbod.hpp:891-1084) over the
C ABI.  Same method flags, setters, units format and evolve() contract as the reference; the
state lives in numpy arrays on the host (authoritative between calls, like the reference's
std::vector<body>) and is uploaded to the device for each evolve() and read back after it.
"""
from __future__ import annotations

import ctypes as C
import math
import re
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

from . import _lib
from ._lib import check, ptr

PI = 3.14159265358979323846

_UNITS_RE = re.compile(
    r"^\s*(m|M)\s*(?=\d{1,18}\s*:)\d*[1-9]+\d*\s*:\s*(?=\d{1,18}\s*,)\d*[1-9]+\d*\s*,\s*(d|D)\s*(?=\d{1,18}\s*:)"
    r"\d*[1-9]+\d*\s*:\s*(?=\d{1,18}\s*,)\d*[1-9]+\d*\s*,\s*(t|T)\s*(?=\d{1,18}\s*:)\d*[1-9]+\d*\s*:\s*"
    r"(?=\d{1,18}\s*$)\d*[1-9]+\d*\s*$", re.ASCII)  # std::regex's \d and \s are ASCII


def _ke(m, v):
    """body::set_ke (gregbod.hpp:325-328): 0.5 * m * |v| * |v|."""
    mag = np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2]) if len(m) else np.zeros(0)
    return 0.5 * m * mag * mag


def _seq_sum(a):
    """Left-to-right sum, the order of the reference's accumulation loops."""
    return float(np.add.accumulate(a)[-1]) if len(a) else 0.0


def units_values(units: str) -> tuple:
    """The six numbers of a units format "Ma:b,Dc:d,Tx:y" in the order the reference keeps them
    (G_vals, gregsys.hpp:275-280) and writes them to .nsys headers: (m_num=b, m_denom=a, d_num=c,
    d_denom=d, t_num=y, t_denom=x)."""
    parse_units(units)
    s = units.strip("MmDdTt ").replace(" ", "")
    m_den, m_num, d_num, d_den, t_den, t_num = [int(x) for x in re.findall(r"\d+", s)]
    return (m_num, m_den, d_num, d_den, t_num, t_den)


def parse_units(units: str) -> float:
    """G for a units format "Ma:b,Dc:d,Tx:y" (gregsys.hpp:245-282): a = mass denominator,
    b = mass numerator, c/d = distance numerator/denominator, x/y = time denominator/numerator;
    G = 66743e-15 * b c^3 y^2 / (a d^3 x^2).  Raises ValueError on a malformed string, as the
    reference throws std::invalid_argument."""
    if not _UNITS_RE.fullmatch(units):
        raise ValueError(f'The units_format string passed, "{units}", does not match the format required:\n'
                         '"Ma:b,Dc:x,Ty:z", where \'a\', \'b\', \'c\', \'x\', \'y\', and \'z\' represent any '
                         'positive integer number of 1-18 characters starting with at least one non-zero '
                         'character.\n')
    s = units.strip("MmDdTt ").replace(" ", "")
    nums = [int(x) for x in re.findall(r"\d+", s)]
    m_den, m_num, d_num, d_den, t_den, t_num = nums
    g = Fraction(66743) * m_num * d_num ** 3 * t_num ** 2 / (m_den * d_den ** 3 * t_den ** 2) / 10 ** 15
    return float(g)


class _DeviceCallback:
    """An evolve callback that runs on the GPU."""


class RestFromCom(_DeviceCallback):
    """random_comet's for_all_bods (gregsys.hpp:1966-1984) as device work: every step the carried
    centre becomes (com + sum of positions) / N -- or (com + sum m x) / M with mass_weighted (the
    GREGSYS_MERGERS form) -- with N and M taken at evolve() entry, then every body gets
    rest = max_cor - (max_cor - min_cor) d^n_exp / (d^n_exp + scale_factor), d its distance to the
    centre.  ``com`` holds the carried centre after evolve(), as the reference's lambda leaves its
    captured _com."""

    def __init__(self, min_cor, max_cor, scale_factor, n_exp, com, mass_weighted=False):
        self.min_cor, self.max_cor, self.scale_factor, self.n_exp = min_cor, max_cor, scale_factor, n_exp
        self.com = np.asarray(com, dtype=np.float64).reshape(3).copy()
        self.mass_weighted = mass_weighted


class WhileRestBelow(_DeviceCallback):
    """random_comet's continue_ev_if (gregsys.hpp:1936-1963) on the device: true while some body
    has rest < min_max_cor (resetting a counter), then for probing_iters more evaluations."""

    def __init__(self, min_max_cor, probing_iters):
        self.min_max_cor, self.probing_iters = min_max_cor, probing_iters


class DeviceHook(_DeviceCallback):
    """A caller's own device callback: ``fn`` is the address of a C function
    ``int fn(void *user, const gtd_device_bodies *bodies)`` that enqueues GPU work on
    ``bodies->stream`` (include/gtd_b200.h); ``user`` is passed back to it."""

    def __init__(self, fn: int, user: int = 0):
        self.fn, self.user = int(fn), int(user)


@dataclass
class Body:
    """gtd::body<M,R,T,0> fields that the force-and-step path reads and writes."""
    mass: float = 1.0
    radius: float = 1.0
    pos: tuple = (0.0, 0.0, 0.0)
    vel: tuple = (0.0, 0.0, 0.0)
    restitution: float = 1.0
    acc: tuple = field(default=(0.0, 0.0, 0.0))


class System:
    """gtd::system on the B200.  ``precision`` is "f64" (the reference's arithmetic) or "mixed"
    (FP32 pair forces, FP64 Kahan sums and state)."""

    two_body = 1
    euler = 2
    modified_euler = 4
    midpoint = 8
    leapfrog_kdk = 16
    leapfrog_dkd = 32
    rk4 = 64
    rk3_8 = 128
    barnes_hut = 65536
    fast_multipole = 131072
    no_coll_check = 0
    overlap_coll_check = 3
    pred_coll_check = 7
    G_SI = 6.6743e-11

    def __init__(self, m=None, x=None, v=None, r=None, rest=None, timestep: float = 1.0,
                 num_iterations: int = 1000, units_format: str = "M1:1,D1:1,T1:1",
                 allow_overlapping_bodies: bool = True, precision: str = "f64", collisions: int = 0,
                 merge_overlapping: bool = False, device: int = 0, mem_freq: int = 0):
        L = _lib.load()
        if timestep <= 0:
            raise ValueError("Time-step cannot be zero or negative.\n")  # check_dt, gregsys.hpp:1401-1405
        self.dt = float(timestep)
        self.iterations = int(num_iterations)
        self.G = parse_units(units_format)
        self.g_vals = units_values(units_format)
        self.eps = 0.0
        self.theta = PI / 3
        self.collisions = collisions
        self.merge = merge_overlapping
        self.precision = {"f64": _lib.PREC_F64, "mixed": _lib.PREC_MIXED}[precision]
        n = 0 if m is None else len(m)
        self.m = np.ascontiguousarray(np.zeros(0) if m is None else np.asarray(m, np.float64))
        self.x = np.ascontiguousarray(np.zeros((n, 3)) if x is None else np.asarray(x, np.float64).reshape(n, 3))
        self.v = np.ascontiguousarray(np.zeros((n, 3)) if v is None else np.asarray(v, np.float64).reshape(n, 3))
        self.r = np.ascontiguousarray(np.zeros(n) if r is None else np.asarray(r, np.float64))
        self.rest = np.ascontiguousarray(np.ones(n) if rest is None else np.asarray(rest, np.float64))
        self.a = np.zeros((n, 3))
        if (self.m < 0).any():
            raise _lib.NbodyError(_lib.ERR_INVALID_ARGUMENT, "negative mass")
        h = C.c_void_p()
        check(L.gtd_system_create(C.byref(h), device, self.precision))
        self._h = h
        self._L = L
        self.time_elapsed = 0.0
        # memFreq recordings (gregbod.hpp:304-320, gregsys.hpp:219-227); curr_ke is each body's
        # kinetic energy as last recorded (set at construction, gregbod.hpp:325-328)
        self.mem_freq = int(mem_freq)
        check(L.gtd_system_set_recording(h, self.mem_freq))
        self.curr_ke = _ke(self.m, self.v)
        self._clear_recordings()
        self.allow_overlap = allow_overlapping_bodies
        if not allow_overlapping_bodies:
            self.check_overlap()

    def check_overlap(self) -> None:
        """check_overlap (gregsys.hpp:307-342) on the device: raises OverlappingBodiesError for the
        first overlapping pair, or with merge_overlapping=True merges them (body::operator+=)."""
        if len(self.m) < 2:
            return
        self._push()
        pair = np.zeros(2, np.int32)
        check(self._L.gtd_system_check_overlap(self._h, 1 if self.merge else 0, ptr(pair)))
        if self.merge:
            self._pull()

    # ---- reference accessors / setters (gregsys.hpp:1627-1672) --------------------------------
    def num_bodies(self) -> int:
        return len(self.m)

    def G_val(self) -> float:
        return self.G

    def elapsed_time(self) -> float:
        return self.time_elapsed

    def set_iterations(self, number: int) -> bool:
        if not number:
            return False
        self.iterations = int(number)
        return True

    def set_timestep(self, delta_t: float) -> bool:
        if delta_t <= 0:
            return False
        self.dt = float(delta_t)
        return True

    def set_G_units(self, units_format: str) -> None:
        self.G = parse_units(units_format)
        self.g_vals = units_values(units_format)

    # ---- .nsys snapshots (gregsys.hpp:943-1400, 3214-3258) ------------------------------------
    _SIZES = {"float": 4, "double": 8, "long double": 16}

    def to_nsys(self, path: str | None, M: str = "double", R: str = "double", T: str = "double",
                wait: bool = True) -> int | None:
        """system::to_nsys: writes the bodies as a .nsys file with the chunk layout of the given
        M, R, T types ("float", "double" or "long double"); returns the bytes written (0 when path
        is None or the file cannot be opened).  wait=False returns once the snapshot is taken on
        the device; a host thread writes the file (nsys_wait() collects the result)."""
        if path is None:
            return 0
        self._push()
        gv = np.array(self.g_vals, dtype=np.uint64)
        args = (self._h, str(path).encode(), self.time_elapsed, self.dt, gv.ctypes.data, self._SIZES[M],
                self._SIZES[R], self._SIZES[T])
        if not wait:
            check(self._L.gtd_system_to_nsys_async(*args))
            return None
        nb = C.c_int64()
        check(self._L.gtd_system_to_nsys(*args, C.byref(nb)))
        return nb.value

    def nsys_wait(self) -> int:
        """Waits for the snapshot writes started with to_nsys(wait=False); the size of the last."""
        nb = C.c_int64()
        check(self._L.gtd_system_nsys_wait(self._h, C.byref(nb)))
        return nb.value

    @classmethod
    def from_nsys(cls, path: str, alloc_chunks: bool = True, check_nan_inf: bool = True,
                  allow_overlapping_bodies: bool = True, M: str = "double", R: str = "double", T: str = "double",
                  precision: str = "f64", device: int = 0) -> "System":
        """The system(const char *nsys_path, alloc_chunks, check_nan_inf, allow_overlapping_bodies)
        constructor.  alloc_chunks only chose between two host read strategies in the reference;
        here the chunks always travel in one copy and are unpacked on the device."""
        if path is None:
            raise ValueError("nullptr passed as .nsys file path.\n")
        s = cls(precision=precision, device=device)
        te, dt, G = C.c_double(), C.c_double(), C.c_double()
        gv = np.zeros(6, dtype=np.uint64)
        check(s._L.gtd_system_load_nsys(s._h, str(path).encode(), 1 if check_nan_inf else 0, cls._SIZES[M],
                                        cls._SIZES[R], cls._SIZES[T], C.byref(te), C.byref(dt), gv.ctypes.data,
                                        C.byref(G)))
        s.time_elapsed, s.dt, s.G = te.value, dt.value, G.value
        s.g_vals = tuple(int(g) for g in gv)
        s._pull()
        s.curr_ke = _ke(s.m, s.v)
        s._clear_recordings()
        s.allow_overlap = allow_overlapping_bodies
        if not allow_overlapping_bodies:
            s.check_overlap()
        return s

    def set_softening(self, epsilon: float) -> bool:
        # the reference rejects eps < sqrt(LDBL_MIN) (~1.8e-2466): for a double that is eps <= 0
        # (NaN compares false and is accepted, as there)
        if epsilon <= 0:
            return False
        self.eps = float(epsilon)
        return True

    def set_bh_opening_angle(self, theta: float) -> bool:
        # the reference compares with its long double pi: the double nearest pi lies below it and is
        # accepted, every larger double is not
        if theta < 0 or theta > math.pi:
            return False
        self.theta = float(theta)
        return True

    # ---- device round trip ------------------------------------------------------------------
    def _push(self) -> None:
        L = self._L
        check(L.gtd_system_set_params(self._h, self.G, self.dt, max(self.iterations, 1), self.eps, self.theta))
        mode = _lib.MERGE_COLL if self.merge and self.collisions else self.collisions
        check(L.gtd_system_set_collisions(self._h, mode))
        check(L.gtd_bh_set_tree_float(self._h, 1 if getattr(self, "_bh_float", True) else 0))
        check(L.gtd_system_upload(self._h, len(self.m), ptr(self.m), ptr(self.r), ptr(self.rest), ptr(self.x),
                                  ptr(self.v)))

    def _pull(self) -> None:
        n = C.c_int64()
        L = self._L
        check(L.gtd_system_num_bodies(self._h, C.byref(n)))
        k = n.value
        m, r, rest = np.zeros(k), np.zeros(k), np.zeros(k)
        x, v, a = np.zeros((k, 3)), np.zeros((k, 3)), np.zeros((k, 3))
        check(L.gtd_system_download(self._h, C.byref(n), ptr(m), ptr(r), ptr(rest), ptr(x), ptr(v), ptr(a)))
        self.m, self.r, self.rest, self.x, self.v, self.a = m, r, rest, x, v, a
        if len(getattr(self, "curr_ke", ())) != k:
            self.curr_ke = _ke(m, v)

    def evolve(self, integration_method: int = 16, continue_ev_if=None, for_each_bod=None,
               for_all_bods=None, max_steps: int = 0) -> int:
        """gtd::system::evolve (gregsys.hpp:2593-3071).  Returns the elapsed device time in ns.

        Callbacks are host callables -- continue_ev_if(), for_each_bod(system, i),
        for_all_bods(system) -- which see the state every step (the reference's contract; the state
        makes a host round trip for them), or device callbacks (RestFromCom, WhileRestBelow,
        DeviceHook) that run on the GPU, with the bodies and the predicate kept on the device.  The
        two kinds cannot be mixed.  max_steps (device callbacks only) stops a loop whose predicate
        never turns false.  Per step, as in the reference (gregsys.hpp:16-106, 2970-2987):
        continue_ev_if, the update, for_all_bods, the collision pass, for_each_bod."""
        cbs = [c for c in (continue_ev_if, for_each_bod, for_all_bods) if c is not None]
        if cbs and any(isinstance(c, _DeviceCallback) for c in cbs):
            if not all(isinstance(c, _DeviceCallback) for c in cbs):
                raise TypeError("device callbacks and host callables cannot be mixed in one evolve")
            return self._evolve_device(integration_method, continue_ev_if, for_each_bod, for_all_bods, max_steps)
        self._push()
        ns = C.c_int64()
        if not cbs:
            x0, v0 = self.x.copy(), self.v.copy()
            check(self._L.gtd_system_evolve(self._h, integration_method, C.byref(ns)))
            self._pull()
            self._recordings_from(x0, v0, integration_method)
            self.time_elapsed = self.iterations * self.dt
            return ns.value
        x0, v0 = self.x.copy(), self.v.copy()
        if (integration_method & System.barnes_hut) == System.barnes_hut:
            # the Barnes-Hut branch calls no callback (gregsys.hpp:2893-2945)
            check(self._L.gtd_system_evolve(self._h, integration_method, C.byref(ns)))
            self._pull()
            self._recordings_from(x0, v0, integration_method)
            self.time_elapsed = self.iterations * self.dt
            return ns.value
        err = []

        def step_hook(_user):
            try:
                self._pull()
                for_all_bods(self)
                self._update()
                return 0
            except BaseException as e:  # re-raised below, after the engine unwinds
                err.append(e)
                return _lib.ERR_CALLBACK

        hook = _lib.STEP_HOOK(step_hook) if for_all_bods is not None else None
        L = self._L
        try:
            if hook is not None:
                check(L.gtd_system_set_step_hook(self._h, C.cast(hook, C.c_void_p), None))
            check(L.gtd_system_evolve_begin(self._h, integration_method))
            steps = 0
            while (continue_ev_if() if continue_ev_if is not None else steps < self.iterations):
                rc = L.gtd_system_evolve_steps(self._h, 1)
                if err:
                    raise err[0]
                check(rc)
                steps += 1
                if for_each_bod is not None:
                    self._pull()
                    for i in range(len(self.m)):
                        for_each_bod(self, i)
                    self._update()
        finally:
            if hook is not None:
                L.gtd_system_set_step_hook(self._h, None, None)
        self._pull()
        self._recordings_from(x0, v0, integration_method)
        self.time_elapsed = self.iterations * self.dt  # gregsys.hpp:3069, whatever the steps taken
        self.steps_taken = steps
        return 0

    def _update(self) -> None:
        """A callback's writes, sent back without restarting the evolve in progress (the body count
        cannot change inside a callback)."""
        n = C.c_int64()
        check(self._L.gtd_system_num_bodies(self._h, C.byref(n)))
        if len(self.m) != n.value:
            raise ValueError("an evolve callback changed the number of bodies")
        self.m, self.r, self.rest = (np.ascontiguousarray(a, dtype=np.float64) for a in (self.m, self.r, self.rest))
        self.x, self.v = (np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 3) for a in (self.x, self.v))
        check(self._L.gtd_system_update_bodies(self._h, ptr(self.m), ptr(self.r), ptr(self.rest), ptr(self.x),
                                               ptr(self.v)))

    def _evolve_device(self, method, cont, each, all_, max_steps) -> int:
        L, h = self._L, self._h
        x0, v0 = self.x.copy(), self.v.copy()
        self._push()
        hooks = []
        for cb in (cont, each, all_):
            if isinstance(cb, DeviceHook):
                hooks += [C.c_void_p(cb.fn), C.c_void_p(cb.user)]
            else:
                hooks += [None, None]
        check(L.gtd_system_set_device_callbacks(h, *hooks))
        if isinstance(cont, WhileRestBelow):
            check(L.gtd_system_set_continue_while_rest_below(h, float(cont.min_max_cor), int(cont.probing_iters)))
        if isinstance(all_, RestFromCom):
            com = np.ascontiguousarray(all_.com, dtype=np.float64).reshape(3)
            check(L.gtd_system_set_rest_from_com(h, float(all_.min_cor), float(all_.max_cor), float(all_.scale_factor),
                                                 float(all_.n_exp), ptr(com), 1 if all_.mass_weighted else 0))
        if isinstance(each, (WhileRestBelow, RestFromCom)) or isinstance(cont, RestFromCom) or \
                isinstance(all_, WhileRestBelow):
            raise TypeError("a built-in device callback was passed in the wrong position")
        steps, ns = C.c_uint64(), C.c_int64()
        try:
            check(L.gtd_system_evolve_callbacks(h, method, int(max_steps), C.byref(steps), C.byref(ns)))
        finally:
            L.gtd_system_set_device_callbacks(h, None, None, None, None, None, None)
        self._pull()
        self._recordings_from(x0, v0, method)
        if isinstance(all_, RestFromCom):
            c = np.zeros(3)
            check(L.gtd_system_rest_from_com_centre(h, ptr(c)))
            all_.com = c
        self.time_elapsed = self.iterations * self.dt  # gregsys.hpp:3069, whatever the steps taken
        self.steps_taken = steps.value
        return ns.value

    def callback_stats(self) -> dict:
        """How the last device-callback evolve ran: host waits (one per 64-step graph chunk, or per
        step in the eager form) and whether the CUDA-graph loop ran."""
        w, g = C.c_uint64(), C.c_int()
        check(self._L.gtd_system_callback_stats(self._h, C.byref(w), C.byref(g)))
        return {"host_waits": w.value, "graph_loop": bool(g.value)}

    # ---- memFreq recordings ------------------------------------------------------------------
    def _clear_recordings(self) -> None:
        """clear_evolution (gregsys.hpp:2569-2586) / body::clear (gregbod.hpp:621-628): one frame,
        the current state with the last recorded kinetic energy; no energy records."""
        n = len(self.m)
        self.positions = self.x.reshape(1, n, 3).copy()
        self.velocities = self.v.reshape(1, n, 3).copy()
        self.kinetic_energies = self.curr_ke.reshape(1, n).copy()
        self.pe = np.zeros((0, n))
        self.energies = np.zeros((0, n))
        self.tot_pe, self.tot_ke, self.tot_e = np.zeros(0), np.zeros(0), np.zeros(0)

    def _recordings_from(self, x0, v0, method: int) -> None:
        """The last evolve's records, its first frame the state (x0, v0) it started from."""
        if self.mem_freq and len(self.m):
            self.x, self.v, cur = x0, v0, (self.x, self.v)
            self._collect_recordings(method)
            self.x, self.v = cur

    def _collect_recordings(self, method: int) -> None:
        """The records the reference keeps (fileFreq = 0, the only setting with which its evolve
        compiles): FUNC_TEMPL_SELECT (gregsys.hpp:15-105) never takes its recording branch, so
        trajectories beyond the first frame come only from the collision pass (s_coll<true>, with
        collisions on); energies come from calc_acc_and_e / calc_energy (every frame of Euler,
        modified Euler and midpoint; only the first for the leapfrogs without collisions, whose
        per-step energy records sit behind that branch) and from the leapfrogs' collision path.
        Energies use each body's last recorded kinetic energy.  Barnes-Hut branches record nothing."""
        self._clear_recordings()
        f = C.c_int64()
        nb = C.c_int64()
        check(self._L.gtd_system_recording(self._h, C.byref(f), C.byref(nb), None, None))
        if f.value == 0 or method & self.barnes_hut:
            return
        n = nb.value
        states = np.zeros(f.value, np.int64)
        fr = np.zeros((f.value, n, 8))
        check(self._L.gtd_system_recording(self._h, None, None, ptr(states), ptr(fr)))
        branch = next((b for b in (1, 2, 4, 8, 16, 32, 64, 128) if method & b == b), 0)
        coll = self.collisions != 0
        if coll and f.value > 1:
            self.positions = np.concatenate([self.positions, fr[1:, :, 0:3]])
            self.velocities = np.concatenate([self.velocities, fr[1:, :, 3:6]])
            self.kinetic_energies = np.concatenate([self.kinetic_energies, fr[1:, :, 6]])
        n_e = 1 if (branch in (self.leapfrog_kdk, self.leapfrog_dkd) and not coll) else f.value
        ke_at = [self.curr_ke if (k == 0 or not coll) else fr[k, :, 6] for k in range(n_e)]
        self.pe = fr[:n_e, :, 7].copy()
        self.energies = np.array([ke_at[k] + self.pe[k] for k in range(n_e)]).reshape(n_e, n)
        self.tot_pe = np.array([_seq_sum(self.pe[k]) for k in range(n_e)])
        self.tot_ke = np.array([_seq_sum(ke_at[k]) for k in range(n_e)])
        self.tot_e = self.tot_pe + self.tot_ke
        if coll and f.value > 1:
            self.curr_ke = fr[-1, :, 6].copy()

    def accelerations(self, method: int = 0) -> np.ndarray:
        self._push()
        a = np.zeros((len(self.m), 3))
        check(self._L.gtd_system_accelerations(self._h, method, ptr(a)))
        return a

    def energy(self):
        """(KE, PE, momentum[3], com[3]) in FP64 on the device (calc_energy, gregsys.hpp:608-630)."""
        self._push()
        ke, pe = C.c_double(), C.c_double()
        p, com = np.zeros(3), np.zeros(3)
        check(self._L.gtd_system_energy(self._h, C.byref(ke), C.byref(pe), ptr(p), ptr(com)))
        return ke.value, pe.value, p, com

    # ---- Barnes-Hut (greg8tree.hpp) ---------------------------------------------------------
    def bh_build(self, tree_float: bool = True) -> None:
        """bh_tree::add_bodies + calc_com (greg8tree.hpp:1062-1078) on the device."""
        self._push()
        check(self._L.gtd_bh_set_walk_variant(self._h, getattr(self, "_walk_variant", -1)))
        check(self._L.gtd_bh_build(self._h, 1 if tree_float else 0))

    def bh_tree(self) -> dict:
        """The last built octree: sorted Morton codes, slot -> body, and per node in DFS pre-order
        depth, leaf flag, first slot, body count, skip link, mass, centre of mass, cell width."""
        L = self._L
        nn, nl = C.c_int64(), C.c_int64()
        box = np.zeros(6)
        check(L.gtd_bh_tree_size(self._h, C.byref(nn), C.byref(nl), ptr(box)))
        n, k = len(self.m), nn.value
        out = dict(n_nodes=k, n_leaves=nl.value, box=box, code=np.zeros(n, np.uint64), perm=np.zeros(n, np.int32),
                   depth=np.zeros(k, np.int8), is_leaf=np.zeros(k, np.int8), first=np.zeros(k, np.int32),
                   count=np.zeros(k, np.int32), skip=np.zeros(k, np.int32), mass=np.zeros(k),
                   com=np.zeros((k, 3)), width=np.zeros(k))
        check(L.gtd_bh_tree_download(self._h, *(ptr(out[f]) for f in ("code", "perm", "depth", "is_leaf", "first",
                                                                      "count", "skip", "mass", "com", "width"))))
        return out

    def bh_accelerations(self, tree_float: bool = True):
        """Barnes-Hut accelerations with the reference walk (greg8tree.hpp:702-833, bh_acc
        gregsys.hpp:371-375 accumulated) and the interactions each body took."""
        self.bh_build(tree_float)
        a = np.zeros((len(self.m), 3))
        cnt = np.zeros(len(self.m), np.uint32)
        check(self._L.gtd_bh_accelerations(self._h, ptr(a), ptr(cnt)))
        return a, cnt

    def set_bh_walk_variant(self, variant: int) -> None:
        """Float-tree walk (-1 default = 2, 0 per-lane walk with separate node arrays, 1 per-lane
        walk with interleaved 32-byte records, 2 list walk); all take the same interactions per
        body, 0 and 1 in the same order, 2 summed in another order."""
        if variant < -1 or variant > 2:
            raise ValueError(f"walk variant {variant} out of range")
        self._walk_variant = int(variant)

    def bh_tree_float(self, tree_float: bool) -> None:
        """Selects T=float (True, the default) or T=double geometry for the Barnes-Hut evolve."""
        self._bh_float = bool(tree_float)

    def launch_count(self) -> int:
        c = C.c_uint64()
        check(self._L.gtd_system_launch_count(self._h, C.byref(c)))
        return c.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.gtd_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
