"""ctypes access to the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* ``Oracle``    - oracle/liboracle.so, the plain-C restatement (nbody_oracle.c).  Builds on any box
                  with gcc (``ensure_built`` runs make).
* ``RefOracle`` - oracle/_ref/libgtdref.so, the unmodified reference headers behind ref_oracle.cpp.
                  Present only where it was built from the reference tree (it travels as a built
                  file; it cannot be rebuilt where the reference sources are absent).

Only tests/, the golden-fixture generator, ``__graft_entry__.smoke()`` and the CPU legs of
bench.py import this module.  The product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REFLIB = os.path.join(HERE, "_ref", "libgtdref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")

EULER, MODIFIED_EULER, MIDPOINT, LEAPFROG_KDK, LEAPFROG_DKD = 2, 4, 8, 16, 32


def reference_tree() -> str | None:
    """The reference checkout the Makefile reads (GTD_REFERENCE_DIR, else the Makefile's default),
    or None when it is not present on this machine."""
    try:
        r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, timeout=60)
        path = r.stdout.strip()
    except Exception:
        return None
    return path if path and os.path.isdir(path) else None


def ensure_built(ref: bool = False) -> None:
    """Compile the C restatement (and, when asked and the reference tree is present, the
    reference-backed driver) with oracle/Makefile."""
    targets = [LIB]
    need = not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
        os.path.getmtime(os.path.join(HERE, f)) for f in ("nbody_oracle.c", "nbody_oracle.h"))
    if need:
        subprocess.run(["make", "-s", "-C", HERE, LIB], check=True)
    tree = reference_tree() if ref else None
    if tree:
        if (not os.path.exists(REFLIB) or
                os.path.getmtime(REFLIB) < os.path.getmtime(os.path.join(HERE, "ref_oracle.cpp"))):
            subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={tree}"], check=True)
    del targets


def _c3(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


class _Tree(C.Structure):
    _fields_ = [("n", C.c_int), ("n_nodes", C.c_int), ("n_leaves", C.c_int),
                ("code", C.POINTER(C.c_uint64)), ("perm", C.POINTER(C.c_int32)),
                ("depth", C.POINTER(C.c_int8)), ("is_leaf", C.POINTER(C.c_int8)),
                ("first", C.POINTER(C.c_int32)), ("count", C.POINTER(C.c_int32)),
                ("skip", C.POINTER(C.c_int32)), ("mass", C.POINTER(C.c_double)),
                ("com3", C.POINTER(C.c_double)), ("width", C.POINTER(C.c_double)),
                ("box6", C.c_double * 6)]


class Oracle:
    """The plain-C restatement of the reference arithmetic."""

    def __init__(self):
        ensure_built()
        L = self.lib = C.CDLL(LIB)
        L.orc_G_units.restype = C.c_longdouble
        L.orc_G_units.argtypes = [C.c_uint64] * 6
        L.orc_G_units_into.argtypes = [C.c_uint64] * 6 + [C.POINTER(C.c_longdouble)]
        L.orc_direct_acc.argtypes = [C.c_int, _dp, _dp, C.POINTER(C.c_longdouble), _dp]
        L.orc_direct_acc_rows.argtypes = [C.c_int, _dp, _dp, C.POINTER(C.c_longdouble), _ip, C.c_int, _dp,
                                          C.c_void_p, C.c_int]
        L.orc_evolve.restype = C.c_int
        L.orc_evolve.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_longdouble,
                                 C.c_uint64, C.POINTER(C.c_longdouble)]
        L.orc_s_coll.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.orc_energy.argtypes = [C.c_int, _dp, _dp, _dp, C.POINTER(C.c_longdouble), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]
        L.orc_merge_pair.argtypes = [_dp, _dp]
        L.orc_merge_overlapping.restype = C.c_int
        L.orc_merge_overlapping.argtypes = [C.c_int, _dp]
        L.orc_bh_root_box.argtypes = [C.c_int, _dp, C.c_int, _dp]
        L.orc_bh_build.restype = C.c_int
        L.orc_bh_build.argtypes = [C.c_int, _dp, _dp, C.c_int, C.POINTER(_Tree)]
        L.orc_bh_free.argtypes = [C.POINTER(_Tree)]
        L.orc_bh_acc.argtypes = [C.POINTER(_Tree), _dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _up]
        L.orc_bh_s_coll.restype = C.c_int
        L.orc_bh_s_coll.argtypes = [C.POINTER(_Tree), _dp, _dp, _dp, _dp, _dp, C.c_int]
        L.orc_bench_kdk.restype = C.c_int
        L.orc_bench_kdk.argtypes = [C.c_int, _dp, _dp, _dp, C.c_longdouble, C.c_uint64, C.POINTER(C.c_longdouble),
                                    C.c_int, C.POINTER(C.c_longlong)]

    def bench_kdk(self, m, x, v, dt, steps, G, threads):
        """Wall seconds for `threads` concurrent copies of orc_evolve(leapfrog_kdk)."""
        ns = C.c_longlong()
        self.lib.orc_bench_kdk(len(m), _c3(m), _c3(x), _c3(v), dt, steps, C.byref(G), threads, C.byref(ns))
        return ns.value * 1e-9

    @staticmethod
    def G_units(units: str):
        """The reference's G for a units string, as a Python float of the long double."""
        parts = units.replace(" ", "").split(",")
        nums = []
        for p in parts:
            a, b = p[1:].split(":")
            nums += [int(a), int(b)]
        return nums

    def G(self, units: str = "M66743:66740,D1:1,T1:1"):
        """The reference's G as a ctypes long double (all 64 mantissa bits kept; a Python float
        would round it to double)."""
        g = C.c_longdouble()
        self.lib.orc_G_units_into(*self.G_units(units), C.byref(g))
        return g

    def direct_acc(self, m, x, G):
        n = len(m)
        a = np.zeros(3 * n)
        self.lib.orc_direct_acc(n, _c3(m), _c3(x), C.byref(G), a)
        return a.reshape(n, 3)

    def direct_acc_rows(self, m, x, G, rows, threads=1):
        """orc_direct_acc for the bodies `rows` only (the same bits), and per row the scale
        sum_j G m_j / r_ij^2 of the summed force.  Returns (a[len(rows), 3], gross[len(rows)])."""
        rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int32))
        a = np.zeros(3 * len(rows))
        gross = np.zeros(len(rows))
        self.lib.orc_direct_acc_rows(len(m), _c3(m), _c3(x), C.byref(G), rows, len(rows), a,
                                     gross.ctypes.data, int(threads))
        return a.reshape(-1, 3), gross

    def evolve(self, method, m, x, v, dt, steps, G, r=None, rest=None, coll=0):
        n = len(m)
        x3, v3, a3 = _c3(x).copy(), _c3(v).copy(), np.zeros(3 * n)
        r = _c3(np.zeros(n) if r is None else r)
        rest = _c3(np.ones(n) if rest is None else rest)
        rc = self.lib.orc_evolve(method, coll, n, _c3(m), r, rest, x3, v3, a3, dt, steps, C.byref(G))
        if rc:
            raise RuntimeError(f"orc_evolve failed ({rc})")
        return x3.reshape(n, 3), v3.reshape(n, 3), a3.reshape(n, 3)

    def s_coll(self, m, r, rest, x, v):
        n = len(m)
        v3 = _c3(v).copy()
        self.lib.orc_s_coll(n, _c3(m), _c3(r), _c3(rest), _c3(x), v3)
        return v3.reshape(n, 3)

    def energy(self, m, x, v, G):
        ke, pe = C.c_double(), C.c_double()
        self.lib.orc_energy(len(m), _c3(m), _c3(x), _c3(v), C.byref(G), C.byref(ke), C.byref(pe))
        return ke.value, pe.value

    def merge_pair(self, a12, b12):
        a = _c3(a12).copy()
        self.lib.orc_merge_pair(a, _c3(b12))
        return a

    def merge_overlapping(self, rows12):
        rows = _c3(rows12).copy()
        n = self.lib.orc_merge_overlapping(len(rows) // 12, rows)
        return rows.reshape(-1, 12)[:n].copy()

    def root_box(self, x, is_float):
        box = np.zeros(6)
        self.lib.orc_bh_root_box(len(x), _c3(x), int(is_float), box)
        return box

    def bh_tree(self, x, m, is_float):
        """Host rebuild of the linear octree; returns a dict of numpy arrays."""
        t = _Tree()
        n = len(m)
        rc = self.lib.orc_bh_build(n, _c3(x), _c3(m), int(is_float), C.byref(t))
        if rc:
            raise RuntimeError(f"orc_bh_build failed ({rc})")
        nn = t.n_nodes

        def arr(p, k, dt):
            return np.ctypeslib.as_array(p, shape=(k,)).astype(dt).copy() if k else np.zeros(0, dt)

        out = dict(n=n, n_nodes=nn, n_leaves=t.n_leaves, box=np.array(t.box6[:]),
                   code=arr(t.code, n, np.uint64), perm=arr(t.perm, n, np.int32),
                   depth=arr(t.depth, nn, np.int8), is_leaf=arr(t.is_leaf, nn, np.int8),
                   first=arr(t.first, nn, np.int32), count=arr(t.count, nn, np.int32),
                   skip=arr(t.skip, nn, np.int32), mass=arr(t.mass, nn, np.float64),
                   com=arr(t.com3, 3 * nn, np.float64).reshape(nn, 3), width=arr(t.width, nn, np.float64))
        out["_tree"] = t
        return out

    def bh_s_coll(self, tree, m, r, rest, x, v, is_float):
        """bh_s_coll over `tree` (built at x); returns the new velocities."""
        n = tree["n"]
        v3 = _c3(v).copy()
        rc = self.lib.orc_bh_s_coll(C.byref(tree["_tree"]), _c3(m), _c3(r), _c3(rest), _c3(x), v3, int(is_float))
        if rc:
            raise RuntimeError(f"orc_bh_s_coll failed ({rc})")
        return v3.reshape(n, 3)

    def bh_free(self, tree):
        self.lib.orc_bh_free(C.byref(tree["_tree"]))

    def bh_acc(self, tree, x, m, is_float, theta, eps, G):
        n = tree["n"]
        a = np.zeros(3 * n)
        cnt = np.zeros(n, np.uint32)
        self.lib.orc_bh_acc(C.byref(tree["_tree"]), _c3(x), _c3(m), int(is_float), theta, eps, G, a, cnt)
        return a.reshape(n, 3), cnt


class RefOracle:
    """The unmodified reference headers behind ref_oracle.cpp (oracle/_ref/libgtdref.so)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFLIB)

    def __init__(self):
        if not os.path.exists(REFLIB):
            raise FileNotFoundError(REFLIB)
        L = self.lib = C.CDLL(REFLIB)
        L.ref_last_error.restype = C.c_char_p
        L.ref_evolve.restype = C.c_int
        L.ref_evolve.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_uint64,
                                 C.c_char_p, _dp, _dp, _dp, C.POINTER(C.c_longlong)]
        L.ref_G.restype = C.c_int
        L.ref_G.argtypes = [C.c_char_p, C.POINTER(C.c_longdouble)]
        L.ref_setters.restype = C.c_int
        L.ref_setters.argtypes = [C.c_longdouble, C.c_uint64, C.c_longdouble, C.c_longdouble, _ip]
        L.ref_check_option.restype = C.c_int
        L.ref_check_option.argtypes = [C.c_int]
        L.ref_construct_dt.restype = C.c_int
        L.ref_construct_dt.argtypes = [C.c_longdouble]
        L.ref_energy.restype = C.c_int
        L.ref_energy.argtypes = [C.c_int, _dp, _dp, _dp, C.c_char_p, C.POINTER(C.c_longdouble),
                                 C.POINTER(C.c_longdouble)]
        L.ref_check_overlap_merge.restype = C.c_int
        L.ref_check_overlap_merge.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int), _dp, _dp, _dp,
                                              _dp]
        L.ref_merge_pair.restype = C.c_int
        L.ref_merge_pair.argtypes = [_dp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double), _dp, _dp, _dp,
                                     C.POINTER(C.c_double)]
        L.ref_bh_tree_dump.restype = C.c_long
        L.ref_bh_tree_dump.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_long, _ip, _ip, _dp, _dp, _dp, _dp, _dp]
        L.ref_bh_acc.restype = C.c_int
        L.ref_bh_acc.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_char_p, _dp,
                                 C.POINTER(C.c_uint64)]
        L.ref_bench_kdk.restype = C.c_int
        L.ref_bench_kdk.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, C.c_uint64, C.c_char_p, C.c_int,
                                    C.POINTER(C.c_longlong)]
        L.ref_to_nsys.restype = C.c_int
        L.ref_to_nsys.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_uint64, C.c_char_p,
                                  C.c_char_p, C.POINTER(C.c_longlong)]
        L.ref_load_nsys.restype = C.c_int
        L.ref_load_nsys.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), _dp, _dp,
                                    _dp, _dp, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]
        L.ref_evolve_record.restype = C.c_int
        L.ref_evolve_record.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double,
                                        C.c_uint64, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                        C.POINTER(C.c_int), _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_bh_kdk_coll.restype = C.c_int
        L.ref_bh_kdk_coll.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_uint64, C.c_double,
                                      C.c_char_p, _dp, _dp]
        L.ref_bh_s_coll.restype = C.c_int
        L.ref_bh_s_coll.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_bh_kdk.restype = C.c_int
        L.ref_bh_kdk.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double, C.c_uint64, C.c_double, C.c_double,
                                 C.c_char_p, _dp, _dp, _dp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]

        L.ref_evolve_callbacks.restype = C.c_int
        L.ref_evolve_callbacks.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_uint64,
                                           C.c_char_p, C.c_int, C.c_double, C.c_uint64, C.c_int, C.c_double,
                                           C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double,
                                           C.c_uint64, _dp, _dp, _dp, _dp, C.POINTER(C.c_uint64)]
        L.ref_evolve_record_callbacks.restype = C.c_int
        L.ref_evolve_record_callbacks.argtypes = (
            [C.c_int, C.c_int, C.c_uint64, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_uint64, C.c_char_p,
             C.c_int, C.c_double, C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
             C.c_int, C.c_double, C.c_uint64, _dp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
            + [_dp] * 9 + [C.POINTER(C.c_uint64)])

    def _chk(self, rc):
        if rc < 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return rc

    def evolve_callbacks(self, method, m, x, v, dt, iterations, units, r=None, rest=None, coll=0, cont=None,
                         rest_from_com=None, each_factor=None, max_steps=0):
        """The reference's evolve(method, continue_ev_if, for_each_bod, for_all_bods) with random_comet's
        callbacks (ref_oracle.cpp, ref_access::evolve_callbacks).  cont: (min_max_cor, probing_iters)
        or None; rest_from_com: (min_cor, max_cor, scale_factor, n_exp, com3, mass_weighted) or None;
        each_factor: velocity scale of for_each_bod, or None.  Returns x, v, rest, steps, com."""
        n = len(m)
        xo, vo, ro = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n)
        r = _c3(np.zeros(n) if r is None else r)
        rest = _c3(np.ones(n) if rest is None else rest)
        mmc, probing = cont if cont is not None else (0.0, 0)
        mn, mx, sc, ne, com, mw = rest_from_com if rest_from_com is not None else (0.0, 1.0, 1.0, 1.0, (0, 0, 0), 0)
        com = np.ascontiguousarray(np.asarray(com, dtype=np.float64).copy())
        steps = C.c_uint64()
        self._chk(self.lib.ref_evolve_callbacks(
            method, coll, n, _c3(m), r, rest, _c3(x), _c3(v), dt, iterations, units.encode(),
            1 if cont is not None else 0, mmc, probing, 1 if rest_from_com is not None else 0, mn, mx, sc, ne,
            int(mw), 1 if each_factor is not None else 0, each_factor or 1.0, max_steps, com, xo, vo, ro,
            C.byref(steps)))
        return xo.reshape(n, 3), vo.reshape(n, 3), ro, steps.value, com

    def evolve_record_callbacks(self, method, m, x, v, dt, iterations, units, mem_freq, r=None, rest=None, coll=0,
                                cont=None, rest_from_com=None, each_factor=None, max_steps=0, max_frames=None):
        """evolve_callbacks of a system with memFreq = mem_freq (1, 2 or 3): the recordings as
        evolve_record, plus x, v, rest, steps and the carried centre (com)."""
        n = len(m)
        F = max_frames or (max(iterations, max_steps) + 2)
        pos, vel = np.zeros(F * n * 3), np.zeros(F * n * 3)
        ke, pe, en, tot = np.zeros(F * n), np.zeros(F * n), np.zeros(F * n), np.zeros(F * 3)
        xo, vo, ro = np.zeros(3 * n), np.zeros(3 * n), np.zeros(n)
        pf, ef = C.c_int(), C.c_int()
        r = _c3(np.zeros(n) if r is None else r)
        rest = _c3(np.ones(n) if rest is None else rest)
        mmc, probing = cont if cont is not None else (0.0, 0)
        mn, mx, sc, ne, com, mw = rest_from_com if rest_from_com is not None else (0.0, 1.0, 1.0, 1.0, (0, 0, 0), 0)
        com = np.ascontiguousarray(np.asarray(com, dtype=np.float64).copy())
        steps = C.c_uint64()
        self._chk(self.lib.ref_evolve_record_callbacks(
            method, coll, mem_freq, n, _c3(m), r, rest, _c3(x), _c3(v), dt, iterations, units.encode(),
            1 if cont is not None else 0, mmc, probing, 1 if rest_from_com is not None else 0, mn, mx, sc, ne,
            int(mw), 1 if each_factor is not None else 0, each_factor or 1.0, max_steps, com, F, C.byref(pf),
            C.byref(ef), pos, vel, ke, pe, en, tot, xo, vo, ro, C.byref(steps)))
        p, e = pf.value, ef.value
        if max(p, e) > F:
            raise RuntimeError(f"{max(p, e)} frames recorded, room for {F}")
        return dict(pos=pos[:p * n * 3].reshape(p, n, 3), vel=vel[:p * n * 3].reshape(p, n, 3),
                    ke=ke[:p * n].reshape(p, n), pe=pe[:e * n].reshape(e, n), energy=en[:e * n].reshape(e, n),
                    tot=tot[:e * 3].reshape(e, 3), x=xo.reshape(n, 3), v=vo.reshape(n, 3), rest=ro,
                    steps=steps.value, com=com)

    def G(self, units="M66743:66740,D1:1,T1:1"):
        g = C.c_longdouble()
        self._chk(self.lib.ref_G(units.encode(), C.byref(g)))
        return g.value

    def units(self, units: str):
        """(True, G as ctypes long double) when the reference accepts the units format, else
        (False, the message of its std::invalid_argument)."""
        g = C.c_longdouble()
        if self.lib.ref_G(units.encode(), C.byref(g)) == 0:
            return True, g
        return False, self.lib.ref_last_error().decode()

    def setters(self, dt, iterations, eps, theta):
        """The reference's set_timestep, set_iterations, set_softening, set_bh_opening_angle results."""
        out = np.zeros(4, np.int32)
        self._chk(self.lib.ref_setters(dt, iterations, eps, theta, out))
        return tuple(bool(b) for b in out)

    def check_option(self, option: int) -> bool:
        return bool(self.lib.ref_check_option(option))

    def construct_dt(self, dt):
        """None when a system with time step dt constructs, else the exception message."""
        if self.lib.ref_construct_dt(dt) == 0:
            return None
        return self.lib.ref_last_error().decode()

    def bench_kdk(self, m, x, v, dt, steps, threads, units="M66743:66740,D1:1,T1:1"):
        """Wall seconds for `threads` concurrent reference evolve(leapfrog_kdk) calls."""
        ns = C.c_longlong()
        self._chk(self.lib.ref_bench_kdk(len(m), _c3(m), _c3(x), _c3(v), dt, steps, units.encode(), threads,
                                         C.byref(ns)))
        return ns.value * 1e-9

    def evolve(self, method, m, x, v, dt, steps, units="M66743:66740,D1:1,T1:1", r=None, rest=None, coll=0):
        n = len(m)
        xo, vo, ao = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
        r = _c3(np.zeros(n) if r is None else r)
        rest = _c3(np.ones(n) if rest is None else rest)
        ns = C.c_longlong()
        self._chk(self.lib.ref_evolve(method, coll, n, _c3(m), r, rest, _c3(x), _c3(v), dt, steps, units.encode(),
                                      xo, vo, ao, C.byref(ns)))
        return xo.reshape(n, 3), vo.reshape(n, 3), ao.reshape(n, 3), ns.value

    def energy(self, m, x, v, units="M66743:66740,D1:1,T1:1"):
        ke, pe = C.c_longdouble(), C.c_longdouble()
        self._chk(self.lib.ref_energy(len(m), _c3(m), _c3(x), _c3(v), units.encode(), C.byref(ke), C.byref(pe)))
        return float(ke.value), float(pe.value)

    def check_overlap_merge(self, m, r, rest, x, v):
        n = len(m)
        no = C.c_int()
        mo, ro, xo, vo = np.zeros(n), np.zeros(n), np.zeros(3 * n), np.zeros(3 * n)
        self._chk(self.lib.ref_check_overlap_merge(n, _c3(m), _c3(r), _c3(rest), _c3(x), _c3(v), C.byref(no), mo,
                                                   ro, xo, vo))
        k = no.value
        return mo[:k], ro[:k], xo.reshape(n, 3)[:k], vo.reshape(n, 3)[:k]

    def merge_pair(self, a12, b12):
        m, r, rest = C.c_double(), C.c_double(), C.c_double()
        x, v, a = np.zeros(3), np.zeros(3), np.zeros(3)
        self._chk(self.lib.ref_merge_pair(_c3(a12), _c3(b12), C.byref(m), C.byref(r), x, v, a, C.byref(rest)))
        return np.concatenate([[m.value, r.value, rest.value], x, v, a])

    def bh_tree_dump(self, x, m, is_float, max_nodes=None):
        n = len(m)
        cap = max_nodes or 8 * n + 64
        depth, body = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
        mass, com, btm, top = np.zeros(cap), np.zeros(3 * cap), np.zeros(3 * cap), np.zeros(3 * cap)
        box = np.zeros(6)
        k = self._chk(self.lib.ref_bh_tree_dump(int(is_float), n, _c3(x), _c3(m), cap, depth, body, mass, com, btm,
                                                top, box))
        if k > cap:
            return self.bh_tree_dump(x, m, is_float, k)
        return dict(n_nodes=k, depth=depth[:k], body=body[:k], mass=mass[:k], com=com.reshape(-1, 3)[:k],
                    btm=btm.reshape(-1, 3)[:k], top=top.reshape(-1, 3)[:k], box=box)

    def bh_acc(self, x, m, theta, eps=0.0, units="M66743:66740,D1:1,T1:1"):
        n = len(m)
        a = np.zeros(3 * n)
        cnt = C.c_uint64()
        self._chk(self.lib.ref_bh_acc(n, _c3(x), _c3(m), theta, eps, units.encode(), a, C.byref(cnt)))
        return a.reshape(n, 3), cnt.value

    def bh_kdk(self, m, x, v, dt, steps, theta, eps=0.0, units="M66743:66740,D1:1,T1:1"):
        n = len(m)
        xo, vo, ao = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
        tb, tw = C.c_longlong(), C.c_longlong()
        self._chk(self.lib.ref_bh_kdk(n, _c3(m), _c3(x), _c3(v), dt, steps, theta, eps, units.encode(), xo, vo, ao,
                                      C.byref(tb), C.byref(tw)))
        return xo.reshape(n, 3), vo.reshape(n, 3), ao.reshape(n, 3), tb.value, tw.value

    def bh_s_coll(self, m, r, rest, x, v):
        """One reference bh_s_coll (gregsys.hpp:631-688) on a T=double tree built at x."""
        n = len(m)
        vo = np.zeros(3 * n)
        self._chk(self.lib.ref_bh_s_coll(n, _c3(m), _c3(r), _c3(rest), _c3(x), _c3(v), vo))
        return vo.reshape(n, 3)

    def bh_kdk_coll(self, m, r, rest, x, v, dt, steps, theta, units="M66743:66740,D1:1,T1:1"):
        """ref_bh_kdk with the reference's bh_s_coll after every full kick."""
        n = len(m)
        xo, vo = np.zeros(3 * n), np.zeros(3 * n)
        self._chk(self.lib.ref_bh_kdk_coll(n, _c3(m), _c3(r), _c3(rest), _c3(x), _c3(v), dt, steps, theta,
                                           units.encode(), xo, vo))
        return xo.reshape(n, 3), vo.reshape(n, 3)

    NSYS_KINDS = {"ddd": 0, "fff": 1, "lll": 2, "ffd": 3}

    def to_nsys(self, kind, m, r, rest, x, v, dt, steps, path, units="M66743:66740,D1:1,T1:1"):
        """system<M,R,T>::to_nsys after `steps` leapfrog KDK steps; kind "ddd", "fff", "lll" or
        "ffd" names M, R, T (double, float, long double).  Returns the bytes written."""
        nb = C.c_longlong()
        self._chk(self.lib.ref_to_nsys(self.NSYS_KINDS[kind], len(m), _c3(m), _c3(r), _c3(rest), _c3(x), _c3(v), dt,
                                       steps, units.encode(), str(path).encode(), C.byref(nb)))
        return nb.value

    def load_nsys(self, kind, path, check=True, max_n=1 << 20, alloc_chunks=False):
        """The system<M,R,T>(path, alloc_chunks, check) constructor.  Returns (status, message,
        state dict): status 0, -1 (nsys_load_error), -2 (nsys_format_error) or -3 (another
        exception).  alloc_chunks defaults to False: with True the reference crashes on a NaN/Inf
        chunk (it deletes its stream twice)."""
        k = max_n
        m, r, rest = np.zeros(k), np.zeros(k), np.zeros(k)
        x, v = np.zeros(3 * k), np.zeros(3 * k)
        n, te, dt, G = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        rc = self.lib.ref_load_nsys(self.NSYS_KINDS[kind], str(path).encode(), int(alloc_chunks), int(check), k,
                                    C.byref(n), m, r, rest, x, v, C.byref(te), C.byref(dt), C.byref(G))
        if rc:
            return rc, self.lib.ref_last_error().decode(), None
        nn = n.value
        return 0, "", dict(m=m[:nn], r=r[:nn], rest=rest[:nn], x=x[:3 * nn].reshape(nn, 3),
                           v=v[:3 * nn].reshape(nn, 3), time=te.value, dt=dt.value, G=G.value)

    def evolve_record(self, method, m, x, v, dt, steps, mem_freq, calls=1, r=None, rest=None, coll=0,
                      units="M66743:66740,D1:1,T1:1", file_freq=0):
        """evolve(method) of a system with memFreq = mem_freq (1, 2 or 3), `calls` times; returns the
        last call's recordings: pos/vel [frames, n, 3], ke [frames, n], pe/energy [pe_frames, n],
        totals [pe_frames, 3] (pe, ke, e), and the final x, v."""
        n = len(m)
        F = steps + 2
        pos, vel = np.zeros(F * n * 3), np.zeros(F * n * 3)
        ke, pe, en, tot = np.zeros(F * n), np.zeros(F * n), np.zeros(F * n), np.zeros(F * 3)
        xo, vo = np.zeros(3 * n), np.zeros(3 * n)
        pf, ef = C.c_int(), C.c_int()
        r = np.zeros(n) if r is None else r
        rest = np.ones(n) if rest is None else rest
        self._chk(self.lib.ref_evolve_record(method, coll, mem_freq, file_freq, n, _c3(m), _c3(r), _c3(rest), _c3(x), _c3(v), dt,
                                             steps,
                                             units.encode(), calls, F, C.byref(pf), C.byref(ef), pos, vel, ke, pe, en,
                                             tot, xo, vo))
        p, e = pf.value, ef.value
        return dict(pos=pos[:p * n * 3].reshape(p, n, 3), vel=vel[:p * n * 3].reshape(p, n, 3),
                    ke=ke[:p * n].reshape(p, n), pe=pe[:e * n].reshape(e, n), energy=en[:e * n].reshape(e, n),
                    tot=tot[:e * 3].reshape(e, 3), x=xo.reshape(n, 3), v=vo.reshape(n, 3))
