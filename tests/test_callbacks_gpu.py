"""evolve(method, continue_ev_if, for_each_bod, for_all_bods) (gregsys.hpp:2593-3071) against the
reference's own loop run with random_comet's callbacks (gregsys.hpp:1935-1984; fixtures from
tests/golden/make_golden.py, callback_fixtures).

Per step the reference calls continue_ev_if, the update, for_all_bods, the collision pass and
for_each_bod; the restitution a step's collision pass uses is the one that step's for_all_bods set.

Tolerances.  Fixed short runs (8 collisional steps, or collisionless Plummer steps): 1e-12 relative
to the largest coordinate, the FP64 bar.  The comet runs are chaotic, so their state is checked
against the reference's own sensitivity: perturbing its initial positions by 1e-16 (relative)
moves its final state by 3e-8 / 4e-7 (positions / velocities) after the 183 steps of the
equal-mass comet, checked here at 1e-5 / 1e-4, and by 3e-10 / 3e-9 after 131 steps of the
m-weighted one, checked at 1e-7 / 1e-6.  The equal-mass comet ends on step 183 under 24 such
perturbations out of 24, so its end step is checked exactly; the m-weighted one ends anywhere from
step 244 to 368 under them (263 unperturbed), so its full run is checked for an end in that range
only.  The engine's per-step differences are FP64 rounding against the reference's long-double
intermediates."""

import numpy as np
import pytest

from gregpackagescpp_b200 import DeviceHook, RestFromCom, System, WhileRestBelow, _lib
from gregpackagescpp_b200.ics import UNITS_G6674

pytestmark = pytest.mark.gpu

METHODS = {"euler": 2, "modified_euler": 4, "midpoint": 8, "leapfrog_kdk": 16, "leapfrog_dkd": 32}
CB_UNITS = "M1:1,D1:1,T1:1"


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def _comet_system(g, tag, iterations=1000):
    return System(g[f"{tag}_m"], g[f"{tag}_x"], g[f"{tag}_v"], r=g[f"{tag}_r"], rest=g[f"{tag}_rest"], timestep=0.25,
                  num_iterations=iterations, units_format=CB_UNITS, collisions=3)


@pytest.mark.parametrize("tag,weighted", [("cbk", False), ("cbw", True)])
def test_comet_device_callbacks(gpu, golden, tag, weighted):
    """random_comet's evolve stage with both callbacks on the device: the loop runs as CUDA-graph
    chunks (one host wait per 64 steps) and ends where the reference's does (see the module
    docstring for the m-weighted comet)."""
    g = golden
    mmc, sf = g[f"{tag}_par"]
    s = _comet_system(g, tag)
    fab = RestFromCom(0.5, 1.0, sf, 2.0, g[f"{tag}_com"], mass_weighted=weighted)
    s.evolve(System.leapfrog_kdk, WhileRestBelow(mmc, 20), None, fab, max_steps=3000)
    st = s.callback_stats()
    assert st["graph_loop"] and st["host_waits"] == s.steps_taken // 64 + 1
    assert s.time_elapsed == 1000 * 0.25  # iterations * dt, whatever the steps (gregsys.hpp:3069)
    assert _rel(fab.com, g[f"{tag}_como"]) < 1e-9  # the carried centre follows the conserved mean
    if weighted:
        assert 244 <= s.steps_taken <= 368
    else:
        assert s.steps_taken == int(g[f"{tag}_steps"])
        assert _rel(s.x, g[f"{tag}_xo"]) < 1e-5
        assert _rel(s.v, g[f"{tag}_vo"]) < 1e-4
        assert _rel(s.rest, g[f"{tag}_ro"]) < 1e-5
        return
    # the m-weighted comet at step 131, before chaos takes over (a max_steps stop at an odd step)
    s = _comet_system(g, tag)
    fab = RestFromCom(0.5, 1.0, sf, 2.0, g[f"{tag}_com"], mass_weighted=True)
    s.evolve(System.leapfrog_kdk, WhileRestBelow(mmc, 20), None, fab, max_steps=131)
    assert s.steps_taken == int(g["cbw131_steps"]) == 131
    assert _rel(s.x, g["cbw131_xo"]) < 1e-7
    assert _rel(s.v, g["cbw131_vo"]) < 1e-6
    assert _rel(s.rest, g["cbw131_ro"]) < 1e-7
    assert _rel(fab.com, g["cbw131_como"]) < 1e-9


def test_comet_graph_and_eager_bit_identical(gpu, golden):
    """The graph form and the eager form (forced by force-kernel timing) run the same kernels in
    the same order: bit-identical results."""
    g = golden
    mmc, sf = g["cbk_par"]
    out = []
    for eager in (False, True):
        s = _comet_system(g, "cbk")
        s._push()
        _lib.check(s._L.gtd_system_time_force_kernels(s._h, 1 if eager else 0))
        fab = RestFromCom(0.5, 1.0, sf, 2.0, g["cbk_com"])
        s.evolve(System.leapfrog_kdk, WhileRestBelow(mmc, 20), None, fab, max_steps=3000)
        st = s.callback_stats()
        assert st["graph_loop"] == (not eager)
        if eager:
            assert st["host_waits"] == s.steps_taken + 1
        out.append((s.steps_taken, s.x.copy(), s.v.copy(), s.rest.copy(), fab.com.copy()))
    (k0, x0, v0, r0, c0), (k1, x1, v1, r1, c1) = out
    assert k0 == k1
    for a, b in ((x0, x1), (v0, v1), (r0, r1), (c0, c1)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", list(METHODS))
def test_host_callbacks_in_reference_order(gpu, golden, name):
    """Host callables: for_all_bods (rest from the carried centre, numpy) runs inside the step,
    before the collision pass that uses it; for_each_bod scales every velocity after it."""
    g = golden
    mmc, sf = g["cbs_par"]
    s = System(g["cbs_m"], g["cbs_x"], g["cbs_v"], r=g["cbs_r"], rest=g["cbs_rest"], timestep=0.25,
               num_iterations=8, units_format=CB_UNITS, collisions=3)
    com = g["cbs_com"].copy()
    n = len(g["cbs_m"])

    def for_all(sys_):
        nonlocal com
        acc = com.copy()
        for i in range(n):  # the reference's sequential sum
            acc = acc + sys_.x[i]
        com = acc / n
        d = np.sqrt(np.sum((sys_.x - com) ** 2, axis=1))
        de = d ** 2.0
        sys_.rest = 1.0 - (1.0 - 0.5) * (de / (de + sf))

    def for_each(sys_, i):
        sys_.v[i] = sys_.v[i] * 0.999

    s.evolve(METHODS[name], None, for_each, for_all)
    assert _rel(s.x, g[f"cbs_{name}_xo"]) < 1e-12
    assert _rel(s.v, g[f"cbs_{name}_vo"]) < 1e-12
    assert _rel(s.rest, g[f"cbs_{name}_ro"]) < 1e-12
    assert _rel(com, g[f"cbs_{name}_como"]) < 1e-14


@pytest.mark.parametrize("name", list(METHODS))
def test_device_callbacks_every_method(gpu, golden, hooks, name):
    """The same 8 steps with the built-in for_all_bods and a user for_each_bod hook (its own
    kernel, enqueued on the handle's stream) for every direct method."""
    g = golden
    mmc, sf = g["cbs_par"]
    s = System(g["cbs_m"], g["cbs_x"], g["cbs_v"], r=g["cbs_r"], rest=g["cbs_rest"], timestep=0.25,
               num_iterations=8, units_format=CB_UNITS, collisions=3)
    args = hooks.make_scale_args(0.999)
    try:
        fab = RestFromCom(0.5, 1.0, sf, 2.0, g["cbs_com"])
        s.evolve(METHODS[name], None, DeviceHook(hooks.addr("hook_scale_velocities"), args), fab)
    finally:
        hooks.free_args(args, 0)
    assert s.steps_taken == 8 and s.callback_stats()["graph_loop"]
    assert _rel(s.x, g[f"cbs_{name}_xo"]) < 1e-12
    assert _rel(s.v, g[f"cbs_{name}_vo"]) < 1e-12
    assert _rel(s.rest, g[f"cbs_{name}_ro"]) < 1e-12
    assert _rel(fab.com, g[f"cbs_{name}_como"]) < 1e-14


def test_predicate_around_graph_chunks(gpu, golden):
    """The predicate alone: 0, 63, 64 and 70 steps (inside, at and across the 64-step chunks) and a
    predicate that never ends stopped by max_steps at an odd step (the position buffers' parity),
    for a method with one buffer flip per step (KDK, Euler) and one with two (DKD)."""
    g = golden
    for key in g["cbp_cases"]:
        key = str(key)
        parts = key.split("_")  # cbp_<method>_<probing>_<lo>_<cap>
        meth_name, (probing, lo, cap) = "_".join(parts[1:-3]), parts[-3:]
        s = System(g["cbp_m"], g["cbp_x"], g["cbp_v"], rest=g["cbp_rest_lo"] if lo == "1" else g["cbp_rest_hi"],
                   timestep=3600.0, num_iterations=1000, units_format=UNITS_G6674)
        s.evolve(METHODS[meth_name], WhileRestBelow(0.5, int(probing)), max_steps=int(cap))
        assert s.steps_taken == int(g[f"{key}_steps"]), key
        if s.steps_taken:
            assert _rel(s.x, g[f"{key}_xo"]) < 1e-11, key
            assert _rel(s.v, g[f"{key}_vo"]) < 1e-11, key
        else:
            assert np.array_equal(s.x, g["cbp_x"]) and np.array_equal(s.v, g["cbp_v"]), key


def test_user_continue_hook(gpu, golden, hooks):
    """A user continue_ev_if hook (a device counter) true for 70 evaluations: the reference's 70
    steps, across a chunk boundary; a second evolve with the counter reset repeats it."""
    g = golden
    args = hooks.make_count_args(70)
    try:
        for _ in range(2):
            s = System(g["cbp_m"], g["cbp_x"], g["cbp_v"], timestep=3600.0, num_iterations=1000,
                       units_format=UNITS_G6674)
            assert hooks.reset_count_args(args) == 0
            s.evolve(System.leapfrog_kdk, DeviceHook(hooks.addr("hook_count_steps"), args))
            assert s.steps_taken == 70
            assert _rel(s.x, g["cbp_leapfrog_kdk_70_0_0_xo"]) < 1e-11
            assert _rel(s.v, g["cbp_leapfrog_kdk_70_0_0_vo"]) < 1e-11
    finally:
        hooks.free_args(args, 1)


def test_failing_hook_and_mixing(gpu, golden, hooks):
    g = golden
    s = System(g["cbp_m"], g["cbp_x"], g["cbp_v"], timestep=3600.0, num_iterations=10, units_format=UNITS_G6674)
    with pytest.raises(_lib.CallbackError):
        s.evolve(System.leapfrog_kdk, None, None, DeviceHook(hooks.addr("hook_fail")))
    with pytest.raises(TypeError):
        s.evolve(System.leapfrog_kdk, lambda: False, None, RestFromCom(0.5, 1.0, 1.0, 2.0, (0, 0, 0)))

    def bad(sys_):
        raise KeyError("from a host callback")
    with pytest.raises(KeyError):
        s.evolve(System.leapfrog_kdk, None, None, bad)
    # the handle is still usable afterwards
    s.evolve(System.leapfrog_kdk)
    assert np.isfinite(s.x).all()


def test_barnes_hut_ignores_callbacks(gpu, golden):
    """The Barnes-Hut branch calls no callback and runs `iterations` steps (gregsys.hpp:2893-2945)."""
    g = golden
    a = System(g["bhk_m"], g["bhk_x"], g["bhk_v"], timestep=3600.0, num_iterations=5, units_format=UNITS_G6674)
    b = System(g["bhk_m"], g["bhk_x"], g["bhk_v"], timestep=3600.0, num_iterations=5, units_format=UNITS_G6674)
    meth = System.leapfrog_kdk | System.barnes_hut
    a.evolve(meth)
    b.evolve(meth, WhileRestBelow(2.0, 0))  # would stop at once if it were evaluated
    c = System(g["bhk_m"], g["bhk_x"], g["bhk_v"], timestep=3600.0, num_iterations=5, units_format=UNITS_G6674)
    c.evolve(meth, lambda: False)
    for s in (b, c):
        assert np.array_equal(s.x, a.x) and np.array_equal(s.v, a.v)


def _counting(k):
    """A host predicate true for the first k evaluations."""
    state = {"n": 0}

    def cont():
        state["n"] += 1
        return state["n"] <= k
    return cont


@pytest.mark.parametrize("precision,coll,merge,graph", [("f64", 3, True, False), ("mixed", 0, False, False),
                                                         ("mixed", 3, False, True)])
def test_device_predicate_matches_host_predicate(gpu, precision, coll, merge, graph):
    """The same loop driven by the device predicate and by a host callable is bit-identical: with
    merging collisions (the eager form: the body count changes), with the mixed-precision path and
    its periodic Morton reorder (eager form), and with mixed precision and overlap collisions (the
    graph form)."""
    from gregpackagescpp_b200.ics import AU, plummer
    m, x, v = plummer(3000 if precision == "mixed" else 400, 66)
    r = np.full(len(m), 0.03 * AU if merge else 0.02 * AU)
    kw = dict(r=r, timestep=3600.0, num_iterations=1000, units_format=UNITS_G6674, collisions=coll,
              merge_overlapping=merge, precision=precision)
    a = System(m, x, v, **kw)
    a.evolve(System.leapfrog_kdk, WhileRestBelow(0.0, 40))  # rest never below 0: exactly 40 steps
    st = a.callback_stats()
    assert a.steps_taken == 40 and st["graph_loop"] == graph
    assert st["host_waits"] == (1 if graph else 41)
    b = System(m, x, v, **kw)
    b.evolve(System.leapfrog_kdk, _counting(40))
    if merge:
        assert len(a.m) < len(m)  # merges happened
    assert len(a.m) == len(b.m)
    for p, q in ((a.m, b.m), (a.x, b.x), (a.v, b.v)):
        assert np.array_equal(p, q)
