"""memFreq recordings (trajectories gregbod.hpp:304-320; per-body and system energies
gregsys.hpp:219-227) against the reference's own recordings (tests/golden, fileFreq = 0: with a
non-zero fileFreq the reference's evolve does not compile).  Every direct method, memFreq 1-3,
collisions off and on, one evolve call or two (the second clears the first's records).

Tolerances: positions and velocities as the FP64 evolve parity (1e-12 / 1e-10 relative to the
largest value); energies 1e-12 relative to the largest magnitude (the engine sums the potential in
FP64, the reference with long-double terms)."""
import numpy as np
import pytest

from gregpackagescpp_b200 import System
from gregpackagescpp_b200.ics import UNITS_G6674

pytestmark = pytest.mark.gpu

METHODS = {"euler": 2, "modified_euler": 4, "midpoint": 8, "leapfrog_kdk": 16, "leapfrog_dkd": 32}


def rel(a, b):
    scale = np.abs(b).max() if b.size else 1.0
    return np.abs(a - b).max() / scale if b.size else 0.0


@pytest.mark.parametrize("coll", [0, 3])
@pytest.mark.parametrize("name", list(METHODS))
def test_recordings_match_reference(gpu, golden, name, coll):
    g = golden
    for f in (1, 2, 3):
        for calls in (1, 2):
            key = f"rec_{name}_{f}_{coll}_{calls}"
            pre = "coll" if coll else "direct"
            kw = dict(r=g["coll_r"], rest=g["coll_rest"], collisions=3) if coll else {}
            s = System(g[f"{pre}_m"], g[f"{pre}_x"], g[f"{pre}_v"], timestep=3600.0, num_iterations=7,
                       units_format=UNITS_G6674, mem_freq=f, **kw)
            for _ in range(calls):
                s.evolve(METHODS[name])
            assert s.positions.shape == g[f"{key}_pos"].shape, key
            assert s.pe.shape == g[f"{key}_pe"].shape, key
            assert rel(s.positions, g[f"{key}_pos"]) < 1e-12, key
            assert rel(s.velocities, g[f"{key}_vel"]) < 1e-10, key
            assert rel(s.kinetic_energies, g[f"{key}_ke"]) < 1e-10, key
            assert rel(s.pe, g[f"{key}_pe"]) < 1e-12, key
            assert rel(s.energies, g[f"{key}_energy"]) < 1e-10, key
            tot = np.stack([s.tot_pe, s.tot_ke, s.tot_e], 1) if len(s.tot_pe) else np.zeros((0, 3))
            assert rel(tot, g[f"{key}_tot"]) < 1e-10, key
            assert rel(s.x, g[f"{key}_x"]) < 1e-12 and rel(s.v, g[f"{key}_v"]) < 1e-10, key


def test_frames_in_upload_order_after_mixed_reordering(gpu):
    """The mixed path reorders bodies on the device; frames are still in upload order (checked
    against the FP64 path's frames at the mixed tolerance)."""
    from gregpackagescpp_b200.ics import plummer
    m, x, v = plummer(3000, 51)
    r = np.full(3000, 1.0)
    a = System(m, x, v, r=r, timestep=3600.0, num_iterations=6, units_format=UNITS_G6674, mem_freq=2,
               collisions=3)
    b = System(m, x, v, r=r, timestep=3600.0, num_iterations=6, units_format=UNITS_G6674, mem_freq=2,
               collisions=3, precision="mixed")
    a.evolve(16)
    b.evolve(16)
    assert a.positions.shape == b.positions.shape == (4, 3000, 3)
    assert rel(b.positions, a.positions) < 1e-9
    assert rel(b.pe, a.pe) < 1e-9


# ---- recordings with evolve callbacks (FUNC_TEMPL_SELECT inside the callback loops) -----------
CB_UNITS = "M1:1,D1:1,T1:1"


def _check_records(s, g, key):
    assert s.positions.shape == g[f"{key}_pos"].shape, key
    assert s.pe.shape == g[f"{key}_pe"].shape, key
    assert rel(s.positions, g[f"{key}_pos"]) < 1e-12, key
    assert rel(s.velocities, g[f"{key}_vel"]) < 1e-10, key
    assert rel(s.kinetic_energies, g[f"{key}_ke"]) < 1e-10, key
    assert rel(s.pe, g[f"{key}_pe"]) < 1e-12, key
    assert rel(s.energies, g[f"{key}_energy"]) < 1e-10, key
    tot = np.stack([s.tot_pe, s.tot_ke, s.tot_e], 1) if len(s.tot_pe) else np.zeros((0, 3))
    assert rel(tot, g[f"{key}_tot"]) < 1e-10, key
    assert rel(s.x, g[f"{key}_x"]) < 1e-12 and rel(s.v, g[f"{key}_v"]) < 1e-10, key


def _cbs_system(g, f):
    return System(g["cbs_m"], g["cbs_x"], g["cbs_v"], r=g["cbs_r"], rest=g["cbs_rest"], timestep=0.25,
                  num_iterations=8, units_format=CB_UNITS, collisions=3, mem_freq=f)


@pytest.mark.parametrize("f", [1, 3])
@pytest.mark.parametrize("name", list(METHODS))
def test_recordings_with_host_callbacks(gpu, golden, name, f):
    """8 collisional steps with host for_all_bods (restitution from the carried centre) and
    for_each_bod (velocities x 0.999): the frames are taken after the collision pass and before
    for_each_bod, every f-th step, as the reference's."""
    g = golden
    _, sf = g["cbs_par"]
    s = _cbs_system(g, f)
    com = g["cbs_com"].copy()
    n = len(g["cbs_m"])

    def for_all(sys_):
        nonlocal com
        acc = com.copy()
        for i in range(n):
            acc = acc + sys_.x[i]
        com = acc / n
        de = np.sum((sys_.x - com) ** 2, axis=1)
        sys_.rest = 1.0 - (1.0 - 0.5) * (de / (de + sf))

    def for_each(sys_, i):
        sys_.v[i] = sys_.v[i] * 0.999

    s.evolve(METHODS[name], None, for_each, for_all)
    _check_records(s, g, f"rcb_{name}_{f}")
    assert rel(s.rest, g[f"rcb_{name}_{f}_rest"]) < 1e-12


@pytest.mark.parametrize("f", [1, 3])
@pytest.mark.parametrize("name", list(METHODS))
def test_recordings_with_device_callbacks(gpu, golden, hooks, name, f):
    """The same steps with the built-in for_all_bods and a user for_each_bod hook on the device: a
    recording evolve runs the callback loop eagerly and reads each frame back when it is made."""
    from gregpackagescpp_b200 import DeviceHook, RestFromCom
    g = golden
    _, sf = g["cbs_par"]
    s = _cbs_system(g, f)
    args = hooks.make_scale_args(0.999)
    try:
        fab = RestFromCom(0.5, 1.0, sf, 2.0, g["cbs_com"])
        s.evolve(METHODS[name], None, DeviceHook(hooks.addr("hook_scale_velocities"), args), fab)
    finally:
        hooks.free_args(args, 0)
    assert s.steps_taken == 8 and not s.callback_stats()["graph_loop"]
    _check_records(s, g, f"rcb_{name}_{f}")
    assert rel(s.rest, g[f"rcb_{name}_{f}_rest"]) < 1e-12
    assert rel(fab.com, g[f"rcb_{name}_{f}_com"]) < 1e-14


@pytest.mark.parametrize("name", ["leapfrog_kdk", "leapfrog_dkd", "euler"])
def test_recordings_with_predicate(gpu, golden, name):
    """continue_ev_if alone (7 probing steps of the rest-below predicate, collisions off), memFreq 2:
    as a host callable and as the device predicate, the reference's records."""
    from gregpackagescpp_b200 import WhileRestBelow
    g = golden
    key = f"rcp_{name}"
    assert int(g[f"{key}_steps"]) == 7
    for device in (False, True):
        s = System(g["cbp_m"], g["cbp_x"], g["cbp_v"], rest=g["cbp_rest_hi"], timestep=3600.0, num_iterations=1000,
                   units_format=UNITS_G6674, mem_freq=2)
        if device:
            s.evolve(METHODS[name], WhileRestBelow(0.5, 7))
        else:
            k = [0]

            def cont():
                k[0] += 1
                return k[0] <= 7

            s.evolve(METHODS[name], cont)
        assert s.steps_taken == 7
        _check_records(s, g, key)
