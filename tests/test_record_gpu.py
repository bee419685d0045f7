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
