"""Radius-overlap collisions on the B200 through the C ABI.

* Restitution (collisions = 3, s_coll gregsys.hpp:690-914): every integrator with collisions
  against the reference's own golden vectors.
* Merges (body::operator+=, check_overlap scan): against the oracle, including chains of merges
  where the reference's own loop would delete bodies it never merged.
"""
import numpy as np
import pytest

from gregpackagescpp_b200 import OverlappingBodiesError, System
from gregpackagescpp_b200.ics import AU, UNITS_G6674, plummer

pytestmark = pytest.mark.gpu
METHODS = {"euler": 2, "modified_euler": 4, "midpoint": 8, "leapfrog_kdk": 16, "leapfrog_dkd": 32}


@pytest.mark.parametrize("name", list(METHODS))
def test_restitution_vs_reference_golden(gpu, golden, name):
    g = golden
    s = System(g["coll_m"], g["coll_x"], g["coll_v"], r=g["coll_r"], rest=g["coll_rest"], timestep=3600.0,
               num_iterations=5, units_format=UNITS_G6674, collisions=3)
    s.evolve(METHODS[name])
    assert np.abs(s.x - g[f"coll_{name}_x"]).max() / np.abs(g[f"coll_{name}_x"]).max() < 1e-12
    assert np.abs(s.v - g[f"coll_{name}_v"]).max() / np.abs(g[f"coll_{name}_v"]).max() < 1e-10


def test_restitution_vs_oracle_many_steps(gpu, oracle):
    m, x, v = plummer(300, 61)
    r = np.full(300, 0.05 * AU)
    rest = np.random.default_rng(1).uniform(0.0, 1.0, 300)
    s = System(m, x, v, r=r, rest=rest, timestep=3600.0, num_iterations=20, units_format=UNITS_G6674,
               collisions=3)
    s.evolve(16)
    xo, vo, _ = oracle.evolve(16, m, x, v, 3600.0, 20, oracle.G(UNITS_G6674), r=r, rest=rest, coll=3)
    assert np.abs(s.x - xo).max() / np.abs(xo).max() < 1e-11
    assert np.abs(s.v - vo).max() / np.abs(vo).max() < 1e-9


def _cluster(n, seed, rscale):
    """Bodies in a 0.05 AU cube with radii of the order of their spacing times rscale."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, (n, 3)) * 0.05 * AU
    v = rng.normal(0.0, 3e3, (n, 3))
    m = np.exp(rng.uniform(np.log(1e24), np.log(1e28), n))
    r = rscale * 0.02 * AU * n ** (-1.0 / 3.0) * rng.uniform(0.5, 3.0, n)
    rest = rng.uniform(0.3, 1.0, n)
    return m, r, rest, x, v


@pytest.mark.parametrize("n,rscale,pairs", [(500, 1.0, 354), (500, 2.0, 2534), (1200, 2.0, 7260)])
def test_single_pass_vs_oracle(gpu, oracle, n, rscale, pairs):
    """One s_coll pass on dense clusters: 354 and 2534 overlapping pairs (the one-CTA resolution,
    depth-ordered groups) and 7260 (above its 4096-pair capacity: the sequential form), against
    the oracle's restatement of gregsys.hpp:690-914.  An Euler step of dt = 1 s with masses of
    1e-24 of the cluster's leaves gravity below the last bit of the velocities, so the state after
    it is exactly s_coll(x + v, v); restitution only sees mass ratios."""
    m, r, rest, x, v = _cluster(n, 7, rscale)
    x1 = x + v
    d = np.sqrt(((x1[:, None, :] - x1[None, :, :]) ** 2).sum(-1))
    assert np.triu(r[:, None] + r[None, :] > d, 1).sum() == pairs
    m = m * 1e-24
    s = System(m, x, v, r=r, rest=rest, timestep=1.0, num_iterations=1, collisions=3)
    s.evolve(System.euler)
    assert np.array_equal(s.x, x1)
    want = oracle.s_coll(m, r, rest, x1, v)
    assert np.abs(want - v).max() > 1.0  # the pass changes velocities
    assert np.abs(s.v - want).max() / np.abs(want).max() < 1e-13


def test_check_overlap_raises_like_reference(gpu):
    m, x, v = plummer(50, 62)
    x[30] = x[7] + 10.0
    with pytest.raises(OverlappingBodiesError):
        System(m, x, v, r=np.full(50, 100.0), allow_overlapping_bodies=False)


def test_merge_golden_case(gpu, golden):
    """The one case the reference's own merge loop gets right: the last two bodies overlap."""
    g = golden
    s = System(g["ovl_m"], g["ovl_x"], g["ovl_v"], r=g["ovl_r"], rest=g["ovl_rest"], merge_overlapping=True,
               allow_overlapping_bodies=False)
    assert s.num_bodies() == len(g["ovl_out_m"])
    np.testing.assert_array_equal(s.m, g["ovl_out_m"])
    np.testing.assert_allclose(s.r, g["ovl_out_r"], rtol=4e-16)
    np.testing.assert_array_equal(s.x, g["ovl_out_x"])
    np.testing.assert_array_equal(s.v, g["ovl_out_v"])


@pytest.mark.parametrize("n,seed,rad", [(200, 63, 0.2), (1500, 64, 0.08), (3000, 65, 0.05)])
def test_merge_chains_vs_oracle(gpu, oracle, n, seed, rad):
    m, x, v = plummer(n, seed)
    r = np.random.default_rng(seed).uniform(0.2, 1.0, n) * rad * AU
    rest = np.random.default_rng(seed + 1).uniform(0.0, 1.0, n)
    s = System(m, x, v, r=r, rest=rest, merge_overlapping=True, allow_overlapping_bodies=False)
    rows = np.concatenate([m[:, None], r[:, None], rest[:, None], x, v, np.zeros((n, 3))], axis=1)
    want = oracle.merge_overlapping(rows)
    assert len(want) < n - 5  # chains of merges really happen
    assert s.num_bodies() == len(want)
    np.testing.assert_array_equal(s.m, want[:, 0])
    np.testing.assert_allclose(s.r, want[:, 1], rtol=1e-15)
    np.testing.assert_allclose(s.x, want[:, 3:6], rtol=0, atol=1e-15 * np.abs(want[:, 3:6]).max())
    np.testing.assert_allclose(s.v, want[:, 6:9], rtol=0, atol=1e-15 * np.abs(want[:, 6:9]).max())


def test_merging_evolve_conserves_momentum(gpu):
    m, x, v = plummer(400, 66)
    r = np.full(400, 0.03 * AU)
    s = System(m, x, v, r=r, timestep=3600.0, num_iterations=10, units_format=UNITS_G6674, collisions=3,
               merge_overlapping=True)
    p0 = (m[:, None] * v).sum(0)
    s.evolve(16)
    assert s.num_bodies() < 400
    assert abs(s.m.sum() - m.sum()) <= 1e-12 * m.sum()
    p1 = (s.m[:, None] * s.v).sum(0)
    scale = (m[:, None] * np.abs(v)).sum()
    assert np.abs(p1 - p0).max() / scale < 1e-13
