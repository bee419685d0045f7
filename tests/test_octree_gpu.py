"""Barnes-Hut on the B200 through the C ABI.

* Topology: Morton codes, slot order, every node's depth / leaf flag / range / skip link / cell
  width and the FP64 centres of mass are bit-exact against the host rebuild (oracle/), which is
  itself pinned to the reference's pointer octree (tests/test_oracle_pins.py).
* Walk: per-body interaction counts equal the host rebuild's exactly; accelerations match the
  reference's corrected walk (FP64 tree) to 1e-12 and the FP32 walk to 1e-5.
"""
import numpy as np
import pytest

from gregpackagescpp_b200 import IndistinguishableBodies, InvalidBodyPlacement, System
from gregpackagescpp_b200.ics import AU, UNITS_G6674, plummer, two_plummer

pytestmark = pytest.mark.gpu
G = 6.674e-11


def gpu_tree(m, x, tree_float):
    s = System(m, x, np.zeros_like(x), units_format=UNITS_G6674)
    s.bh_build(tree_float)
    return s, s.bh_tree()


def compare_tree(t, o):
    assert t["n_nodes"] == o["n_nodes"]
    assert t["n_leaves"] == o["n_leaves"]
    assert np.array_equal(t["box"], o["box"])
    assert np.array_equal(t["code"], o["code"])
    assert np.array_equal(t["perm"], o["perm"])
    for f in ("depth", "is_leaf", "first", "count", "skip", "width", "mass"):
        assert np.array_equal(t[f], o[f]), f
    assert np.array_equal(t["com"], o["com"])


@pytest.mark.parametrize("tree_float", [0, 1])
@pytest.mark.parametrize("n,seed", [(2, 1), (3, 2), (100, 3), (2000, 7), (20000, 9), (65537, 10)])
def test_topology_bit_exact_vs_host_rebuild(gpu, oracle, tree_float, n, seed):
    m, x, _ = plummer(n, seed)
    s, t = gpu_tree(m, x, tree_float)
    o = oracle.bh_tree(x, m, tree_float)
    try:
        compare_tree(t, o)
    finally:
        oracle.bh_free(o)


def test_topology_two_spheres(gpu, oracle):
    m, x, _ = two_plummer(50000, 4)
    s, t = gpu_tree(m, x, 1)
    o = oracle.bh_tree(x, m, 1)
    try:
        compare_tree(t, o)
    finally:
        oracle.bh_free(o)


@pytest.mark.parametrize("isf", [0, 1])
def test_topology_vs_reference_golden(gpu, golden, isf):
    g = golden
    s, t = gpu_tree(g["bh_m"], g["bh_x"], isf)
    assert t["n_nodes"] == len(g[f"bh_tree{isf}_depth"])
    assert np.array_equal(t["depth"], g[f"bh_tree{isf}_depth"])
    leaf_body = np.where(t["is_leaf"] == 1, t["perm"][t["first"]], -1)
    assert np.array_equal(leaf_body, g[f"bh_tree{isf}_body"])
    assert np.array_equal(t["box"], g[f"bh_tree{isf}_box"])
    assert np.array_equal(t["width"], g[f"bh_tree{isf}_width"])


def test_fp64_walk_vs_reference_golden(gpu, golden, oracle):
    g = golden
    s = System(g["bh_m"], g["bh_x"], np.zeros_like(g["bh_x"]), units_format=UNITS_G6674)
    s.set_bh_opening_angle(0.5)
    a, cnt = s.bh_accelerations(tree_float=False)
    assert int(cnt.sum()) == int(g["bh_count"])
    rel = np.linalg.norm(a - g["bh_acc"], axis=1) / np.linalg.norm(g["bh_acc"], axis=1)
    assert rel.max() < 1e-12
    t = oracle.bh_tree(g["bh_x"], g["bh_m"], 0)
    try:
        _, ocnt = oracle.bh_acc(t, g["bh_x"], g["bh_m"], 0, 0.5, 0.0, G)
    finally:
        oracle.bh_free(t)
    assert np.array_equal(cnt, ocnt)


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("n,theta", [(5000, 0.5), (30000, 0.5), (30000, 1.0), (3000, 0.0)])
def test_fp32_walk_vs_host_rebuild(gpu, oracle, n, theta, variant):
    m, x, _ = plummer(n, 30 + n)
    s = System(m, x, np.zeros_like(x), units_format=UNITS_G6674)
    s.set_bh_opening_angle(theta)
    s.set_bh_walk_variant(variant)
    a, cnt = s.bh_accelerations(tree_float=True)
    t = oracle.bh_tree(x, m, 1)
    try:
        ao, ocnt = oracle.bh_acc(t, x, m, 1, theta, 0.0, G)
    finally:
        oracle.bh_free(t)
    assert np.array_equal(cnt, ocnt)
    rel = np.linalg.norm(a - ao, axis=1) / np.linalg.norm(ao, axis=1)
    assert np.sqrt((rel ** 2).mean()) < 1e-5 and rel.max() < 1e-3


def test_walk_record_layouts_bit_identical(gpu):
    """Interleaved and separate node records change how the warp fetches a node, not what any body
    computes: interaction counts and accelerations agree bit for bit (odd N)."""
    m, x, _ = plummer(20001, 77)
    out = []
    for variant in (0, 1):
        s = System(m, x, np.zeros_like(x), units_format=UNITS_G6674)
        s.set_bh_walk_variant(variant)
        out.append(s.bh_accelerations(tree_float=True))
    for o in out[1:]:
        assert np.array_equal(out[0][1], o[1])
        assert np.array_equal(out[0][0], o[0])
    with pytest.raises(ValueError):
        System(m, x, np.zeros_like(x), units_format=UNITS_G6674).set_bh_walk_variant(3)


@pytest.mark.parametrize("n,theta,eps", [(1, 0.5, 0.0), (2, 0.5, 0.0), (33, 0.5, 0.0), (20001, 0.5, 0.0),
                                         (20001, 0.7, 1e9), (4099, 1.5, 0.0), (4099, 0.2, 0.0)])
def test_list_walk_same_interactions(gpu, oracle, n, theta, eps):
    """The list walk (variant 2) against the per-lane walk (variant 1) and the oracle: every
    body's interaction count equal, accelerations equal up to the order of the FP32 sum.  Odd
    sizes leave a partial last warp; softening changes only the terms; bodies 7 and 8 share a
    depth-21 cell (a bucket leaf of two bodies, 1e5 m apart at 1 AU scale)."""
    if n == 1:
        m, x = np.array([1e30]), np.zeros((1, 3))
    else:
        m, x, _ = plummer(n, 90 + n)
    if n > 8:
        x[8] = x[7] + np.array([1e5, 0.0, 0.0])
    out = []
    for variant in (1, 2):
        s = System(m, x, np.zeros_like(x), units_format=UNITS_G6674)
        s.set_bh_opening_angle(theta)
        if eps:
            s.set_softening(eps)
        s.set_bh_walk_variant(variant)
        if n == 1:
            with pytest.raises(InvalidBodyPlacement):
                s.bh_accelerations(tree_float=True)
            return
        out.append(s.bh_accelerations(tree_float=True))
    (a1, c1), (a2, c2) = out
    assert np.array_equal(c1, c2)
    if n > 8:
        t = s.bh_tree()
        assert (t["count"][t["is_leaf"] == 1] > 1).any()  # the bucket leaf is there
    rel = np.linalg.norm(a2 - a1, axis=1) / np.linalg.norm(a1, axis=1)
    assert np.sqrt((rel ** 2).mean()) < 1e-5 and rel.max() < 1e-3  # the FP32 bar of the walk vs the oracle
    t = oracle.bh_tree(x, m, 1)
    try:
        ao, ocnt = oracle.bh_acc(t, x, m, 1, theta, eps, G)
    finally:
        oracle.bh_free(t)
    assert np.array_equal(c2, ocnt)


def test_theta_zero_is_direct_sum(gpu, oracle):
    """theta = 0 opens every cell: the walk degenerates to direct summation over leaves."""
    m, x, _ = plummer(1500, 41)
    s = System(m, x, np.zeros_like(x), units_format=UNITS_G6674)
    s.set_bh_opening_angle(0.0)
    a, cnt = s.bh_accelerations(tree_float=False)
    assert np.all(cnt == len(m) - 1)
    ad = oracle.direct_acc(m, x, oracle.G(UNITS_G6674))
    rel = np.linalg.norm(a - ad, axis=1) / np.linalg.norm(ad, axis=1)
    assert rel.max() < 1e-12


def test_bh_kdk_vs_reference_golden(gpu, golden):
    g = golden
    s = System(g["bhk_m"], g["bhk_x"], g["bhk_v"], timestep=3600.0, num_iterations=5, units_format=UNITS_G6674)
    s.set_bh_opening_angle(0.5)
    s.bh_tree_float(False)
    s.evolve(System.leapfrog_kdk | System.barnes_hut)
    assert np.abs(s.x - g["bhk_xo"]).max() / np.abs(g["bhk_xo"]).max() < 1e-12
    assert np.abs(s.v - g["bhk_vo"]).max() / np.abs(g["bhk_vo"]).max() < 1e-10


def test_single_body_rejected_like_reference(gpu):
    s = System(np.array([1e30]), np.zeros((1, 3)), np.zeros((1, 3)))
    with pytest.raises(InvalidBodyPlacement):
        s.bh_build(True)


def test_coincident_bodies_rejected(gpu):
    m, x, _ = plummer(100, 5)
    x[17] = x[42]
    s = System(m, x, np.zeros_like(x))
    with pytest.raises(IndistinguishableBodies):
        s.bh_build(False)


def test_nonfinite_position_rejected(gpu):
    m, x, _ = plummer(100, 6)
    x[3, 1] = np.nan
    s = System(m, x, np.zeros_like(x))
    with pytest.raises(InvalidBodyPlacement):
        s.bh_build(True)


def _bh_coll_kdk_oracle(oracle, m, r, rest, x, v, dt, steps, theta, G, is_float):
    """The reference's Barnes-Hut KDK schedule with bh_s_coll after each full kick, from the
    oracle's tree, walk and collision pass."""
    x, v = x.copy(), v.copy()

    def walk():
        t = oracle.bh_tree(x, m, is_float)
        a, _ = oracle.bh_acc(t, x, m, is_float, theta, 0.0, G)
        return t, a

    t, a = walk()
    oracle.bh_free(t)
    v = v + 0.5 * dt * a
    for _ in range(steps):
        x = x + dt * v
        t, a = walk()
        v = v + dt * a
        v = oracle.bh_s_coll(t, m, r, rest, x, v, is_float)
        oracle.bh_free(t)
    return x, v


def test_bh_collisions_vs_reference_golden(gpu, golden):
    """Barnes-Hut KDK with collisions on (bh_s_coll after every full kick) against the reference
    run on the same overlapping cluster, T=double tree."""
    g = golden
    s = System(g["bhck_m"], g["bhck_x"], g["bhck_v"], r=g["bhck_r"], rest=g["bhck_rest"], timestep=3600.0,
               num_iterations=5, units_format=UNITS_G6674, collisions=System.overlap_coll_check)
    s.set_bh_opening_angle(0.5)
    s.bh_tree_float(False)
    s.evolve(System.leapfrog_kdk | System.barnes_hut)
    no = System(g["bhck_m"], g["bhck_x"], g["bhck_v"], r=g["bhck_r"], rest=g["bhck_rest"], timestep=3600.0,
                num_iterations=5, units_format=UNITS_G6674)
    no.set_bh_opening_angle(0.5)
    no.bh_tree_float(False)
    no.evolve(System.leapfrog_kdk | System.barnes_hut)
    vmax = np.abs(g["bhck_vo"]).max()
    assert np.abs(s.x - g["bhck_xo"]).max() / np.abs(g["bhck_xo"]).max() < 1e-12
    assert np.abs(s.v - g["bhck_vo"]).max() / vmax < 1e-10
    assert np.abs(no.v - g["bhck_vo"]).max() / vmax > 1e-3  # the collisions changed the run


@pytest.mark.parametrize("tree_float", [False, True])
def test_bh_collisions_vs_oracle(gpu, oracle, tree_float):
    """The same on a denser cluster, float and double trees, against the oracle's composition.
    Masses of 1e-3..10 kg make gravity negligible, so the float tree's FP32 forces between
    near-coincident bodies (no softening) do not mask what is checked here: the float tree's cells,
    the neighbour order and the FP64 impulses."""
    rng = np.random.default_rng(31)
    n = 1500
    x = rng.uniform(-1.0, 1.0, (n, 3)) * 0.05 * AU
    v = rng.normal(0.0, 3e3, (n, 3))
    m = np.exp(rng.uniform(np.log(1e-3), np.log(10.0), n))
    r = 0.02 * AU * n ** (-1.0 / 3.0) * rng.uniform(0.5, 3.0, n)
    rest = rng.uniform(0.3, 1.0, n)
    s = System(m, x, v, r=r, rest=rest, timestep=3600.0, num_iterations=3, units_format=UNITS_G6674,
               collisions=System.overlap_coll_check)
    s.set_bh_opening_angle(0.5)
    s.bh_tree_float(tree_float)
    s.evolve(System.leapfrog_kdk | System.barnes_hut)
    xo, vo = _bh_coll_kdk_oracle(oracle, m, r, rest, x, v, 3600.0, 3, 0.5, 6.674e-11, tree_float)
    assert np.abs(s.x - xo).max() / np.abs(xo).max() < 1e-12
    assert np.abs(s.v - vo).max() / np.abs(vo).max() < 1e-10
    assert np.abs(vo - v).max() > 1.0  # the collisions changed the velocities


def test_topology_full_size(gpu, oracle):
    """The Barnes-Hut workload's size: two Plummer spheres of 2^21 bodies.  Codes, order, depths,
    skips, widths and FP64 moments bit-exact against the host rebuild, and every body in exactly
    one leaf (counts of the leaves sum to N)."""
    m, x, _ = two_plummer(1 << 21, 1)
    s, t = gpu_tree(m, x, 1)
    o = oracle.bh_tree(x, m, 1)
    try:
        compare_tree(t, o)
        assert int(t["count"][t["is_leaf"] == 1].sum()) == len(m)
    finally:
        oracle.bh_free(o)
