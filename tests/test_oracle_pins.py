"""The CPU oracle (oracle/nbody_oracle.c) against golden vectors produced by the unmodified
reference headers (tests/golden/make_golden.py).  Direct summation, collisions, energy, merges
and the octree topology must agree bit for bit; Barnes-Hut accelerations to 1e-12 (the oracle
sums moments in a different order than calc_com)."""
import ctypes as C

import numpy as np
import pytest

from gregpackagescpp_b200.ics import UNITS_G6674

METHODS = {"euler": 2, "modified_euler": 4, "midpoint": 8, "leapfrog_kdk": 16, "leapfrog_dkd": 32}


def test_G_matches_reference(oracle, golden):
    assert oracle.G(UNITS_G6674).value == float(golden["G_6674"])
    assert oracle.G("M1:1,D1:1,T1:1").value == float(golden["G_SI"])
    assert oracle.G("M3:7,D2:5,T11:13").value == float(golden["G_odd"])


@pytest.mark.parametrize("name", list(METHODS))
def test_direct_methods_bit_exact(oracle, golden, name):
    g = golden
    x, v, a = oracle.evolve(METHODS[name], g["direct_m"], g["direct_x"], g["direct_v"], 3600.0, 10,
                            oracle.G(UNITS_G6674))
    assert np.array_equal(x, g[f"direct_{name}_x"])
    assert np.array_equal(v, g[f"direct_{name}_v"])
    assert np.array_equal(a, g[f"direct_{name}_a"])


def test_direct_odd_n(oracle, golden):
    g = golden
    x, v, a = oracle.evolve(16, g["odd_m"], g["odd_x"], g["odd_v"], 3600.0, 10, oracle.G(UNITS_G6674))
    assert np.array_equal(x, g["odd_kdk_x"]) and np.array_equal(v, g["odd_kdk_v"])


@pytest.mark.parametrize("name", list(METHODS))
def test_collisions_bit_exact(oracle, golden, name):
    g = golden
    x, v, _ = oracle.evolve(METHODS[name], g["coll_m"], g["coll_x"], g["coll_v"], 3600.0, 5, oracle.G(UNITS_G6674),
                            r=g["coll_r"], rest=g["coll_rest"], coll=3)
    assert np.array_equal(x, g[f"coll_{name}_x"])
    assert np.array_equal(v, g[f"coll_{name}_v"])
    # the fixture really exercises collisions
    x0, v0, _ = oracle.evolve(METHODS[name], g["coll_m"], g["coll_x"], g["coll_v"], 3600.0, 5, oracle.G(UNITS_G6674))
    assert not np.array_equal(v0, g[f"coll_{name}_v"])


def test_energy_bit_exact(oracle, golden):
    ke, pe = oracle.energy(golden["direct_m"], golden["direct_x"], golden["direct_v"], oracle.G(UNITS_G6674))
    assert ke == float(golden["energy_ke"]) and pe == float(golden["energy_pe"])


def test_merge_pair_bit_exact(oracle, golden):
    for a, b, want in zip(golden["merge_a"], golden["merge_b"], golden["merge_out"]):
        got = oracle.merge_pair(a, b)
        # layout: oracle row {m,r,rest,x3,v3,a3}; reference dump {m,r,rest,x3,v3,a3}
        assert np.array_equal(got, want)


def test_check_overlap_merge(oracle, golden):
    g = golden
    rows = np.concatenate([g["ovl_m"][:, None], g["ovl_r"][:, None], g["ovl_rest"][:, None], g["ovl_x"], g["ovl_v"],
                           np.zeros((len(g["ovl_m"]), 3))], axis=1)
    out = oracle.merge_overlapping(rows)
    assert len(out) == len(g["ovl_out_m"]) == len(g["ovl_m"]) - 1
    assert np.array_equal(out[:, 0], g["ovl_out_m"])
    assert np.array_equal(out[:, 1], g["ovl_out_r"])
    assert np.array_equal(out[:, 3:6], g["ovl_out_x"])
    assert np.array_equal(out[:, 6:9], g["ovl_out_v"])


@pytest.mark.parametrize("isf", [0, 1])
def test_octree_topology_matches_reference(oracle, golden, isf):
    g = golden
    t = oracle.bh_tree(g["bh_x"], g["bh_m"], isf)
    try:
        assert t["n_nodes"] == len(g[f"bh_tree{isf}_depth"])
        assert np.array_equal(t["depth"], g[f"bh_tree{isf}_depth"])
        leaf_body = np.where(t["is_leaf"] == 1, t["perm"][t["first"]], -1)
        assert np.array_equal(leaf_body, g[f"bh_tree{isf}_body"])
        assert np.array_equal(t["box"], g[f"bh_tree{isf}_box"])
        assert np.array_equal(t["width"], g[f"bh_tree{isf}_width"])
        if isf == 0:
            assert np.array_equal(t["mass"][t["is_leaf"] == 1], g["bh_tree0_mass"][t["is_leaf"] == 1])
            np.testing.assert_allclose(t["com"], g["bh_tree0_com"], rtol=0, atol=1e-12 * np.abs(g["bh_x"]).max())
    finally:
        oracle.bh_free(t)


def test_barnes_hut_acc_matches_reference_walk(oracle, golden):
    g = golden
    t = oracle.bh_tree(g["bh_x"], g["bh_m"], 0)
    try:
        a, cnt = oracle.bh_acc(t, g["bh_x"], g["bh_m"], 0, 0.5, 0.0, 6.674e-11)
    finally:
        oracle.bh_free(t)
    assert int(cnt.sum()) == int(g["bh_count"])
    rel = np.linalg.norm(a - g["bh_acc"], axis=1) / np.linalg.norm(g["bh_acc"], axis=1)
    assert rel.max() < 1e-12


def test_bh_s_coll_bit_exact(oracle, golden):
    """bh_s_coll (gregsys.hpp:631-688): leaf-cube neighbours, ascending distance, restitution
    impulses; the oracle on its own T=double tree against the reference's pass."""
    g = golden
    t = oracle.bh_tree(g["bhc_x"], g["bhc_m"], 0)
    try:
        v = oracle.bh_s_coll(t, g["bhc_m"], g["bhc_r"], g["bhc_rest"], g["bhc_x"], g["bhc_v"], 0)
    finally:
        oracle.bh_free(t)
    assert np.array_equal(v, g["bhc_v_out"])
    assert (np.abs(g["bhc_v_out"] - g["bhc_v"]).max(1) > 0).sum() > 50  # the fixture really collides
