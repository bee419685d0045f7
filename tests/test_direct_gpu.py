"""Direct-summation evolve on the B200 through the C ABI against the CPU oracle (a restatement of
the reference pinned bit for bit to it) and the reference's own golden vectors.

Bar (FP64): positions and velocities within 1e-12 relative after 10 steps."""
import numpy as np
import pytest

from gregpackagescpp_b200 import System
from gregpackagescpp_b200.ics import UNITS_G6674, plummer

pytestmark = pytest.mark.gpu

METHODS = {"euler": 2, "modified_euler": 4, "midpoint": 8, "leapfrog_kdk": 16, "leapfrog_dkd": 32}
RTOL = 1e-12


def rel_err(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("name", list(METHODS))
def test_methods_vs_reference_golden(gpu, golden, name):
    g = golden
    s = System(g["direct_m"], g["direct_x"], g["direct_v"], timestep=3600.0, num_iterations=10,
               units_format=UNITS_G6674)
    s.evolve(METHODS[name])
    assert rel_err(s.x, g[f"direct_{name}_x"]) < RTOL
    assert rel_err(s.v, g[f"direct_{name}_v"]) < RTOL
    assert rel_err(s.a, g[f"direct_{name}_a"]) < 1e-11


@pytest.mark.parametrize("n", [1, 2, 3, 37, 255, 256, 257, 511, 512, 513, 1500])
@pytest.mark.parametrize("name", ["leapfrog_kdk", "modified_euler"])
def test_ragged_sizes_vs_oracle(gpu, oracle, n, name):
    m, x, v = plummer(n, 100 + n)
    s = System(m, x, v, timestep=3600.0, num_iterations=10, units_format=UNITS_G6674)
    s.evolve(METHODS[name])
    xo, vo, ao = oracle.evolve(METHODS[name], m, x, v, 3600.0, 10, oracle.G(UNITS_G6674))
    assert rel_err(s.x, xo) < RTOL
    assert rel_err(s.v, vo) < RTOL or n == 1


def test_empty_system_is_noop(gpu):
    s = System(np.zeros(0), np.zeros((0, 3)), np.zeros((0, 3)), timestep=1.0, num_iterations=5)
    assert s.evolve(16) == 0
    assert s.num_bodies() == 0


def test_kdk_1024_thousand_steps_energy(gpu, oracle):
    """The reference's CPU configuration: N=1024 Plummer, KDK, dt=3600 s; 100 steps here (the full
    1000-step run is in the benchmark)."""
    m, x, v = plummer(1024, 1)
    s = System(m, x, v, timestep=3600.0, num_iterations=100, units_format=UNITS_G6674)
    ke0, pe0, _, _ = s.energy()
    s.evolve(16)
    ke1, pe1, p1, _ = s.energy()
    xo, vo, _ = oracle.evolve(16, m, x, v, 3600.0, 100, oracle.G(UNITS_G6674))
    assert rel_err(s.x, xo) < 1e-10
    assert abs((ke1 + pe1) - (ke0 + pe0)) / abs(ke0 + pe0) < 1e-6


def test_energy_over_1000_steps_vs_reference(gpu):
    """The reference's own evolve(leapfrog_kdk) and calc_energy (gregsys.hpp:608-630) next to the
    FP64 GPU path over 1000 steps of dt = 3600 s at N = 2048: the two energies agree at step 0 and
    at step 1000, so the drift |dE/E| the GPU path shows is the integrator's (the reference drifts
    by the same amount), not an error of the GPU arithmetic."""
    from oracle.oracle import RefOracle
    if not RefOracle.available():
        pytest.skip("the reference-backed oracle library was not built here")
    ref = RefOracle()
    m, x, v = plummer(2048, 2)
    s = System(m, x, v, timestep=3600.0, num_iterations=1000, units_format=UNITS_G6674)
    ke0, pe0, _, _ = s.energy()
    rk0, rp0 = ref.energy(m, x, v, UNITS_G6674)
    s.evolve(16)
    ke1, pe1, _, _ = s.energy()
    xr, vr, _, _ = ref.evolve(16, m, x, v, 3600.0, 1000, UNITS_G6674)
    rk1, rp1 = ref.energy(m, xr, vr, UNITS_G6674)
    e0, e1, r0, r1 = ke0 + pe0, ke1 + pe1, rk0 + rp0, rk1 + rp1
    assert abs(e0 - r0) <= 1e-13 * abs(r0), (e0, r0)
    drift_gpu, drift_ref = (e1 - e0) / abs(e0), (r1 - r0) / abs(r0)
    print(f"|dE/E| over 1000 steps: GPU {drift_gpu:.6e}, reference {drift_ref:.6e}")
    assert abs(e1 - r1) <= 1e-9 * abs(r1), (drift_gpu, drift_ref)


def test_energy_diagnostic_vs_oracle(gpu, oracle, golden):
    g = golden
    s = System(g["direct_m"], g["direct_x"], g["direct_v"], units_format=UNITS_G6674)
    ke, pe, p, com = s.energy()
    assert abs(ke - float(g["energy_ke"])) <= 1e-13 * abs(ke)
    assert abs(pe - float(g["energy_pe"])) <= 1e-13 * abs(pe)


def test_mixed_acceleration_error(gpu):
    """Mixed path: relative acceleration error against the FP64 path (bar: 1e-6, RMS over bodies)."""
    m, x, v = plummer(16384, 21)
    s64 = System(m, x, v, units_format=UNITS_G6674)
    a64 = s64.accelerations()
    smx = System(m, x, v, units_format=UNITS_G6674, precision="mixed")
    amx = smx.accelerations()
    rel = np.linalg.norm(amx - a64, axis=1) / np.linalg.norm(a64, axis=1)
    rms = float(np.sqrt((rel ** 2).mean()))
    assert rms < 1e-6, (rms, float(np.median(rel)), float(rel.max()))


def test_mixed_kdk_tracks_fp64(gpu):
    m, x, v = plummer(4096, 22)
    a = System(m, x, v, timestep=3600.0, num_iterations=20, units_format=UNITS_G6674)
    b = System(m, x, v, timestep=3600.0, num_iterations=20, units_format=UNITS_G6674, precision="mixed")
    a.evolve(16)
    b.evolve(16)
    assert rel_err(b.x, a.x) < 1e-9
    assert rel_err(b.v, a.v) < 1e-6


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_every_force_variant(gpu, prec):
    """Each force-kernel variant, pinned on the handle, against the FP64 default (FP64 variants to
    1e-13 relative, mixed ones to the mixed bar of 1e-6 RMS), on a ragged N (above the size up to
    which FP64 evaluations take the fused single-launch kernel instead of the variants)."""
    import ctypes as C

    from gregpackagescpp_b200 import _lib
    L = _lib.load()
    m, x, v = plummer(5001, 23)
    want = System(m, x, v, units_format=UNITS_G6674).accelerations()
    p = _lib.PREC_MIXED if prec == "mixed" else _lib.PREC_F64
    count = C.c_int()
    _lib.check(L.gtd_direct_variant_count(p, C.byref(count)))
    assert count.value >= 1
    s = System(m, x, v, units_format=UNITS_G6674, precision=prec)
    for var in range(count.value):
        _lib.check(L.gtd_system_set_direct_variant(s._h, var))
        got = s.accelerations()
        rel = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
        if prec == "f64":
            assert rel.max() < 1e-13, (var, float(rel.max()))
        else:
            assert np.sqrt((rel ** 2).mean()) < 1e-6, (var, float(np.sqrt((rel ** 2).mean())))
    assert L.gtd_system_set_direct_variant(s._h, count.value) == _lib.ERR_INVALID_ARGUMENT


def test_autotune_result_reaches_other_handles(gpu):
    """gtd_system_autotune_direct remembers its choice for the process: a new handle of the same
    precision and size class computes bit-identically to a handle pinned to that variant, and so
    does a pinned handle after unpinning."""
    import ctypes as C

    from gregpackagescpp_b200 import _lib
    L = _lib.load()
    m, x, v = plummer(5000, 24)
    a = System(m, x, v, units_format=UNITS_G6674, precision="mixed")
    a.accelerations()  # uploads the bodies
    best = C.c_int()
    _lib.check(L.gtd_system_autotune_direct(a._h, 1, C.byref(best), None))
    pinned = System(m, x, v, units_format=UNITS_G6674, precision="mixed")
    _lib.check(L.gtd_system_set_direct_variant(pinned._h, best.value))
    fresh = System(m, x, v, units_format=UNITS_G6674, precision="mixed")
    assert np.array_equal(fresh.accelerations(), pinned.accelerations())
    other = (best.value + 1) % 9
    _lib.check(L.gtd_system_set_direct_variant(pinned._h, other))
    _lib.check(L.gtd_system_set_direct_variant(pinned._h, -1))  # unpinned: back to the tuned variant
    assert np.array_equal(fresh.accelerations(), pinned.accelerations())


def test_full_size_mixed_accuracy_and_fp64_momentum(gpu):
    """The headline size, N = 262144: the mixed force within the 1e-6 RMS bar of the FP64 one, and
    the FP64 forces' momentum balance sum m_i a_i ~ 0 (pairwise antisymmetry) to 1e-12 of sum m|a|."""
    m, x, v = plummer(262144, 1)
    a64 = System(m, x, v, units_format=UNITS_G6674).accelerations()
    amx = System(m, x, v, units_format=UNITS_G6674, precision="mixed").accelerations()
    rel = np.linalg.norm(amx - a64, axis=1) / np.linalg.norm(a64, axis=1)
    assert np.sqrt((rel ** 2).mean()) < 1e-6
    p = (m[:, None] * a64).sum(0)
    assert np.abs(p).max() / (m * np.linalg.norm(a64, axis=1)).sum() < 1e-12


def _rows_vs_oracle(oracle, m, x, a, rows):
    """Per-row error of accelerations `a` (all bodies) against the oracle's rows: relative to |a_i|
    and relative to the force scale sum_j G m_j / r_ij^2 of the row."""
    want, gross = oracle.direct_acc_rows(m, x, oracle.G(UNITS_G6674), rows, threads=8)
    err = np.linalg.norm(a[rows] - want, axis=1)
    return err / np.linalg.norm(want, axis=1), err / gross


def test_headline_size_vs_oracle_rows(gpu, oracle):
    """N = 262144 (the mixed-precision configuration) against the oracle on 96 seeded rows: the
    FP64 path within 1e-12 relative per body; the mixed path within 1e-6 of each row's force scale
    sum_j G m_j / r_ij^2 (the size of the terms an FP32 sum rounds) and within 1e-6 relative for
    99 % of the rows, with a relative RMS below 2e-7.  Bodies whose acceleration nearly cancels
    (|a_i| a few hundred times below their force scale) can exceed 1e-6 relative to |a_i|."""
    m, x, v = plummer(262144, 1)
    rows = np.random.default_rng(5).choice(len(m), 96, replace=False)
    a64 = System(m, x, v, units_format=UNITS_G6674).accelerations()
    rel64, _ = _rows_vs_oracle(oracle, m, x, a64, rows)
    assert rel64.max() < 1e-12, float(rel64.max())
    amx = System(m, x, v, units_format=UNITS_G6674, precision="mixed").accelerations()
    rel, scaled = _rows_vs_oracle(oracle, m, x, amx, rows)
    assert scaled.max() < 1e-6, float(scaled.max())
    assert np.quantile(rel, 0.99) < 1e-6, float(np.quantile(rel, 0.99))
    assert np.sqrt((rel ** 2).mean()) < 2e-7, float(np.sqrt((rel ** 2).mean()))


def test_mixed_close_pairs_take_precise_path(gpu, oracle):
    """Pairs much closer than their distance from the row's frame centre: with the precise path off
    (near factor 0) their FP32 coordinate rounding shows as a large relative error; with the default
    factor the same bodies meet the 1e-6 bar against the oracle."""
    from gregpackagescpp_b200 import _lib
    m, x, v = plummer(8192, 31)
    rng = np.random.default_rng(6)
    pairs = rng.choice(len(m), 64, replace=False)
    # move 32 bodies next to 32 others, 1e-5 AU apart
    x = x.copy()
    d = rng.normal(size=(32, 3))
    x[pairs[32:]] = x[pairs[:32]] + 1.495978707e6 * d / np.linalg.norm(d, axis=1)[:, None]
    rows = np.sort(pairs)
    errs = {}
    for k in (0.0, 8.0):
        s = System(m, x, v, units_format=UNITS_G6674, precision="mixed")
        _lib.check(s._L.gtd_system_set_mixed_near_factor(s._h, k))
        rel, _ = _rows_vs_oracle(oracle, m, x, s.accelerations(), rows)
        errs[k] = rel
    assert errs[0.0].max() > 1e-5, float(errs[0.0].max())
    assert errs[8.0].max() < 1e-6, float(errs[8.0].max())


@pytest.mark.parametrize("name", list(METHODS))
def test_graph_replayed_steps_are_bit_identical(gpu, name):
    """FP64 steady-state steps run from a captured CUDA graph; with force-kernel timing on, the same
    steps are launched one by one.  Both give bit-identical states (and match the oracle)."""
    from gregpackagescpp_b200 import _lib
    m, x, v = plummer(1024, 61)
    a = System(m, x, v, timestep=3600.0, num_iterations=50, units_format=UNITS_G6674)
    b = System(m, x, v, timestep=3600.0, num_iterations=50, units_format=UNITS_G6674)
    _lib.check(b._L.gtd_system_time_force_kernels(b._h, 1))
    a.evolve(METHODS[name])
    b.evolve(METHODS[name])
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v)


@pytest.mark.parametrize("n", [37, 4096])
def test_graph_replayed_small_n_bit_identical(gpu, n):
    """The one-launch-per-step FP64 kernel replayed from the step graph: 40 graph-replayed KDK
    steps equal 40 steps launched one by one, bit for bit, for an odd N and for N = 4096, whose
    grid (1024 CTAs) is larger than what the GPU holds at once."""
    from gregpackagescpp_b200 import _lib
    m, x, v = plummer(n, 900 + n)
    a = System(m, x, v, timestep=3600.0, num_iterations=40, units_format=UNITS_G6674)
    b = System(m, x, v, timestep=3600.0, num_iterations=40, units_format=UNITS_G6674)
    _lib.check(b._L.gtd_system_time_force_kernels(b._h, 1))
    a.evolve(METHODS["leapfrog_kdk"])
    b.evolve(METHODS["leapfrog_kdk"])
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v)


@pytest.mark.parametrize("n", [1, 2, 31, 1024, 4096, 4097])
def test_fused_small_path_vs_oracle(gpu, oracle, n):
    """FP64 systems up to 4096 bodies evaluate each force with its update in one launch (a warp per
    body); at 4097 the stream-K kernels take over.  Both against the oracle at the FP64 bar."""
    m, x, v = plummer(n, 300 + n)
    s = System(m, x, v, timestep=3600.0, num_iterations=10, units_format=UNITS_G6674)
    s.evolve(METHODS["leapfrog_kdk"])
    xo, vo, _ = oracle.evolve(METHODS["leapfrog_kdk"], m, x, v, 3600.0, 10, oracle.G(UNITS_G6674))
    assert rel_err(s.x, xo) < RTOL
    if n > 1:  # a lone body has no velocity to compare against
        assert rel_err(s.v, vo) < RTOL
