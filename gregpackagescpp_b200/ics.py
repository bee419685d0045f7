"""Seeded synthetic initial conditions for the gtd:: workloads (host side, numpy, FP64, SI units).

These are inputs, not the hot path: they stand in for the reference drivers' generators
(random_comet / hcp_comet, gregsys.hpp:1761-2520), which are not part of the force-and-step path.

* ``plummer``      - Plummer sphere, Aarseth, Henon & Wielen (1974) sampling: radii from the
                     inverted cumulative mass, speeds by von Neumann rejection on
                     q^2 (1 - q^2)^{7/2}, isotropic directions, then a centre-of-mass shift.
* ``two_plummer``  - two equal spheres on a parabolic approach (Barnes-Hut workload).
* ``ensemble``     - many independent few-body systems of uneven size with radii from a constant
                     density (batched collision workload).
* ``comet_stage``  - the collapsing cloud of random_comet's evolve stage and the constants of its
                     callbacks (callback-driven evolve workload).
"""
from __future__ import annotations

import numpy as np

AU = 1.495978707e11
G_DEFAULT = 6.674e-11
# "M66743:66740,D1:1,T1:1" makes the reference's G exactly 66743 * 66740 / 66743 * 1e-15 = 6.674e-11
# (units parse, gregsys.hpp:245-282).
UNITS_G6674 = "M66743:66740,D1:1,T1:1"


def _isotropic(rng: np.random.Generator, n: int) -> np.ndarray:
    cz = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(1.0 - cz * cz)
    return np.stack([s * np.cos(phi), s * np.sin(phi), cz], axis=1)


def plummer(n: int, seed: int, a: float = AU, total_mass: float = 1e30, G: float = G_DEFAULT,
            r_max: float = 50.0):
    """n equal-mass bodies of a Plummer sphere with scale radius ``a`` and mass ``total_mass``.

    Returns (m[n], x[n,3], v[n,3]) in SI, centre of mass at rest at the origin.  Radii beyond
    ``r_max * a`` are redrawn (they hold ~1e-5 of the mass at r_max=50)."""
    rng = np.random.default_rng(seed)
    m = np.full(n, total_mass / n, dtype=np.float64)
    r = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        x1 = rng.uniform(1e-10, 1.0, todo.size)
        rr = 1.0 / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)
        ok = rr <= r_max
        r[todo[ok]] = rr[ok]
        todo = todo[~ok]
    pos = _isotropic(rng, n) * (r * a)[:, None]
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        qq = rng.uniform(0.0, 1.0, todo.size)
        yy = rng.uniform(0.0, 0.1, todo.size)
        ok = yy < qq * qq * (1.0 - qq * qq) ** 3.5
        q[todo[ok]] = qq[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0 * G * total_mass / a) * (1.0 + r * r) ** -0.25
    vel = _isotropic(rng, n) * (q * vesc)[:, None]
    pos -= (m[:, None] * pos).sum(0) / m.sum()
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    return m, np.ascontiguousarray(pos), np.ascontiguousarray(vel)


def two_plummer(n_each: int, seed: int, a: float = AU, mass_each: float = 1e30, sep: float = 20 * AU,
                peri: float = 2 * AU, G: float = G_DEFAULT):
    """Two Plummer spheres centred at -/+ sep/2 on x, on a parabolic orbit with pericentre ``peri``.

    Relative speed sqrt(2 G (2M) / sep); the angular momentum sqrt(2 G (2M) peri) sets the
    tangential (y) component, the rest is radial (approach along -x / +x)."""
    m1, x1, v1 = plummer(n_each, seed, a, mass_each, G)
    m2, x2, v2 = plummer(n_each, seed + 1000003, a, mass_each, G)
    mu = G * 2.0 * mass_each
    vrel = np.sqrt(2.0 * mu / sep)
    vt = np.sqrt(2.0 * mu * peri) / sep
    vr = np.sqrt(max(vrel * vrel - vt * vt, 0.0))
    x1[:, 0] -= sep / 2
    x2[:, 0] += sep / 2
    v1 += np.array([+vr / 2, +vt / 2, 0.0])
    v2 += np.array([-vr / 2, -vt / 2, 0.0])
    return (np.concatenate([m1, m2]), np.ascontiguousarray(np.concatenate([x1, x2])),
            np.ascontiguousarray(np.concatenate([v1, v2])))


def ensemble(n_systems: int, seed: int, n_min: int = 3, n_max: int = 2048, m_lo: float = 1e24,
             m_hi: float = 1e30, density: float = 1500.0, r_ball: float = 10 * AU, sigma_v: float = 5e3):
    """Independent few-body systems.  Returns (offsets[n_systems+1], m, r, x[.,3], v[.,3]) with the
    bodies of system s in [offsets[s], offsets[s+1]).  N_s ~ U{n_min..n_max}; masses log-uniform;
    radii (3m / (4 pi rho))^{1/3}; positions uniform in a ball; velocities Gaussian per axis."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_min, n_max + 1, n_systems)
    off = np.zeros(n_systems + 1, dtype=np.int64)
    off[1:] = np.cumsum(ns)
    tot = int(off[-1])
    m = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), tot))
    r = np.cbrt(3.0 * m / (4.0 * np.pi * density))
    u = rng.uniform(0.0, 1.0, tot) ** (1.0 / 3.0)
    x = _isotropic(rng, tot) * (u * r_ball)[:, None]
    v = rng.normal(0.0, sigma_v, (tot, 3))
    return off, m, r, np.ascontiguousarray(x), np.ascontiguousarray(v)


def comet_stage(n: int, bounding_rad: float, b_rad: float, b_mass: float, n_exp: float, d_scale: float = 0.0,
                min_cor: float = 0.5, max_cor: float = 1.0, dist_tol: float = 0.0, seed: int = 0) -> dict:
    """The evolve stage of random_comet (gregsys.hpp:1881-1984): n bodies of radius b_rad and mass
    b_mass at rest, uniform in a ball of radius bounding_rad (r = R cbrt(u), isotropic direction)
    with any body closer than 2 b_rad to an earlier one redrawn (gregsys.hpp:1798-1836; numpy's
    generator instead of mt19937_64), their mean position ``com``, and the callbacks' constants:
    max_dist = cbrt(n v_b / (pi/6) * 3 / (4 pi)) with v_b the body volume; scale_factor =
    d_scale^n_exp (d_scale <= 0: max_dist); max_dist *= 1 + dist_tol; min_max_cor = max_cor -
    (max_cor - min_cor) max_dist^n_exp / (max_dist^n_exp + scale_factor); every body's rest =
    max_cor - (max_cor - min_cor) d^n_exp / (d^n_exp + scale_factor), d its distance to com."""
    rng = np.random.default_rng(seed)
    x = np.empty((n, 3))
    k = 0
    while k < n:
        r = bounding_rad * np.cbrt(rng.uniform(0.0, 1.0))
        phi = rng.uniform(0.0, 2.0 * np.pi)
        cth = 1.0 - 2.0 * rng.uniform(0.0, 1.0)
        sth = np.sqrt(max(0.0, 1.0 - cth * cth))
        p = np.array([r * sth * np.cos(phi), r * sth * np.sin(phi), r * cth])
        if k and (np.sqrt(((x[:k] - p) ** 2).sum(axis=1)) < 2.0 * b_rad).any():
            continue
        x[k] = p
        k += 1
    com = x.mean(axis=0)
    small_vol = 4.0 / 3.0 * np.pi * b_rad ** 3
    max_dist = np.cbrt(small_vol * n / (np.pi / 6.0) * 3.0 / (4.0 * np.pi))
    if d_scale <= 0:
        d_scale = max_dist
    scale_factor = d_scale ** n_exp
    max_dist *= 1.0 + dist_tol
    mde = max_dist ** n_exp
    min_max_cor = max_cor - (max_cor - min_cor) * (mde / (mde + scale_factor))
    de = np.sqrt(((x - com) ** 2).sum(axis=1)) ** n_exp
    rest = max_cor - (max_cor - min_cor) * (de / (de + scale_factor))
    return {"m": np.full(n, float(b_mass)), "x": x, "v": np.zeros((n, 3)), "r": np.full(n, float(b_rad)),
            "rest": rest, "com": com, "scale_factor": float(scale_factor), "min_max_cor": float(min_max_cor),
            "n_exp": float(n_exp), "min_cor": float(min_cor), "max_cor": float(max_cor)}

