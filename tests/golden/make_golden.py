"""Generates the golden fixtures in tests/golden/ by running the UNMODIFIED reference headers
(through oracle/_ref/libgtdref.so, built from the reference tree by oracle/Makefile).

Run here, where the reference tree is mounted:  python tests/golden/make_golden.py
(``python tests/golden/make_golden.py tree`` regenerates only the tree-walk fixture.)
The fixtures are small .npz / text files; the tests read them, never the reference tree.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gregpackagescpp_b200.ics import AU, UNITS_G6674, plummer  # noqa: E402
from oracle.oracle import RefOracle, ensure_built  # noqa: E402

METHODS = {"euler": 2, "modified_euler": 4, "midpoint": 8, "leapfrog_kdk": 16, "leapfrog_dkd": 32}


def _mut(fn):
    def wrap(b):
        b = bytearray(b)
        fn(b)
        return bytes(b)
    return wrap


def _set_f64(off, val):
    return _mut(lambda b: b.__setitem__(slice(off, off + 8), np.float64(val).tobytes()))


def _set_x87(off, val):
    return _mut(lambda b: b.__setitem__(slice(off, off + 16), np.array([val], dtype=np.longdouble).tobytes()))


def record_fixtures(r, out):
    """memFreq recordings of the reference (fileFreq = 0, the only setting with which its evolve
    compiles): every direct method, memFreq 1, 2 and 3, collisions off (Plummer sphere) and on (the
    colliding "coll" cluster), one evolve call or two (the second clears the first's recordings);
    7 steps of one hour."""
    for meth_name, meth in METHODS.items():
        for f in (1, 2, 3):
            for coll in (0, 3):
                for calls in (1, 2):
                    if coll:
                        args = dict(r=out["coll_r"], rest=out["coll_rest"], coll=3)
                        m, x, v = out["coll_m"], out["coll_x"], out["coll_v"]
                    else:
                        args = {}
                        m, x, v = out["direct_m"], out["direct_x"], out["direct_v"]
                    d = r.evolve_record(meth, m, x, v, 3600.0, 7, f, calls, units=UNITS_G6674, **args)
                    key = f"rec_{meth_name}_{f}_{coll}_{calls}"
                    for k in ("pos", "vel", "ke", "pe", "energy", "tot", "x", "v"):
                        out[f"{key}_{k}"] = d[k]


def nsys_fixtures(r, out):
    """.nsys files written by the reference's to_nsys (after 3 KDK steps) for four M/R/T choices,
    the state its loader reads back, and corrupted copies with the reference loader's verdicts
    (read with alloc_chunks = false: with true the reference crashes on a NaN/Inf chunk)."""
    import tempfile
    m, x, v = plummer(37, 3)
    rad = np.linspace(1e3, 5e3, 37)
    rest = np.linspace(0.2, 1.0, 37)
    out["nsys_m"], out["nsys_x"], out["nsys_v"], out["nsys_r"], out["nsys_rest"] = m, x, v, rad, rest
    cases = {
        "sig_both": _mut(lambda b: b.__setitem__(slice(0, 2), b"XY")),
        "sig_first_only": _mut(lambda b: b.__setitem__(0, ord("X"))),
        "dtypes_bit6": _mut(lambda b: b.__setitem__(2, b[2] | 0x40)),
        "m_integral": _mut(lambda b: b.__setitem__(2, b[2] & ~0x02)),
        "t_size": _mut(lambda b: b.__setitem__(38, 4)),
        "rest_size_12": _mut(lambda b: b.__setitem__(39, 12)),
        "rest_size_32": _mut(lambda b: b.__setitem__(39, 32)),
        "rest_size_8": _mut(lambda b: b.__setitem__(39, 8)),
        "truncated": lambda b: b[:-4],
        "short": lambda b: b[:50],
        "time_size_12": _mut(lambda b: b.__setitem__(3, 12)),
        "time_integral": _mut(lambda b: (b.__setitem__(2, b[2] & ~0x01), b.__setitem__(3, 8),
                                         b.__setitem__(slice(4, 12), np.uint64(7200).tobytes()),
                                         b.__setitem__(slice(20, 28), np.uint64(600).tobytes()))),
        "dt_zero": _set_x87(20, 0.0),
        "dt_inf": _set_x87(20, np.inf),
        "nan_zpos_5": _set_f64(96 + 5 * 80 + 48, np.nan),
        "inf_mass_9": _set_f64(96 + 9 * 80 + 16, -np.inf),
        "nan_rcoeff_2": _set_x87(96 + 2 * 80, np.nan),
        "zero_bodies": lambda b: b[:88] + np.uint64(0).tobytes(),
    }
    with tempfile.TemporaryDirectory() as d:
        for kind in ("ddd", "fff", "lll", "ffd"):
            p = os.path.join(d, kind + ".nsys")
            r.to_nsys(kind, m, rad, rest, x, v, 3600.0, 3, p, UNITS_G6674)
            with open(p, "rb") as f:
                out[f"nsys_{kind}_bytes"] = np.frombuffer(f.read(), dtype=np.uint8).copy()
            rc, msg, st = r.load_nsys(kind, p)
            assert rc == 0, msg
            for k in ("m", "r", "rest", "x", "v"):
                out[f"nsys_{kind}_{k}"] = st[k]
            out[f"nsys_{kind}_meta"] = np.array([st["time"], st["dt"], st["G"]])
        base = bytes(out["nsys_ddd_bytes"])
        names, rcs, msgs = [], [], []
        for name, fn in cases.items():
            p = os.path.join(d, name + ".nsys")
            data = fn(base)
            with open(p, "wb") as f:
                f.write(data)
            rc, msg, st = r.load_nsys("ddd", p)
            out[f"nsysbad_{name}_bytes"] = np.frombuffer(data, dtype=np.uint8).copy()
            if rc == 0:
                out[f"nsysbad_{name}_meta"] = np.array([st["time"], st["dt"], st["G"], len(st["m"])])
                for k in ("m", "r", "rest", "x", "v"):
                    out[f"nsysbad_{name}_{k}"] = st[k]
            names.append(name)
            rcs.append(rc)
            msgs.append(msg)
        out["nsysbad_names"] = np.array(names)
        out["nsysbad_rc"] = np.array(rcs)
        out["nsysbad_msg"] = np.array(msgs)


def overlap_cluster(n: int, seed: int):
    """n bodies uniform in a 0.05 AU cube with radii of the order of their spacing (many overlaps),
    log-uniform masses 1e24..1e28 kg, Gaussian velocities of 3 km/s and restitution in [0.3, 1]."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, (n, 3)) * 0.05 * AU
    v = rng.normal(0.0, 3e3, (n, 3))
    m = np.exp(rng.uniform(np.log(1e24), np.log(1e28), n))
    r = 0.02 * AU * n ** (-1.0 / 3.0) * rng.uniform(0.5, 3.0, n)
    rest = rng.uniform(0.3, 1.0, n)
    return m, r, rest, x, v


def comet_ball(n: int, R: float, b: float, seed: int):
    """n non-overlapping bodies of radius b uniform in a ball of radius R, at rest (the placement of
    random_comet, gregsys.hpp:1798-1850, with numpy's generator instead of mt19937_64)."""
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < n:
        u = rng.uniform(-1.0, 1.0, 3)
        if u @ u > 1.0:
            continue
        p = u * R
        if all(np.linalg.norm(p - q) >= 2 * b for q in pts):
            pts.append(p)
    return np.array(pts)


CB_UNITS = "M1:1,D1:1,T1:1"


def comet_setup(n=64, R=8.0, b=1.0, mass=1.5e9, seed=3, weighted=False):
    """random_comet's evolve stage (gregsys.hpp:1909-1984) with n_exp = 2 and d_scale = max_dist:
    rest from the distance to the centre, min_cor 0.5, max_cor 1; continue while some body is
    beyond max_dist, then 20 probing steps."""
    x = comet_ball(n, R, b, seed)
    m = np.full(n, mass) if not weighted else mass * np.exp(np.random.default_rng(seed + 1).uniform(-0.2, 0.2, n))
    com = (m @ x) / m.sum() if weighted else x.mean(axis=0)
    md = b * np.cbrt(n / (np.pi / 6))  # max_dist of random_comet for SCP packing
    sf = md ** 2
    mmc = 1.0 - 0.5 * (md ** 2 / (md ** 2 + sf))
    d2 = np.sum((x - com) ** 2, axis=1)
    rest0 = 1.0 - 0.5 * (d2 / (d2 + sf))
    return dict(m=m, x=x, v=np.zeros_like(x), r=np.full(n, b), rest=rest0, com=com, sf=sf, mmc=mmc)


def callback_fixtures(r, out):
    """evolve(method, continue_ev_if, for_each_bod, for_all_bods) of the reference with
    random_comet's callbacks (ref_access::evolve_callbacks in oracle/ref_oracle.cpp)."""
    # (1) the comet stage itself: leapfrog KDK with overlap collisions until the predicate ends it
    for tag, weighted in (("cbk", False), ("cbw", True)):
        c = comet_setup(weighted=weighted)
        xo, vo, ro, steps, com = r.evolve_callbacks(
            16, c["m"], c["x"], c["v"], 0.25, 1000, CB_UNITS, r=c["r"], rest=c["rest"], coll=3,
            cont=(c["mmc"], 20), rest_from_com=(0.5, 1.0, c["sf"], 2.0, c["com"], weighted), max_steps=3000)
        for k in ("m", "x", "v", "r", "rest", "com"):
            out[f"{tag}_{k}"] = c[k]
        out[f"{tag}_par"] = np.array([c["mmc"], c["sf"]])
        out[f"{tag}_xo"], out[f"{tag}_vo"], out[f"{tag}_ro"] = xo, vo, ro
        out[f"{tag}_steps"], out[f"{tag}_como"] = np.array(steps), com
    # the m-weighted run is chaotic well before it ends (a 1e-16 nudge of the initial positions
    # moves its final state by 0.1 and its end anywhere from step 244 to 368): its state is also
    # kept at step 131, where that nudge moves it by 3e-10 (positions) and 3e-9 (velocities);
    # 131 = two 64-step chunks and an odd remainder
    c = comet_setup(weighted=True)
    xo, vo, ro, steps, com = r.evolve_callbacks(
        16, c["m"], c["x"], c["v"], 0.25, 1000, CB_UNITS, r=c["r"], rest=c["rest"], coll=3,
        cont=(c["mmc"], 20), rest_from_com=(0.5, 1.0, c["sf"], 2.0, c["com"], True), max_steps=131)
    out["cbw131_xo"], out["cbw131_vo"], out["cbw131_ro"] = xo, vo, ro
    out["cbw131_steps"], out["cbw131_como"] = np.array(steps), com
    # (2) every method, 8 fixed steps (no predicate), for_all_bods + collisions + for_each_bod:
    # the restitution of each step's collision pass comes from that step's for_all_bods
    c = comet_setup(n=48, R=5.0, b=1.0, mass=4e9, seed=5)
    for k in ("m", "x", "v", "r", "rest", "com"):
        out[f"cbs_{k}"] = c[k]
    out["cbs_par"] = np.array([c["mmc"], c["sf"]])
    for name, meth in METHODS.items():
        xo, vo, ro, steps, com = r.evolve_callbacks(
            meth, c["m"], c["x"], c["v"], 0.25, 8, CB_UNITS, r=c["r"], rest=c["rest"], coll=3,
            rest_from_com=(0.5, 1.0, c["sf"], 2.0, c["com"], False), each_factor=0.999)
        out[f"cbs_{name}_xo"], out[f"cbs_{name}_vo"], out[f"cbs_{name}_ro"] = xo, vo, ro
        out[f"cbs_{name}_como"] = com
    # (3) the predicate alone on a collisionless Plummer sphere (rest never changes): all bodies at
    # or above the bound -> exactly probing_iters steps (0, 63, 64, 70: around the 64-step graph
    # chunks); one body below -> the predicate never ends, max_steps 37 does
    m, x, v = plummer(40, 11)
    out["cbp_m"], out["cbp_x"], out["cbp_v"] = m, x, v
    rest_hi = np.full(40, 0.9)
    rest_lo = rest_hi.copy()
    rest_lo[17] = 0.1
    out["cbp_rest_hi"], out["cbp_rest_lo"] = rest_hi, rest_lo
    cases = []
    for meth_name in ("leapfrog_kdk", "leapfrog_dkd", "euler"):
        for probing, lo, cap in ((0, 0, 0), (63, 0, 0), (64, 0, 0), (70, 0, 0), (5, 1, 37)):
            xo, vo, ro, steps, _ = r.evolve_callbacks(
                METHODS[meth_name], m, x, v, 3600.0, 1000, UNITS_G6674, rest=rest_lo if lo else rest_hi,
                cont=(0.5, probing), max_steps=cap)
            key = f"cbp_{meth_name}_{probing}_{lo}_{cap}"
            out[f"{key}_xo"], out[f"{key}_vo"], out[f"{key}_steps"] = xo, vo, np.array(steps)
            cases.append(key)
    out["cbp_cases"] = np.array(cases)


def record_callback_fixtures(r, out):
    """memFreq recordings of evolve(method, callbacks) (FUNC_TEMPL_SELECT inside the callback loops,
    gregsys.hpp:16-106): (1) the 8 collisional steps of callback_fixtures (2) with for_all_bods and
    for_each_bod, memFreq 1 and 3, every method; (2) the predicate alone on the collisionless
    Plummer sphere, 7 probing steps, memFreq 2, the leapfrogs and Euler."""
    c = comet_setup(n=48, R=5.0, b=1.0, mass=4e9, seed=5)
    for name, meth in METHODS.items():
        for f in (1, 3):
            d = r.evolve_record_callbacks(meth, c["m"], c["x"], c["v"], 0.25, 8, CB_UNITS, f, r=c["r"], rest=c["rest"],
                                          coll=3, rest_from_com=(0.5, 1.0, c["sf"], 2.0, c["com"], False),
                                          each_factor=0.999)
            key = f"rcb_{name}_{f}"
            for k in ("pos", "vel", "ke", "pe", "energy", "tot", "x", "v", "rest", "com"):
                out[f"{key}_{k}"] = d[k]
    m, x, v = plummer(40, 11)
    for name in ("leapfrog_kdk", "leapfrog_dkd", "euler"):
        d = r.evolve_record_callbacks(METHODS[name], m, x, v, 3600.0, 1000, UNITS_G6674, 2, rest=np.full(40, 0.9),
                                      cont=(0.5, 7), max_frames=64)
        key = f"rcp_{name}"
        for k in ("pos", "vel", "ke", "pe", "energy", "tot", "x", "v"):
            out[f"{key}_{k}"] = d[k]
        out[f"{key}_steps"] = np.array(d["steps"])


TREE_WALK_N = 2000


def tree_walk_fixture():
    """tests/cpp/tree_walk_main.cpp - a program written against the reference's bh_tree API -
    compiled against the reference headers and run on TREE_WALK_N bodies; its output (leaf order,
    per-leaf cell_iterator counts and long-double force sums, nn_iterator counts, the children of
    the first yielded cells via operator[]) is the fixture tree_walk_ref.txt."""
    import subprocess
    import tempfile
    from oracle.oracle import reference_tree
    tree = reference_tree()
    if tree is None:
        raise SystemExit("the reference tree is not present here")
    src = os.path.join(ROOT, "tests", "cpp", "tree_walk_main.cpp")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "tree_walk_ref")
        subprocess.run(["g++", "-std=c++20", "-O2", "-include", "cstdint", "-w", "-I", tree, src, "-o", exe],
                       check=True)
        outp = subprocess.run([exe, str(TREE_WALK_N)], check=True, capture_output=True, text=True).stdout
    path = os.path.join(HERE, "tree_walk_ref.txt")
    with open(path, "w") as f:
        f.write(outp)
    print(path, os.path.getsize(path), "bytes")


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "tree":
        tree_walk_fixture()
        return
    ensure_built(ref=True)
    r = RefOracle()
    out = {}
    # direct summation, every method, 10 steps of one hour (the configuration of the 1e-12 bar)
    m, x, v = plummer(64, 1)
    out["direct_m"], out["direct_x"], out["direct_v"] = m, x, v
    for name, meth in METHODS.items():
        xo, vo, ao, _ = r.evolve(meth, m, x, v, 3600.0, 10, UNITS_G6674)
        out[f"direct_{name}_x"], out[f"direct_{name}_v"], out[f"direct_{name}_a"] = xo, vo, ao
    # odd N, other seed, KDK only
    m2, x2, v2 = plummer(37, 2)
    out["odd_m"], out["odd_x"], out["odd_v"] = m2, x2, v2
    xo, vo, ao, _ = r.evolve(16, m2, x2, v2, 3600.0, 10, UNITS_G6674)
    out["odd_kdk_x"], out["odd_kdk_v"], out["odd_kdk_a"] = xo, vo, ao
    # overlap collisions with restitution (collisions = 3)
    m3, x3, v3 = plummer(128, 3)
    rad = np.full(128, 0.08 * AU)
    rest = np.random.default_rng(0).uniform(0.2, 1.0, 128)
    out["coll_m"], out["coll_x"], out["coll_v"], out["coll_r"], out["coll_rest"] = m3, x3, v3, rad, rest
    for name, meth in METHODS.items():
        xo, vo, ao, _ = r.evolve(meth, m3, x3, v3, 3600.0, 5, UNITS_G6674, r=rad, rest=rest, coll=3)
        out[f"coll_{name}_x"], out[f"coll_{name}_v"] = xo, vo
    # energy
    ke, pe = r.energy(m, x, v, UNITS_G6674)
    out["energy_ke"], out["energy_pe"] = np.array(ke), np.array(pe)
    out["G_6674"] = np.array(r.G(UNITS_G6674))
    out["G_SI"] = np.array(r.G("M1:1,D1:1,T1:1"))
    out["G_odd"] = np.array(r.G("M3:7,D2:5,T11:13"))
    # body::operator+= merges
    rng = np.random.default_rng(5)
    pairs_a, pairs_b, merged = [], [], []
    for _ in range(16):
        a = np.concatenate([[rng.uniform(1e24, 1e30), rng.uniform(1e5, 1e7), rng.uniform(0, 1)],
                            rng.normal(0, AU, 3), rng.normal(0, 3e4, 3), rng.normal(0, 1e-3, 3)])
        b = np.concatenate([[rng.uniform(1e24, 1e30), rng.uniform(1e5, 1e7), rng.uniform(0, 1)],
                            rng.normal(0, AU, 3), rng.normal(0, 3e4, 3), rng.normal(0, 1e-3, 3)])
        pairs_a.append(a)
        pairs_b.append(b)
        merged.append(r.merge_pair(a, b))
    out["merge_a"], out["merge_b"], out["merge_out"] = np.array(pairs_a), np.array(pairs_b), np.array(merged)
    # check_overlap with merging: the case the reference's scan handles (overlap of the last two bodies)
    m4, x4, v4 = plummer(12, 4)
    x4[-1] = x4[-2] + np.array([0.3, 0.2, 0.1]) * 1e9
    rad4 = np.full(12, 1e9)
    rest4 = np.linspace(0.3, 0.9, 12)
    mo, ro, xo, vo = r.check_overlap_merge(m4, rad4, rest4, x4, v4)
    out["ovl_m"], out["ovl_x"], out["ovl_v"], out["ovl_r"], out["ovl_rest"] = m4, x4, v4, rad4, rest4
    out["ovl_out_m"], out["ovl_out_r"], out["ovl_out_x"], out["ovl_out_v"] = mo, ro, xo, vo
    # Barnes-Hut: reference octree (T=double and T=float) and the corrected walk
    m5, x5, v5 = plummer(2000, 7)
    out["bh_m"], out["bh_x"], out["bh_v"] = m5, x5, v5
    for isf in (0, 1):
        d = r.bh_tree_dump(x5, m5, isf)
        out[f"bh_tree{isf}_depth"] = d["depth"].astype(np.int8)
        out[f"bh_tree{isf}_body"] = d["body"].astype(np.int32)
        out[f"bh_tree{isf}_box"] = d["box"]
        # cell width as the opening test forms it, top.x - btm.x in T (greg8tree.hpp:753-755)
        if isf:
            out[f"bh_tree{isf}_width"] = (d["top"][:, 0].astype(np.float32) -
                                          d["btm"][:, 0].astype(np.float32)).astype(np.float64)
        else:
            out[f"bh_tree{isf}_width"] = d["top"][:, 0] - d["btm"][:, 0]
        if isf == 0:
            out["bh_tree0_com"] = d["com"]
            out["bh_tree0_mass"] = d["mass"]
    a, cnt = r.bh_acc(x5, m5, 0.5, 0.0, UNITS_G6674)
    out["bh_acc"], out["bh_count"] = a, np.array(cnt)
    m6, x6, v6 = plummer(300, 8)
    out["bhk_m"], out["bhk_x"], out["bhk_v"] = m6, x6, v6
    xo, vo, ao, _, _ = r.bh_kdk(m6, x6, v6, 3600.0, 5, 0.5, 0.0, UNITS_G6674)
    out["bhk_xo"], out["bhk_vo"], out["bhk_ao"] = xo, vo, ao
    # bh_s_coll: a tight cluster of overlapping bodies; one collision pass on a T=double tree, then
    # a Barnes-Hut KDK with the pass after every full kick (collisions != 0)
    mc, rc, ec, xc, vc = overlap_cluster(400, 9)
    out["bhc_m"], out["bhc_r"], out["bhc_rest"], out["bhc_x"], out["bhc_v"] = mc, rc, ec, xc, vc
    out["bhc_v_out"] = r.bh_s_coll(mc, rc, ec, xc, vc)
    mk, rk, ek, xk, vk = overlap_cluster(300, 10)
    out["bhck_m"], out["bhck_r"], out["bhck_rest"], out["bhck_x"], out["bhck_v"] = mk, rk, ek, xk, vk
    out["bhck_xo"], out["bhck_vo"] = r.bh_kdk_coll(mk, rk, ek, xk, vk, 3600.0, 5, 0.5, UNITS_G6674)
    nsys_fixtures(r, out)
    record_fixtures(r, out)
    callback_fixtures(r, out)
    record_callback_fixtures(r, out)
    path = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(out), "arrays")
    tree_walk_fixture()


if __name__ == "__main__":
    main()
