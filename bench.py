#!/usr/bin/env python
"""Benchmark of the gtd:: force-and-step hot path on B200.

Workload (one GPU, the configuration the headline metric is quoted on): mixed-precision direct
summation, N = 262144 equal-mass Plummer sphere (a = 1 AU, M = 1e30 kg, G = 6.674e-11, seeded
synthetic data), leapfrog KDK with dt = 3600 s.  One "step" = one KDK step (kick-drift, one
force evaluation of N(N-1) ordered pair-interactions, kick).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: the hot path runs on one GPU; N > 1 runs N independent replicas (one process
per GPU, no data-path collective; "scaling": "weak").  The reference arm times the reference's
own single-threaded CPU evolve (oracle/_ref, built from the reference headers; the C port under
oracle/ where that library is absent) on all host cores, as independent copies.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import faulthandler

import numpy as np

faulthandler.enable()

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pair-interactions/s mixed vs FP64 GPU at |ΔE/E|≤1e-6; ensemble steps/s"
UNIT = "pair-interactions/s"
FLOPS_PER_INTERACTION = 20
# dram__bytes_read.sum + dram__bytes_write.sum of one force_mixed_kernel launch, from an ncu capture
# (--metrics dram__bytes_read.sum,dram__bytes_write.sum, one launch at N = 262144): (N, variant) ->
# (read, write).  The positions (N x 32 B = 8.39 MB) are read about once; the writes are the work
# units' FP64 partial sums (units x 3 x 8 B per i-body), of which part stays in L2.
NCU_FORCE_TRAFFIC = {(262144, 2): (12255232, 178242304), (262144, 8): (9481216, 176747264)}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=262144)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--fp64-steps", type=int, default=3)
    p.add_argument("--e2e-calls", type=int, default=2)
    p.add_argument("--e2e-iterations", type=int, default=5)
    p.add_argument("--cpu-sample-n", type=int, default=8192)
    p.add_argument("--cpu-sample-steps", type=int, default=3)
    p.add_argument("--cpu-baseline-steps", type=int, default=40,
                   help="steps of the single-core reference sample beside the GPU line (~10 s at N=8192)")
    p.add_argument("--drift-steps", type=int, default=1000,
                   help="after the timed loop (untimed, one GPU): evolve the workload this many steps in both the "
                        "mixed and the FP64 path and report |dE/E| and momentum drift every --drift-every steps "
                        "(0: skip)")
    p.add_argument("--drift-every", type=int, default=100)
    p.add_argument("--drift-only", action="store_true", help="print only the drift series")
    p.add_argument("--oracle-rows", type=int, default=512,
                   help="rows of the N-body force checked against the CPU oracle (untimed)")
    p.add_argument("--configs", choices=["all", "none"], default="all",
                   help="after the headline (untimed, one GPU): the other configurations of the path")
    p.add_argument("--force-prec", choices=["mixed", "f64"], default="mixed",
                   help="--workload force: precision of the force evaluations")
    p.add_argument("--force-calls", type=int, default=3, help="--workload force: evaluations (profiling driver)")
    p.add_argument("--workload", choices=["direct-mixed", "direct-fp64-1024", "bh", "ensemble", "adjoint", "comet",
                                          "force"],
                   default="direct-mixed", help="direct-mixed is the headline; the others print their own line")
    p.add_argument("--bh-n", type=int, default=4194304)
    p.add_argument("--bh-cpu-n", type=int, default=10000)
    p.add_argument("--bh-steps", type=int, default=200, help="evolve(leapfrog_kdk | barnes_hut) steps timed end to end")
    p.add_argument("--bh-walk-variant", type=int, default=-1,
                   help="node records of the float-tree walk: -1 default, 0 separate arrays, 1 interleaved")
    p.add_argument("--ens-systems", type=int, default=4096)
    p.add_argument("--ens-steps", type=int, default=128, help="ensemble steps timed (after the warm-up chunk)")
    p.add_argument("--ens-check-systems", type=int, default=12,
                   help="ensemble systems re-run on the oracle after the timed steps (untimed)")
    p.add_argument("--ens-config", type=str, default="",
                   help="THREADS,BODIES_PER_THREAD for the ensemble kernel instead of the autotuner's choice")
    p.add_argument("--adj-n", type=int, default=16384)
    p.add_argument("--adj-steps", type=int, default=2000)
    p.add_argument("--adj-every", type=int, default=45)
    p.add_argument("--adj-fd", type=int, default=0)
    p.add_argument("--comet-steps", type=int, default=20000)
    p.add_argument("--comet-host-steps", type=int, default=200)
    p.add_argument("--comet-ref-steps", type=int, default=300)
    p.add_argument("--comet-form", choices=["graph", "eager"], default="graph",
                   help="eager: the device-callback loop with one launch per kernel and a host read of the "
                        "verdict per step (the form ncu can profile kernel by kernel)")
    p.add_argument("--mixed-variant", type=int, default=-1,
                   help="use this mixed force-kernel variant instead of the autotuner's choice (with "
                        "--workload force: the variant of --force-prec)")
    return p.parse_args()


# ------------------------------------------------------------------------------------------------
# process group (replicas only; used for barriers and the max-over-ranks of the timed region)
# ------------------------------------------------------------------------------------------------
def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------------------------------------
# CPU baselines (the reference's own evolve, else the C port of it)
# ------------------------------------------------------------------------------------------------
def _cpu_copy(job):
    """One single-threaded evolve(leapfrog_kdk) of an n-body Plummer system in this (spawned)
    process; returns (interactions, evolve seconds, kind).  Construction is excluded: the
    reference gives every body a unique ID by scanning a process-wide set from 0
    (gregbod.hpp:111-117), so building n bodies costs O(n^2) before evolve starts."""
    n_sample, steps, seed = job
    from gregpackagescpp_b200.ics import UNITS_G6674, plummer
    from oracle.oracle import Oracle, RefOracle, ensure_built
    m, x, v = plummer(n_sample, seed)
    inter = float(steps + 1) * n_sample * (n_sample - 1)  # initial acceleration + one evaluation per step
    if RefOracle.available():
        return inter, RefOracle().bench_kdk(m, x, v, 3600.0, steps, 1, UNITS_G6674), "reference"
    ensure_built()
    o = Oracle()
    return inter, o.bench_kdk(m, x, v, 3600.0, steps, o.G(UNITS_G6674), 1), "port"


def cpu_sample(n_sample, steps, seed, copies):
    """Aggregate CPU throughput of `copies` concurrent single-threaded evolve() runs, one process
    each (the reference's evolve is single-threaded; concurrent independent systems are how its
    drivers use several cores, bdsim.cpp:82-113).  Returns (interactions/s, kind, max seconds)."""
    if copies == 1:
        inter, secs, kind = _cpu_copy((n_sample, steps, seed))
        return inter / secs, kind, secs
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(copies) as pool:
        res = pool.map(_cpu_copy, [(n_sample, steps, seed)] * copies)
    return sum(i / s for i, s, _ in res), res[0][2], max(s for _, s, _ in res)


def stage(msg: str) -> None:
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = host_threads()
    n_s, st = args.cpu_sample_n, args.cpu_sample_steps
    for _ in range(max(args.warmup, 0)):
        cpu_sample(n_s, st, args.seed, threads)
    vals, secs_tot, kind = [], 0.0, None
    for _ in range(args.steps):
        val, kind, secs = cpu_sample(n_s, st, args.seed, threads)
        vals.append(val)
        secs_tot += secs
    value = float(np.mean(vals))
    sample = (f"{threads} independent copies of evolve(leapfrog_kdk), N={n_s} Plummer (seed {args.seed}), "
              f"{st} step(s) = {st + 1} force evaluations each, per bench step; single-threaded evolve per copy")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs_tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (long double intermediates)",
        "data": "synthetic (seeded Plummer sphere)",
        "config": {"workload": "direct summation leapfrog KDK on a Plummer sphere (CPU sample of the N=262144 "
                               "mixed-precision workload)", "n_bodies_sample": n_s, "threads": threads},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------
def _dist_stats(rel):
    """Distribution of per-body relative errors."""
    rel = np.asarray(rel, dtype=np.float64)
    return {"rms": float(np.sqrt((rel ** 2).mean())), "median": float(np.median(rel)),
            "p99": float(np.quantile(rel, 0.99)), "p99_9": float(np.quantile(rel, 0.999)), "max": float(rel.max())}


def oracle_rows_check(m, x, accs, n_rows, seed, threads):
    """The checker beside the CPU baseline: accelerations on `n_rows` seeded rows from the oracle
    (the reference's cumulative_acc arithmetic, summed over all other bodies), against each GPU
    path's accelerations.  Per row: the error relative to |a_i| and relative to the row's force
    scale sum_j G m_j / r_ij^2 (what an FP32 sum of the row's terms rounds against)."""
    import ctypes as _C
    from oracle.oracle import Oracle
    o = Oracle()
    rows = np.sort(np.random.default_rng(seed).choice(len(m), n_rows, replace=False))
    t0 = time.perf_counter()
    want, gross = o.direct_acc_rows(m, x, _C.c_longdouble(6.674e-11), rows, threads=threads)
    secs = time.perf_counter() - t0
    amag = np.linalg.norm(want, axis=1)
    out = {"rows": int(n_rows), "row_seed": seed, "oracle_s": secs, "threads": threads,
           "force_scale_over_abs_a": {"median": float(np.median(gross / amag)), "max": float((gross / amag).max())}}
    for name, a in accs.items():
        err = np.linalg.norm(a[rows] - want, axis=1)
        rel = err / amag
        d = _dist_stats(rel)
        d["max_over_force_scale"] = float((err / gross).max())
        worst = np.argsort(rel)[-3:][::-1]
        d["worst_rows"] = [{"row": int(rows[k]), "rel": float(rel[k]),
                            "force_scale_over_abs_a": float(gross[k] / amag[k])} for k in worst]
        out[name] = d
    return out


def measured_peaks(local):
    """HBM denominator: the driver's MEASURED_PEAKS.json (a measured copy on this pool) where present,
    else a device-to-device copy timed here.  The FMA peaks come from the library's microkernel."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]) * 1e9, "MEASURED_PEAKS.json hbm_gbs (measured copy on this pool)"
    except Exception:
        pass
    import torch
    nb = 2 << 30
    a = torch.empty(nb // 4, dtype=torch.float32, device=f"cuda:{local}")
    b = torch.empty_like(a)
    b.copy_(a)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        b.copy_(a)
    e1.record()
    e1.synchronize()
    return 5 * 2 * nb / (e0.elapsed_time(e1) * 1e-3), "device-to-device copy of 2 GiB timed in this run"


def run_ours(args, rank, world, local):
    import torch

    from gregpackagescpp_b200 import _lib
    from gregpackagescpp_b200.ics import plummer
    from gregpackagescpp_b200._lib import check

    torch.cuda.set_device(local)
    L = _lib.load()
    n, K, W = args.n, args.steps, args.warmup
    G, dt = 6.674e-11, 3600.0
    m, x, v = plummer(n, args.seed)
    x3, v3 = np.ascontiguousarray(x.reshape(-1)), np.ascontiguousarray(v.reshape(-1))
    pair = float(n) * (n - 1)

    def make(prec):
        h = C.c_void_p()
        check(L.gtd_system_create(C.byref(h), local, prec))
        check(L.gtd_system_set_params(h, G, dt, 1000, 0.0, 0.5))
        check(L.gtd_system_upload(h, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
        return h

    def stream_of(h):
        p = C.c_void_p()
        check(L.gtd_system_stream(h, C.byref(p)))
        return torch.cuda.ExternalStream(p.value, device=torch.device("cuda", local))

    def energy(h):
        ke, pe = C.c_double(), C.c_double()
        check(L.gtd_system_energy(h, C.byref(ke), C.byref(pe), None, None))
        return ke.value + pe.value

    def launches(h):
        c = C.c_uint64()
        check(L.gtd_system_launch_count(h, C.byref(c)))
        return c.value

    stage("autotune")
    h64, hmx = make(_lib.PREC_F64), make(_lib.PREC_MIXED)
    tuned = {}
    for name, h in (("mixed", hmx), ("fp64", h64)):
        best, best_ms = C.c_int(), C.c_double()
        if name == "mixed" and args.mixed_variant >= 0:
            check(L.gtd_system_set_direct_variant(h, args.mixed_variant))
            best.value, best_ms.value = args.mixed_variant, float("nan")
        else:
            check(L.gtd_system_autotune_direct(h, 3, C.byref(best), C.byref(best_ms)))
        ii, fold = C.c_int(), C.c_int()
        check(L.gtd_direct_variant_info(_lib.PREC_MIXED if name == "mixed" else _lib.PREC_F64, best.value,
                                        C.byref(ii), C.byref(fold)))
        tuned[name] = {"variant": best.value, "i_per_thread": ii.value, "fold": fold.value,
                       "force_ms": best_ms.value}

    units, part_bytes = C.c_int64(), C.c_int64()
    check(L.gtd_system_direct_plan_info(hmx, C.byref(units), C.byref(part_bytes)))

    stage("accuracy")
    # --- accelerations of both paths at the initial state (untimed); checked against the oracle
    # beside the CPU baseline below, and against each other here
    a64, amx = np.zeros(3 * n), np.zeros(3 * n)
    check(L.gtd_system_accelerations(h64, 0, a64.ctypes.data))
    check(L.gtd_system_accelerations(hmx, 0, amx.ctypes.data))
    a64, amx = a64.reshape(n, 3), amx.reshape(n, 3)
    rel = np.linalg.norm(amx - a64, axis=1) / np.linalg.norm(a64, axis=1)

    stage("fp64 throughput")
    # --- FP64 GPU path throughput (same workload, fewer steps)
    check(L.gtd_system_evolve_begin(h64, 16))
    check(L.gtd_system_evolve_steps(h64, 1))
    s64 = stream_of(h64)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s64)
    check(L.gtd_system_evolve_steps(h64, args.fp64_steps))
    e1.record(s64)
    e1.synchronize()
    fp64_value = args.fp64_steps * pair / (e0.elapsed_time(e1) * 1e-3)
    check(L.gtd_system_destroy(h64))

    stage("mixed timed loop")
    # --- mixed path: the timed hot loop
    E0 = energy(hmx)
    check(L.gtd_system_evolve_begin(hmx, 16))
    for _ in range(W):
        check(L.gtd_system_evolve_steps(hmx, 1))
    smx = stream_of(hmx)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")  # > 126 MB L2
    check(L.gtd_system_time_force_kernels(hmx, 1))
    check(L.gtd_system_force_timing(hmx, None, None, 1))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    clocks = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    clocks.start()
    time.sleep(0.4)
    barrier(world)
    torch.cuda.synchronize()
    l0 = launches(hmx)
    for k in range(K):
        with torch.cuda.stream(smx):
            flush.zero_()  # L2 flush between timed steps, outside the timed events
        ev[k][0].record(smx)
        check(L.gtd_system_evolve_steps(hmx, 1))
        ev[k][1].record(smx)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    gpu_launches = launches(hmx) - l0
    t_local = sum(a.elapsed_time(b) for a, b in ev) * 1e-3
    force_ms, force_n = C.c_double(), C.c_uint64()
    check(L.gtd_system_force_timing(hmx, C.byref(force_ms), C.byref(force_n), 1))
    check(L.gtd_system_time_force_kernels(hmx, 0))
    t_max = max_over_ranks(t_local, world)
    total_inter = sum_over_ranks(K * pair, world)
    value = total_inter / t_max
    E1 = energy(hmx)
    drift = abs(E1 - E0) / abs(E0)
    check(L.gtd_system_destroy(hmx))
    del flush

    stage("peaks")
    # --- roofline: the force kernel (FP32 pipe); denominator measured on this GPU
    peak = C.c_double()
    check(L.gtd_measure_fma_peak(local, _lib.PREC_MIXED, C.byref(peak)))
    peak64 = C.c_double()
    check(L.gtd_measure_fma_peak(local, _lib.PREC_F64, C.byref(peak64)))
    avg_force_s = force_ms.value * 1e-3 / max(force_n.value, 1)
    achieved = FLOPS_PER_INTERACTION * pair / avg_force_s
    hbm_peak, hbm_src = measured_peaks(local)

    stage("e2e")
    # --- end to end through the public C ABI with host buffers (upload, evolve, download)
    iters = args.e2e_iterations
    he = C.c_void_p()
    check(L.gtd_system_create(C.byref(he), local, _lib.PREC_MIXED))
    check(L.gtd_system_set_params(he, G, dt, iters, 0.0, 0.5))
    xo, vo, ao = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
    ns = C.c_int64()
    check(L.gtd_system_upload(he, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
    check(L.gtd_system_evolve(he, 16, C.byref(ns)))  # warm-up call
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.e2e_calls):
        check(L.gtd_system_upload(he, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
        check(L.gtd_system_evolve(he, 16, C.byref(ns)))
        check(L.gtd_system_download(he, None, None, None, None, xo.ctypes.data, vo.ctypes.data, ao.ctypes.data))
    t_e2e = max_over_ranks(time.perf_counter() - t0, world)
    check(L.gtd_system_destroy(he))
    e2e_steps = args.e2e_calls * iters
    e2e_value = sum_over_ranks(args.e2e_calls * (iters + 1) * pair, world) / t_e2e
    h2d = (m.nbytes + x3.nbytes + v3.nbytes) * args.e2e_calls / e2e_steps
    d2h = (xo.nbytes + vo.nbytes + ao.nbytes) * args.e2e_calls / e2e_steps

    cpu, oracle_check = None, None
    if rank == 0 and world == 1 and args.cpu_sample_n > 0:
        stage("cpu baseline sample + oracle rows")
        cval, kind, secs = cpu_sample(args.cpu_sample_n, args.cpu_baseline_steps, args.seed, 1)
        cpu = {"value": cval, "unit": UNIT, "cores": 1, "kind": kind,
               "sample": f"the reference evolve(leapfrog_kdk) (single-threaded by design) on an N="
                         f"{args.cpu_sample_n} Plummer sphere, {args.cpu_baseline_steps} step(s) "
                         f"({args.cpu_baseline_steps + 1} force evaluations), {secs:.1f} s of evolve time"}
        if args.oracle_rows > 0:
            oracle_check = oracle_rows_check(m, x, {"fp64": a64, "mixed": amx}, args.oracle_rows, 5, host_threads())

    drift_out, cfgs = None, None
    if rank == 0 and world == 1 and args.drift_steps > 0:
        stage(f"drift series ({args.drift_steps} steps, mixed and fp64)")
        drift_out = drift_series(args, local, autotune=False)
    if rank == 0 and world == 1 and args.configs == "all":
        cfgs = {}
        for name, fn in (("direct_fp64_1024", cfg_fp64_small), ("barnes_hut", cfg_bh), ("ensemble", cfg_ensemble),
                         ("adjoint", cfg_adjoint)):
            stage(f"config {name}")
            try:
                cfgs[name] = fn(args, local, peak.value, peak64.value, hbm_peak)
            except Exception as exc:  # a failing secondary configuration must not hide the headline
                cfgs[name] = {"error": f"{type(exc).__name__}: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": 1e3 * t_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 pair forces + fp64 Kahan sums/state", "data": "synthetic (seeded Plummer sphere)",
            "config": {"workload": "mixed-precision direct summation, leapfrog KDK, equal-mass Plummer sphere "
                                   "a=1 AU M=1e30 kg, dt=3600 s", "n_bodies": n, "G": G,
                       "parallelism": f"replicas{world}" if world > 1 else "1 GPU",
                       "l2": "flushed (512 MB write) between timed steps, outside the timed events"},
            "fp64_gpu": {"value": fp64_value, "unit": UNIT, "steps": args.fp64_steps,
                         "mixed_over_fp64": value / world / fp64_value,
                         "frac_of_fp64_peak": FLOPS_PER_INTERACTION * fp64_value / peak64.value},
            "accuracy": {"mixed_vs_fp64_all_bodies": _dist_stats(rel),
                         "energy_drift_rel": drift, "energy_drift_steps": W + K},
            "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak.value / 1e12,
                         "unit": "TFLOP/s", "frac": achieved / peak.value,
                         "traffic": (sum(NCU_FORCE_TRAFFIC[(n, tuned["mixed"]["variant"])])
                                     if (n, tuned["mixed"]["variant"]) in NCU_FORCE_TRAFFIC else None),
                         "traffic_read_write": NCU_FORCE_TRAFFIC.get((n, tuned["mixed"]["variant"])),
                         "traffic_unit": "bytes per launch (ncu dram read + write)",
                         "algorithmic_bytes": 32 * n + part_bytes.value,
                         "algorithmic_bytes_note": "positions 32 B per body read once + the work units' FP64 "
                                                   f"partial sums ({units.value} units)",
                         "kernel": "force_mixed_kernel", "flops_per_interaction": FLOPS_PER_INTERACTION,
                         "peak_source": "measured FFMA/FFMA2 microkernel on this GPU (gtd_measure_fma_peak)",
                         "fp64_peak": peak64.value / 1e12, "hbm_peak_GBs": hbm_peak / 1e9,
                         "hbm_peak_source": hbm_src},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "calls": args.e2e_calls, "iterations_per_call": iters},
            "gpu_launches": gpu_launches,
            "autotuned": tuned,
            "clocks": clk,
        }
        if oracle_check is not None:
            line["accuracy"]["vs_oracle_rows"] = oracle_check
        if drift_out is not None:
            line["drift"] = drift_out
        if cfgs is not None:
            line["configs"] = cfgs
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)


def drift_series(args, local, autotune=True):
    """Energy and momentum conservation of the workload over a long run, mixed next to FP64:
    |dE/E| and |P|/(sum m|v|) every --drift-every steps (untimed; wall seconds reported)."""
    from gregpackagescpp_b200 import _lib
    from gregpackagescpp_b200._lib import check
    from gregpackagescpp_b200.ics import plummer

    L = _lib.load()
    n = args.n
    m, x, v = plummer(n, args.seed)
    x3, v3 = np.ascontiguousarray(x.reshape(-1)), np.ascontiguousarray(v.reshape(-1))
    out = {"workload": f"N={n} Plummer, leapfrog KDK dt=3600 s", "steps": args.drift_steps,
           "every": args.drift_every, "columns": ["step", "dE_over_E", "abs_P_over_sum_m_abs_v"], "series": {}}
    for name, prec in (("mixed", _lib.PREC_MIXED), ("fp64", _lib.PREC_F64)):
        h = C.c_void_p()
        check(L.gtd_system_create(C.byref(h), local, prec))
        check(L.gtd_system_set_params(h, 6.674e-11, 3600.0, 1000, 0.0, 0.5))
        check(L.gtd_system_upload(h, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
        if autotune:
            best = C.c_int()
            check(L.gtd_system_autotune_direct(h, 2, C.byref(best), None))
        ke, pe, p = C.c_double(), C.c_double(), np.zeros(3)
        check(L.gtd_system_energy(h, C.byref(ke), C.byref(pe), p.ctypes.data, None))
        E0, pscale = ke.value + pe.value, float((m[:, None] * np.abs(v)).sum())
        rows = [(0, 0.0, float(np.linalg.norm(p)) / pscale)]
        check(L.gtd_system_evolve_begin(h, 16))
        t0 = time.perf_counter()
        done = 0
        while done < args.drift_steps:
            k = min(args.drift_every, args.drift_steps - done)
            check(L.gtd_system_evolve_steps(h, k))
            done += k
            check(L.gtd_system_energy(h, C.byref(ke), C.byref(pe), p.ctypes.data, None))
            rows.append((done, (ke.value + pe.value - E0) / abs(E0), float(np.linalg.norm(p)) / pscale))
        out["series"][name] = {"wall_s": time.perf_counter() - t0, "rows": rows}
        check(L.gtd_system_destroy(h))
    mx, fx = out["series"]["mixed"]["rows"], out["series"]["fp64"]["rows"]
    out["max_abs_dE_over_E"] = {"mixed": max(abs(r[1]) for r in mx), "fp64": max(abs(r[1]) for r in fx)}
    out["max_abs_mixed_minus_fp64_dE_over_E"] = max(abs(a[1] - b[1]) for a, b in zip(mx, fx))
    out["max_abs_P_over_sum_m_abs_v"] = {"mixed": max(r[2] for r in mx), "fp64": max(r[2] for r in fx)}
    return out


# ------------------------------------------------------------------------------------------------
# secondary workloads (--workload): the other configurations of the path, one JSON line each
# ------------------------------------------------------------------------------------------------
def _events(stream):
    import torch
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return a, b


def cfg_fp64_small(args, local, peak32=None, peak64=None, hbm=None):
    """Plain direct summation as the reference runs it: N=1024 Plummer, FP64, leapfrog KDK,
    dt=3600 s, 1000 steps; final state against the reference CPU run of the same call."""
    from gregpackagescpp_b200 import System
    from gregpackagescpp_b200.ics import UNITS_G6674, plummer
    n, steps = 1024, 1000
    m, x, v = plummer(n, args.seed)
    s = System(m, x, v, timestep=3600.0, num_iterations=steps, units_format=UNITS_G6674, device=local)
    s.evolve(16)  # warm-up (same call)
    s = System(m, x, v, timestep=3600.0, num_iterations=steps, units_format=UNITS_G6674, device=local)
    t0 = time.perf_counter()
    ns = s.evolve(16)
    wall = time.perf_counter() - t0
    inter = (steps + 1) * n * (n - 1)
    line = {"workload": "direct FP64, N=1024 Plummer, leapfrog KDK dt=3600 s, 1000 steps", "unit": UNIT,
            "device_value": inter / (ns * 1e-9), "e2e_value": inter / wall, "device_s": ns * 1e-9, "e2e_s": wall}
    if peak64:
        line["frac_of_fp64_peak"] = FLOPS_PER_INTERACTION * inter / (ns * 1e-9) / peak64
    try:
        from oracle.oracle import RefOracle
        if RefOracle.available():
            xo, vo, _, ref_ns = RefOracle().evolve(16, m, x, v, 3600.0, steps, UNITS_G6674)
            line["reference_cpu"] = {"value": inter / (ref_ns * 1e-9), "s": ref_ns * 1e-9, "cores": 1}
            line["final_state_rel_err"] = {"x": float(np.abs(s.x - xo).max() / np.abs(xo).max()),
                                           "v": float(np.abs(s.v - vo).max() / np.abs(vo).max())}
    except Exception as exc:  # the reference library is optional on a box
        line["reference_cpu"] = {"unavailable": str(exc)}
    return line


def cfg_bh(args, local, peak32=None, peak64=None, hbm=None):
    """Barnes-Hut: two Plummer spheres of 2^21 bodies each on a parabolic approach, FP32 tree
    (T=float geometry, FP64 moments), theta=0.5, leapfrog KDK dt=3600 s; per-phase device times."""
    from gregpackagescpp_b200 import _lib
    from gregpackagescpp_b200._lib import check
    from gregpackagescpp_b200.ics import two_plummer
    L = _lib.load()
    n_each = args.bh_n // 2
    m, x, v = two_plummer(n_each, args.seed)
    n = len(m)
    x3, v3 = np.ascontiguousarray(x.reshape(-1)), np.ascontiguousarray(v.reshape(-1))
    h = C.c_void_p()
    check(L.gtd_system_create(C.byref(h), local, _lib.PREC_F64))
    check(L.gtd_system_set_params(h, 6.674e-11, 3600.0, args.bh_steps, 0.0, 0.5))
    check(L.gtd_system_upload(h, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
    check(L.gtd_bh_set_tree_float(h, 1))
    check(L.gtd_bh_set_walk_variant(h, args.bh_walk_variant))
    # phase timing: build, walk
    import torch
    p = C.c_void_p()
    check(L.gtd_system_stream(h, C.byref(p)))
    st = torch.cuda.ExternalStream(p.value, device=torch.device("cuda", local))
    cnt = np.zeros(n, np.uint32)
    check(L.gtd_bh_build(h, 1))
    check(L.gtd_bh_accelerations(h, None, cnt.ctypes.data))  # warm-up
    tb, tw = [], []
    for _ in range(3):
        e0, e1 = _events(st)
        e0.record(st)
        check(L.gtd_bh_build(h, 1))
        e1.record(st)
        e1.synchronize()
        tb.append(e0.elapsed_time(e1))
        e0.record(st)
        check(L.gtd_bh_accelerations(h, None, None))
        e1.record(st)
        e1.synchronize()
        tw.append(e0.elapsed_time(e1))
    nn, nl = C.c_int64(), C.c_int64()
    check(L.gtd_bh_tree_size(h, C.byref(nn), C.byref(nl), None))
    inter = float(cnt.astype(np.float64).sum())
    # the reference schedule end to end: evolve(leapfrog_kdk | barnes_hut) for --bh-steps steps
    ns = C.c_int64()
    check(L.gtd_system_set_params(h, 6.674e-11, 3600.0, args.bh_steps, 0.0, 0.5))
    check(L.gtd_system_upload(h, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
    check(L.gtd_system_evolve(h, 16 | 65536, C.byref(ns)))
    check(L.gtd_system_destroy(h))
    build_ms, walk_ms = float(np.median(tb)), float(np.median(tw))
    # algorithmic HBM bytes of one build: codes 16 B/body in + 12 B out, 8 radix passes x 24 B/body,
    # node emission ~48 B/node, moments 32 B/node read + write
    build_bytes = n * (28 + 8 * 24) + nn.value * (48 + 64)
    line = {"workload": f"Barnes-Hut, two Plummer spheres N={n}, theta=0.5, FP32 tree, FP64 moments",
            "n_bodies": n, "n_nodes": nn.value, "n_leaves": nl.value, "interactions_per_walk": inter,
            "interactions_per_body": inter / n, "build_ms": build_ms, "walk_ms": walk_ms,
            "walk_interactions_per_s": inter / (walk_ms * 1e-3),
            "walk_flops_20_per_interaction_TFLOPs": 20 * inter / (walk_ms * 1e-3) / 1e12,
            "build_algorithmic_GBs": build_bytes / (build_ms * 1e-3) / 1e9,
            "walk_variant": args.bh_walk_variant, "evolve_steps": args.bh_steps, "evolve_s": ns.value * 1e-9,
            "steps_per_s": args.bh_steps / (ns.value * 1e-9)}
    if peak32:
        line["walk_frac_of_fp32_peak"] = 20 * inter / (walk_ms * 1e-3) / peak32
    if hbm:
        line["build_frac_of_hbm"] = build_bytes / (build_ms * 1e-3) / hbm
    try:
        from gregpackagescpp_b200.ics import two_plummer as tp
        from oracle.oracle import RefOracle
        if RefOracle.available() and args.bh_cpu_n > 0:
            ms_, xs_, vs_ = tp(args.bh_cpu_n // 2, args.seed)
            _, _, _, b_ns, w_ns = RefOracle().bh_kdk(ms_, xs_, vs_, 3600.0, 0, 0.5)
            _, rcnt = RefOracle().bh_acc(xs_, ms_, 0.5)
            line["reference_cpu"] = {"n_bodies": len(ms_), "build_s": b_ns * 1e-9, "walk_s": w_ns * 1e-9,
                                     "walk_interactions_per_s": rcnt / (w_ns * 1e-9), "cores": 1}
    except Exception as exc:
        line["reference_cpu"] = {"unavailable": str(exc)}
    return line


def cfg_ensemble(args, local, peak32=None, peak64=None, hbm=None):
    """4096 independent systems, N ~ U{3..2048}, log-uniform masses, radii from 1500 kg/m^3,
    positions in a 10 AU ball, sigma_v = 5 km/s; FP64 state, FP32 forces, merges; KDK dt=600 s."""
    from gregpackagescpp_b200.ensemble import Ensemble
    from gregpackagescpp_b200.ics import ensemble
    off, m, r, x, v = ensemble(args.ens_systems, 4)
    e = Ensemble(off, m, x, v, r, merge=True, dt=600.0, device=local)
    if args.ens_config:
        threads, ib = (int(t) for t in args.ens_config.split(","))
        e.set_threads(threads)
        e.set_bodies_per_thread(ib)
    else:
        threads, tune_ms = e.autotune()
    # at least one 16-step chunk in the warm-up, so that the step graph is captured and instantiated
    # before the timed region
    e.evolve(max(args.warmup, 16))
    counts0, merges0, l0 = e.counts()
    K = max(args.ens_steps, 16)
    ns = e.evolve(K)
    counts, merges, l1 = e.counts()
    inter = float((counts.astype(np.float64) * (counts - 1)).sum())
    secs = ns * 1e-9
    line = {"workload": f"ensemble of {len(off) - 1} systems, N~U{{3..2048}}, KDK dt=600 s, merges, FP32 forces",
            "unit": "ensemble steps/s", "value": (len(off) - 1) * K / secs, "system_steps_per_s": (len(off) - 1) * K / secs,
            "steps": K, "ms_per_step": 1e3 * secs / K, "pair_interactions_per_s": inter * K / secs,
            "bodies": int(off[-1]), "merges_during_timed": int(merges - merges0), "autotuned_threads": threads,
            "bodies_per_thread": e.config()[1],
            "gpu_launches": int(l1 - l0), "launch": "one persistent launch per step, replayed from a CUDA graph"}
    if peak32:
        line["frac_of_fp32_peak"] = 20 * inter * K / secs / peak32
    try:
        from oracle.oracle import RefOracle
        if RefOracle.available():
            # the reference's per-system evolve on a sample of systems, one core
            import time as _t
            ro = RefOracle()
            rng = np.random.default_rng(0)
            tot_i, tot_s = 0.0, 0.0
            for s in rng.choice(len(off) - 1, 24, replace=False):
                b, k = off[s], off[s + 1]
                if k - b < 2:
                    continue
                _, _, _, rns = ro.evolve(16, m[b:k], x[b:k], v[b:k], 600.0, 4, "M66743:66740,D1:1,T1:1",
                                         r=r[b:k], coll=0)
                tot_i += 5.0 * (k - b) * (k - b - 1)
                tot_s += rns * 1e-9
            ref_ips = tot_i / tot_s
            line["reference_cpu"] = {"pair_interactions_per_s_per_core": ref_ips,
                                     "ensemble_steps_per_s_per_core_est": ref_ips / (inter / (len(off) - 1)),
                                     "sample": "24 random systems, evolve(leapfrog_kdk) 4 steps, collisions off"}
            line["reference_cpu"]["all_cores"] = ensemble_reference_all_cores(off, m, r, x, v, inter)
    except Exception as exc:
        line["reference_cpu"] = {"unavailable": str(exc)}
    if args.ens_check_systems > 0:
        line["vs_oracle"] = ensemble_oracle_check(off, m, r, x, v, e.config(), local, args.ens_check_systems)
    return line


_ENS_REF = None


def _ens_ref_worker(task):
    """One system of the reference's ensemble timing, in a worker process (each process holds its
    own copy of the reference's global body-ID set, so the workers do not contend on its mutex)."""
    global _ENS_REF
    if _ENS_REF is None:
        from oracle.oracle import RefOracle
        _ENS_REF = RefOracle()
    if task is None:
        return 0.0
    m, r, x, v, steps = task
    n = len(m)
    xo, vo, _, _ = _ENS_REF.evolve(16, m, x, v, 600.0, steps, "M66743:66740,D1:1,T1:1", r=r, coll=0)
    _ENS_REF.check_overlap_merge(m, r, np.ones(n), xo, vo)
    return float(steps) * n * (n - 1)


def ensemble_reference_all_cores(off, m, r, x, v, inter, n_sample=128, steps=4, seed=3):
    """The reference's ensemble pattern on every host core, one process per core (bdsim.cpp:82-113
    runs one gtd::system per std::thread; the reference's bodies take their IDs from one global
    mutex-guarded set, so its threads serialise on system construction, and separate processes
    measure the evolve instead): n_sample seeded systems, each evolve(leapfrog_kdk) for `steps`
    steps in one call (one initial force sweep besides the steps' own, and the system's
    construction) followed by its check_overlap merge scan.  The sample's pair work over the pool's
    wall time, scaled by the whole ensemble's pair work per step, estimates the reference's
    ensemble steps/s (system-steps/s) on this host."""
    import concurrent.futures as cf
    import multiprocessing as mp
    rng = np.random.default_rng(seed)
    pick = [int(s) for s in rng.choice(len(off) - 1, n_sample, replace=False) if off[s + 1] - off[s] >= 2]
    tasks = [(m[off[s]:off[s + 1]].copy(), r[off[s]:off[s + 1]].copy(), x[off[s]:off[s + 1]].copy(),
              v[off[s]:off[s + 1]].copy(), steps) for s in pick]
    procs = os.cpu_count() or 1
    with cf.ProcessPoolExecutor(procs, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_ens_ref_worker, [None] * procs))  # start the workers and load the library, untimed
        t0 = time.perf_counter()
        work = sum(ex.map(_ens_ref_worker, tasks))
        wall = time.perf_counter() - t0
    rate = work / wall
    return {"pair_interactions_per_s": rate, "ensemble_steps_per_s_est": rate / (inter / (len(off) - 1)),
            "processes": procs, "wall_s": wall,
            "sample": f"{len(pick)} seeded systems, evolve(leapfrog_kdk) {steps} steps in one call + check_overlap, "
                      "one system per process at a time"}


def ensemble_oracle_check(off, m, r, x, v, config, local, n_check, steps=60, seed=11):
    """The checker beside the ensemble line (untimed): the same ICs, 60 KDK steps with merges in one
    batch on the GPU (the timed configuration), and n_check seeded systems plus up to four systems
    in which the GPU merged bodies re-run one by one on the
    oracle (the reference's KDK, then its check_overlap merge scan after each step).  Survivors and
    masses must match exactly; positions and velocities are reported relative to each system's
    largest value (the FP32 pair forces carry the mixed bar of 1e-6 relative acceleration)."""
    from gregpackagescpp_b200.ensemble import Ensemble
    from oracle.oracle import Oracle
    o = Oracle()
    Gl = o.G("M66743:66740,D1:1,T1:1")
    e = Ensemble(off, m, x, v, r, merge=True, dt=600.0, device=local)
    e.set_threads(config[0])
    e.set_bodies_per_thread(config[1])
    e.evolve(steps)
    st = e.state()
    counts, merges, _ = e.counts()
    pick = [int(s) for s in np.random.default_rng(seed).choice(len(off) - 1, n_check, replace=False)]
    # and the systems in which merges happened (up to 4), so that merges are compared too
    merged = [int(s) for s in np.nonzero(counts < np.diff(off))[0] if int(s) not in pick]
    pick += merged[:4]
    t0 = time.perf_counter()
    worst_x = worst_v = 0.0
    same_survivors = same_mass = True
    gpu_merges = oracle_merges = 0
    for s in pick:
        b, k = off[s], off[s + 1]
        rows = np.concatenate([m[b:k, None], r[b:k, None], np.ones((k - b, 1)), x[b:k], v[b:k],
                               np.zeros((k - b, 3))], 1)
        rows = o.merge_overlapping(rows)
        for _ in range(steps):
            xo, vo, ao = o.evolve(16, rows[:, 0].copy(), rows[:, 3:6].copy(), rows[:, 6:9].copy(), 600.0, 1, Gl)
            rows = o.merge_overlapping(np.concatenate([rows[:, 0:3], xo, vo, ao], axis=1))
        gpu_merges += int((k - b) - counts[s])
        oracle_merges += int((k - b) - len(rows))
        if counts[s] != len(rows):
            same_survivors = False
            continue
        same_mass &= bool(np.array_equal(st[s]["m"], rows[:, 0]))
        worst_x = max(worst_x, float(np.abs(st[s]["x"] - rows[:, 3:6]).max() / np.abs(rows[:, 3:6]).max()))
        worst_v = max(worst_v, float(np.abs(st[s]["v"] - rows[:, 6:9]).max() / np.abs(rows[:, 6:9]).max()))
    return {"systems": len(pick), "systems_with_merges": len(merged[:4]), "steps": steps,
            "bodies": int(sum(off[s + 1] - off[s] for s in pick)),
            "same_survivors": same_survivors, "same_masses": same_mass, "merges_gpu": gpu_merges,
            "merges_oracle": oracle_merges, "merges_all_systems_gpu": int(merges),
            "x_rel_max": worst_x, "v_rel_max": worst_v, "oracle_s": time.perf_counter() - t0}


def cfg_adjoint(args, local, peak32=None, peak64=None, hbm=None):
    """Adjoint: N=16384 Plummer, FP64 KDK dt=3600 s, 2000 steps, checkpoints every 45 steps;
    loss = mean |x_T - x*|^2 with x* = forward final + N(0, (0.01 AU)^2)."""
    import torch

    from gregpackagescpp_b200.adjoint import leapfrog_final_state
    from gregpackagescpp_b200.ics import AU, plummer
    n, T, every = args.adj_n, args.adj_steps, args.adj_every
    m, x, v = plummer(n, 5)
    dev = torch.device("cuda", local)
    tm, tx, tv = (torch.tensor(a, dtype=torch.float64, device=dev) for a in (m, x, v))
    with torch.no_grad():
        xT, _ = leapfrog_final_state(tx, tv, tm, 6.674e-11, 3600.0, T, every)
    g = torch.Generator(device=dev).manual_seed(7)
    target = xT + 0.01 * AU * torch.randn(xT.shape, dtype=torch.float64, device=dev, generator=g)
    xa, va, ma = tx.clone().requires_grad_(), tv.clone().requires_grad_(), tm.clone().requires_grad_()
    st = torch.cuda.current_stream()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(st)
    xT, _ = leapfrog_final_state(xa, va, ma, 6.674e-11, 3600.0, T, every)
    loss = ((xT - target) ** 2).sum(-1).mean()
    e1.record(st)
    loss.backward()
    e2.record(st)
    torch.cuda.synchronize()
    fwd, bwd = e0.elapsed_time(e1), e1.elapsed_time(e2)
    line = {"workload": f"adjoint KDK N={n}, {T} steps, checkpoints every {every}", "forward_ms": fwd,
            "backward_ms": bwd, "backward_over_forward": bwd / fwd, "total_over_forward": (fwd + bwd) / fwd}
    if peak64:
        line["forward_frac_of_fp64_peak"] = 20.0 * (T + 1) * n * (n - 1) / (fwd * 1e-3) / peak64
    if args.adj_fd > 0:
        # FP64 central differences of the library's own forward on args.adj_fd seeded coordinates,
        # split over positions, velocities and masses.  The forward is chaotic at this size (2000
        # steps with close encounters), so a quotient D(h) carries, besides its O(h^2) truncation,
        # the amplified FP64 roundoff of the two loss values divided by h.  Rule: each coordinate
        # takes D at h = 1e-6, 1e-5 and 1e-4 relative; of the adjacent pairs (1e-6, 1e-5) and
        # (1e-5, 1e-4) the one whose quotients agree best gives the reference D_ref (its smaller
        # step) and the resolution |D(h_a) - D(h_b)|; a component agrees when
        # |g - D_ref| <= max(1e-5 |D_ref|, resolution).  The specified h = 1e-6 is reported on its
        # own beside it.
        rng = np.random.default_rng(8)
        steps_rel = (1e-6, 1e-5, 1e-4)

        def loss_at(args3):
            with torch.no_grad():
                y, _ = leapfrog_final_state(*args3, 6.674e-11, 3600.0, T, every)
                return float(((y - target) ** 2).sum(-1).mean())

        def fd_at(which, idx, hrel):
            base = {"x": tx, "v": tv, "m": tm}[which].reshape(-1)
            hs = hrel * abs(float(base[idx]))
            vals = []
            for sgn in (1, -1):
                args3 = [tx.clone(), tv.clone(), tm.clone()]
                args3["xvm".index(which)].reshape(-1)[idx] += sgn * hs
                vals.append(loss_at(args3))
            return (vals[0] - vals[1]) / (2 * hs)

        per = [len(c) for c in np.array_split(np.arange(args.adj_fd), 3)]  # e.g. 64 = 22 + 21 + 21
        fd_out = {"steps_rel": list(steps_rel),
                  "rule": "D_ref, res = best-agreeing adjacent pair of D(1e-6), D(1e-5), D(1e-4); agree if "
                          "|g - D_ref| <= max(1e-5 |D_ref|, res)"}
        t0 = time.perf_counter()
        for k, (which, grad) in enumerate((("x", xa.grad), ("v", va.grad), ("m", ma.grad))):
            flat = grad.reshape(-1)
            rows = []
            for idx in rng.choice(flat.numel(), per[k], replace=False):
                g = float(flat[idx])
                d = [fd_at(which, int(idx), h) for h in steps_rel]
                pairs = [(abs(d[0] - d[1]) / abs(d[0]), 0), (abs(d[1] - d[2]) / abs(d[1]), 1)]
                _, j = min(pairs)
                ref, res = d[j], abs(d[j] - d[j + 1])
                rows.append({"index": int(idx), "g": g, "D": d, "ref_step": steps_rel[j],
                             "rel": abs(g - ref) / abs(ref), "res_rel": res / abs(ref),
                             "agree": abs(g - ref) <= max(1e-5 * abs(ref), res),
                             "rel_h1e-6": abs(g - d[0]) / abs(d[0]), "res_h1e-6": abs(d[0] - d[1]) / abs(d[0])})
            rel = np.array([r["rel"] for r in rows])
            rel6 = np.array([r["rel_h1e-6"] for r in rows])
            gv = np.array([r["g"] for r in rows])
            dref = np.array([r["D"][int(np.log10(r["ref_step"])) + 6] for r in rows])
            fd_out[which] = {
                "coords": len(rows), "agree_by_rule": int(sum(r["agree"] for r in rows)),
                "within_1e-5_of_D_ref": int((rel <= 1e-5).sum()), "median_rel_vs_D_ref": float(np.median(rel)),
                "max_rel_vs_D_ref": float(rel.max()),
                "normwise_rel_vs_D_ref": float(np.abs(gv - dref).max() / np.abs(dref).max()),
                "h1e-6": {"within_1e-5": int((rel6 <= 1e-5).sum()), "median_rel": float(np.median(rel6)),
                          "max_rel": float(rel6.max())},
                "ref_step_counts": {str(h): int(sum(r["ref_step"] == h for r in rows)) for h in steps_rel[:2]},
                "disagreeing": [r for r in rows if not r["agree"]],
            }
        fd_out["wall_s"] = time.perf_counter() - t0
        line["fd_check"] = fd_out
    return line


def run_force(args, local):
    """Profiling driver: --force-calls direct-sum force evaluations (gtd_system_accelerations) of the
    seeded N = --n Plummer sphere in --force-prec, force-kernel variant --mixed-variant (the
    process default when < 0), near factor 8; prints the CUDA-event time of each call."""
    import torch

    from gregpackagescpp_b200 import _lib
    from gregpackagescpp_b200._lib import check
    from gregpackagescpp_b200.ics import plummer
    L = _lib.load()
    n = args.n
    m, x, v = plummer(n, args.seed)
    x3, v3 = np.ascontiguousarray(x.reshape(-1)), np.ascontiguousarray(v.reshape(-1))
    prec = _lib.PREC_MIXED if args.force_prec == "mixed" else _lib.PREC_F64
    h = C.c_void_p()
    check(L.gtd_system_create(C.byref(h), local, prec))
    check(L.gtd_system_set_params(h, 6.674e-11, 3600.0, 10, 0.0, 0.5))
    check(L.gtd_system_upload(h, n, m.ctypes.data, None, None, x3.ctypes.data, v3.ctypes.data))
    if args.mixed_variant >= 0:
        check(L.gtd_system_set_direct_variant(h, args.mixed_variant))
    a = np.zeros(3 * n)
    ms = []
    for _ in range(args.force_calls):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        check(L.gtd_system_accelerations(h, 0, a.ctypes.data))
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    check(L.gtd_system_destroy(h))
    print(json.dumps({"workload": f"{args.force_prec} force evaluations, N={n}", "variant": args.mixed_variant,
                      "call_ms": ms}), flush=True)


def run_comet(args, local):
    """random_comet's evolve stage as rsl9.cpp drives it (gregsys.hpp:1881-1984): N=727 bodies of
    75 m and 4.197e9 kg at rest in a 1600 m ball, n_exp = 3, d_scale = 1200 m, restitution 0.5..0.95,
    dt = 1/128 s, overlap collisions, leapfrog KDK; continue_ev_if (some body beyond max_dist, then
    50000 probing steps) and for_all_bods (restitution from the carried centre) every step.  The
    predicate stays true far longer than a benchmark runs, so max_steps fixes the steps timed.
    Arms: device callbacks (the CUDA-graph loop), host callables (the reference's contract: a host
    round trip of the state per step), the reference's own evolve on one core."""
    from gregpackagescpp_b200 import RestFromCom, System, WhileRestBelow
    from gregpackagescpp_b200.ics import comet_stage
    c = comet_stage(727, 1600.0, 75.0, 4197481476.49696707306, 3.0, 1200.0, 0.5, 0.95, 0.0, args.seed)
    dt, units, probing = 0.0625 / 8, "M1:1,D1:1,T1:1", 50000
    mmc, sf = c["min_max_cor"], c["scale_factor"]

    def fresh():
        return System(c["m"], c["x"], c["v"], r=c["r"], rest=c["rest"], timestep=dt, num_iterations=100,
                      units_format=units, collisions=3, device=local)

    def launches(s):
        k = C.c_uint64()
        _lib.check(s._L.gtd_system_launch_count(s._h, C.byref(k)))
        return k.value

    from gregpackagescpp_b200 import _lib
    K = args.comet_steps
    s = fresh()
    if args.comet_form == "eager":  # force-kernel timing keeps the loop out of the conditional graph
        s._push()
        _lib.check(s._L.gtd_system_time_force_kernels(s._h, 1))
    fab = RestFromCom(0.5, 0.95, sf, 3.0, c["com"])
    s.evolve(16, WhileRestBelow(mmc, probing), None, fab, max_steps=max(args.warmup, 3) * 64)  # warm-up
    l0 = launches(s)
    t0 = time.perf_counter()
    ns = s.evolve(16, WhileRestBelow(mmc, probing), None, fab, max_steps=K)
    wall = time.perf_counter() - t0
    st = s.callback_stats()
    line = {"workload": "random_comet evolve stage (rsl9.cpp): N=727, leapfrog KDK dt=1/128 s, overlap "
                        "collisions, restitution from the carried centre every step", "unit": "comet steps/s",
            "steps": s.steps_taken, "value": s.steps_taken / (ns * 1e-9), "us_per_step": ns * 1e-3 / s.steps_taken,
            "e2e_value": s.steps_taken / wall, "host_waits": st["host_waits"], "graph_loop": st["graph_loop"],
            "gpu_launches": launches(s) - l0}
    # host callables: the same callbacks in numpy, the state brought back every step
    h = fresh()
    cnt = {"probe": 0, "taken": 0}
    hc = {"com": c["com"].copy()}
    KH = args.comet_host_steps

    def cont():
        if cnt["taken"] >= KH:
            return False
        if (h.rest < mmc).any():
            cnt["probe"] = 0
            go = True
        else:
            go = cnt["probe"] < probing
            cnt["probe"] += 1
        cnt["taken"] += go
        return go

    def for_all(sys_):
        hc["com"] = (hc["com"] + sys_.x.sum(axis=0)) / len(sys_.m)
        de = np.sqrt(((sys_.x - hc["com"]) ** 2).sum(axis=1)) ** 3.0
        sys_.rest = 0.95 - (0.95 - 0.5) * (de / (de + sf))

    t0 = time.perf_counter()
    h.evolve(16, cont, None, for_all)
    line["host_callbacks"] = {"value": h.steps_taken / (time.perf_counter() - t0), "steps": h.steps_taken}
    try:
        from oracle.oracle import RefOracle
        if RefOracle.available():
            ro = RefOracle()
            KR = args.comet_ref_steps
            args_ref = dict(r=c["r"], rest=c["rest"], coll=3, cont=(mmc, probing),
                            rest_from_com=(0.5, 0.95, sf, 3.0, c["com"], 0))
            t0 = time.perf_counter()
            ro.evolve_callbacks(16, c["m"], c["x"], c["v"], dt, 100, units, max_steps=1, **args_ref)
            t1 = time.perf_counter()
            xr, vr, rr, kr, _ = ro.evolve_callbacks(16, c["m"], c["x"], c["v"], dt, 100, units, max_steps=KR,
                                                    **args_ref)
            t2 = time.perf_counter()
            line["reference_cpu"] = {"value": (KR - 1) / ((t2 - t1) - (t1 - t0)), "cores": 1,
                                     "sample": f"{KR} steps (one step subtracted: construction, first force)"}
            d = fresh()
            d.evolve(16, WhileRestBelow(mmc, probing), None, RestFromCom(0.5, 0.95, sf, 3.0, c["com"]),
                     max_steps=KR)
            line["final_state_rel_err"] = {"x": float(np.abs(d.x - xr).max() / np.abs(xr).max()),
                                           "v": float(np.abs(d.v - vr).max() / max(np.abs(vr).max(), 1e-300)),
                                           "steps": KR}
    except Exception as exc:  # the reference library is optional on a box
        line["reference_cpu"] = {"unavailable": str(exc)}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank, world, local = dist_init()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.drift_only:
            if rank == 0:
                print(json.dumps(drift_series(args, local)), flush=True)
        elif args.workload != "direct-mixed":
            if rank == 0:
                if args.workload == "comet":
                    run_comet(args, local)
                elif args.workload == "force":
                    run_force(args, local)
                else:
                    fn = {"direct-fp64-1024": cfg_fp64_small, "bh": cfg_bh, "ensemble": cfg_ensemble,
                          "adjoint": cfg_adjoint}[args.workload]
                    print(json.dumps(fn(args, local)), flush=True)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
