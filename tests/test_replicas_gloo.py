"""The N > 1 path of bench.py is replicas only (one independent system per GPU, no data-path
collective): the ranks meet at barriers, the timed region is the max over ranks and the value is the
sum of the work over ranks.  Exercised here on CPU with two gloo ranks."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, os.environ["ROOT"])
import bench
rank, world, local = bench.dist_init()
t = bench.max_over_ranks(1.0 + rank, world)
s = bench.sum_over_ranks(10.0 * (rank + 1), world)
bench.barrier(world)
print(json.dumps({"rank": rank, "world": world, "max": t, "sum": s}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(code, world=2, extra_env=None):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, ROOT=ROOT, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=240) for p in procs]
    return procs, outs


def test_two_gloo_ranks_reduce_like_the_bench():
    procs, outs = _launch(WORKER)
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    lines = [json.loads(o.strip().splitlines()[-1]) for o, _ in outs]
    for ln in lines:
        assert ln["world"] == 2 and ln["max"] == 2.0 and ln["sum"] == 30.0


def test_reference_arm_runs_on_rank0_only():
    """--impl reference under two ranks: rank 0 prints one line, rank 1 exits 0 without work."""
    code = (f"import sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
            f"'--cpu-sample-n', '256', '--cpu-sample-steps', '1']; sys.path.insert(0, {ROOT!r}); "
            "import bench; bench.main()")
    procs, outs = _launch(code)
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    line0 = [ln for ln in outs[0][0].splitlines() if ln.startswith("{")]
    line1 = [ln for ln in outs[1][0].splitlines() if ln.startswith("{")]
    assert len(line0) == 1 and not line1
    d = json.loads(line0[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
