"""The multi-rank host logic of bench.py on CPU: world size 2 over gloo.

Each rank of `bench.py --gpus N` advances its own box (replicas, no
data-path collective); the only cross-rank step is the maximum of the
ranks' timings, checked here, and the reference arm, which rank 0 alone
runs while the other ranks exit at once.
"""
import json
import os
import subprocess
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(1.5 + rank, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_timing_is_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, 29517, out), nprocs=2, join=True, start_method="spawn")
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_prints_one_line_from_rank_zero():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29518", "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    p = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
