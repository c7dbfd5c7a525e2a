"""Multi-rank logic of bench.py on CPU (gloo, world size 2).

The path shards without exchange: each rank computes its own reference shard
against the same queries, and the timed result is the maximum over ranks.
These tests run two gloo ranks on the host: the shard generation, the
max-over-ranks reduction and barrier, and the reference arm under torchrun
(rank 0 measures and prints, the other rank exits cleanly).
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "cosine-similarity_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    class A:
        n = 64
        seed = 5

    w, r, _ = bench.dist_setup(A)
    assert (w, r) == (world, rank)
    ref, qry = bench.make_data(A, r)
    bench.barrier(w)
    mx = bench.max_over_ranks(float(10 + r), w)
    q.put((r, mx, float(ref.mz.sum()), float(qry.mz.sum())))
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res[0][1] == res[1][1] == 11.0          # max over ranks
    assert res[0][2] != res[1][2]                  # distinct reference shards
    assert res[0][3] == res[1][3]                  # the same queries everywhere


def test_reference_arm_under_torchrun():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    port = 30000 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--spectra", "300", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "pairs/s"
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
