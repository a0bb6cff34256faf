"""The N > 1 path of bench.py on the CPU: ranks are independent replicas that
meet only in a barrier and a max-over-ranks of their device time (gloo), and
the reference arm under torchrun runs on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    dist, r, local, w = bench.dist_init()
    try:
        bench.barrier(dist)
        m = bench.max_over_ranks(dist, 1.5 + r)
        q.put((r, w, local, m))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[0] for g in got] == [0, 1]
    assert all(g[1] == 2 for g in got)
    assert all(g[3] == 2.5 for g in got)  # every rank sees the slowest rank's time


def test_reference_arm_under_torchrun_prints_one_line():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "3", "--ref-L", "8"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def test_replica_ensemble_is_split_between_ranks_without_overlap():
    sys.path.insert(0, str(ROOT))
    import bench

    boxes = bench.dimer_boxes_batched()
    items = list(zip(boxes, range(1, len(boxes) + 1)))
    for world in (1, 2, 4, 8):
        parts = [bench.shard(items, r, world) for r in range(world)]
        seeds = sorted(sd for p in parts for _, sd in p)
        assert seeds == list(range(1, 513))
        assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
