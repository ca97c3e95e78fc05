"""Multi-GPU plumbing of bench.py on CPU: two gloo ranks.

Pairs are independent, so bench.py runs one batch per rank (weak scaling)
with per-rank seeds and reduces only the vector count (sum) and the step
time (max). This checks that plumbing with world_size 2 on the gloo backend:
distinct workloads per rank, the sum of the final-pass vector counts, the
max of the times, no collective on the data path.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "hammerhead.jl_b200"))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    import bench
    import hammerhead_b200 as hb

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    pairs = bench.make_workload(hb, "batch64", rank=rank, limit=2)
    nvec = sum(bench.final_vectors(hb, p) for p in pairs)
    fake_ms = 10.0 + rank
    t = torch.tensor([fake_ms], dtype=torch.float64)
    nv = torch.tensor([float(nvec)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(nv, op=dist.ReduceOp.SUM)
    q.put((rank, [p["seed"] for p in pairs], float(pairs[0]["A"].sum()), nvec, float(t.item()), float(nv.item())))
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, seeds0, s0, n0, t0, tot0), (r1, seeds1, s1, n1, t1, tot1) = out
    assert set(seeds0).isdisjoint(seeds1) and s0 != s1       # each rank analyses its own pairs
    assert t0 == t1 == 11.0                                  # max over ranks
    assert tot0 == tot1 == n0 + n1                           # whole-job vector count
