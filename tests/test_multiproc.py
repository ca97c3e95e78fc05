"""Multi-GPU plumbing on CPU: two gloo ranks.

Pairs are independent, so bench.py runs one batch per rank (weak scaling)
with per-rank seeds and reduces only the vector count (sum) and the step
time (max). This checks that plumbing with world_size 2 on the gloo backend:
distinct workloads per rank, the sum of the final-pass vector counts, the
max of the times, no collective on the data path.

The ensemble mode is the one path with an exchange step: its per-pass plane
and uncertainty sums are all-reduced over the ranks. Its host side is checked
here: the pair sharding, the sum reducer, and that a rank whose share is
malformed or differs from the others makes every rank raise before any
device work, instead of leaving the others waiting in a collective.
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


def _ens_worker(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "hammerhead.jl_b200"))
    import numpy as np
    import torch
    import torch.distributed as dist

    import hammerhead_b200 as hb

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    out = {"shard": hb.shard_pairs(list(range(7)))}
    red = hb.collective_reducer()
    planes = torch.arange(6, dtype=torch.float32) * (rank + 1)
    stats = torch.full((4,), 0.25 * (rank + 1), dtype=torch.float64)
    red(0, planes, stats)
    red(1, planes, None)
    out["planes"], out["stats"] = planes.tolist(), stats.tolist()
    z = np.zeros((64, 64), np.float32)
    p = hb.PIVParameters(window_size=32)
    cases = {
        "size": ([(z, z)] if rank == 0 else [(z[:48], z[:48])], p, None),
        "passes": ([(z, z)], p if rank == 0 else hb.PIVParameters(window_size=32, overlap=8), None),
        "mask": ([(z, z)], p, None if rank == 0 else np.zeros((64, 64), bool)),
        "empty": ([(z, z)] if rank == 0 else [], p, None),
    }
    for name, (pairs, params, mask) in cases.items():
        try:
            hb.run_piv_ensemble(pairs, params, mask=mask, process_group=True)
            out[name] = "no error"
        except hb.ArgumentError as e:
            out[name] = str(e)
    q.put((rank, out))
    dist.destroy_process_group()


def test_two_rank_ensemble_host_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ens_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0]["shard"] == [0, 1, 2] and out[1]["shard"] == [3, 4, 5, 6]   # contiguous, in pair order
    for r in (0, 1):
        assert out[r]["planes"] == [6.0 * k for k in range(6)]               # (1 + 2) * 2 after two sums
        assert out[r]["stats"] == [0.75] * 4                                  # stats reduced once
        assert "image size" in out[r]["size"]
        assert "passes" in out[r]["passes"]
        assert "mask" in out[r]["mask"]
    assert "rank 1 rejected" in out[0]["empty"] and "must not be empty" in out[1]["empty"]
