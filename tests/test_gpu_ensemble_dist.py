"""Ensemble PIV with its pairs split over processes: the per-pass plane and
uncertainty sums (accum[j] .+= plane, src/ensemble.jl:170-171; the Wieneke
sums, :182-183) are reduced across the processes before the analysis.

One GPU only: the two-process case runs both ranks on cuda:0 over a gloo
process group (gloo reduces CUDA tensors through host memory), so neither
rank's kernels wait on the other's; the NCCL path differs only in the
transport, which a group of one rank exercises on the library stream. Sums over processes follow another order than the single-process
pair order, so the fields agree within float rounding, not bit for bit.
"""
import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")


def _pairs(hb, n, shape=(192, 256), seed=700):
    syn = hb.synthetic
    flow = syn.sine_shear_flow(2.0, 200.0)
    return [syn.particle_pair(shape, flow, seed=seed + i, ppp=0.01, noise=0.03) for i in range(n)]


def _close(a, b, q99=1e-4, worst=1e-3, max_outl=2):
    both = ~(a.outliers | b.outliers)
    for k in ("u", "v"):
        d = np.abs(getattr(a, k) - getattr(b, k))[both]
        assert np.quantile(d, 0.99) <= q99 and d.max() <= worst, k
    assert (a.outliers != b.outliers).sum() <= max_outl
    fa, fb = np.isfinite(a.uncertainty_u), np.isfinite(b.uncertainty_u)
    assert (fa != fb).sum() <= max_outl and fa.any()
    fin = fa & fb
    assert np.quantile(np.abs(a.uncertainty_u - b.uncertainty_u)[fin], 0.99) <= 1e-5


def test_reducer_calls_and_identity(hb, ws):
    # an identity reducer sees one call per pass with the documented sizes
    # and leaves the result bit for bit the plain ensemble's
    pairs = _pairs(hb, 4)
    passes = hb.multipass_parameters([32, 16], padding=True, uncertainty=True)
    calls = []

    def rec(k, planes, stats):
        assert planes.is_cuda and planes.dtype.is_floating_point and planes.element_size() == 4
        calls.append((k, planes.numel(), None if stats is None else stats.numel()))

    e0 = hb.run_piv_ensemble(pairs, passes, workspace=ws)
    e1 = hb.run_piv_ensemble(pairs, passes, workspace=ws, reducer=rec)
    for k in FIELDS:
        assert np.array_equal(getattr(e0, k), getattr(e1, k), equal_nan=True), k
    assert [c[0] for c in calls] == [0, 1]
    for (k, npl, nst), p in zip(calls, passes):
        x, y, _, _ = hb.pass_grid(pairs[0][0].shape, p)
        njobs = len(x) * len(y)
        n = 2 * p.window_size[0]                                   # padded plane
        assert npl == njobs * n * n
        assert nst == (njobs * 88 if k == len(passes) - 1 else None)  # uncertainty on the final pass only


def test_reducer_sums_two_shares_single_pass(hb, ws):
    # one pass: the shares run one after the other, the second adding the
    # first's saved partial sums, which is the two-process reduction
    pairs = _pairs(hb, 10)
    p = hb.PIVParameters(window_size=32, overlap=16, uncertainty=True)
    saved = {}

    def keep(k, planes, stats):
        saved[k] = (planes.clone(), None if stats is None else stats.clone())

    def add(k, planes, stats):
        planes += saved[k][0]
        if stats is not None:
            stats += saved[k][1]

    hb.run_piv_ensemble(pairs[6:], p, workspace=ws, reducer=keep)
    split = hb.run_piv_ensemble(pairs[:6], p, workspace=ws, reducer=add)
    whole = hb.run_piv_ensemble(pairs, p, workspace=ws)
    _close(split, whole)


def test_reducer_failure_is_reported_and_context_survives(hb, ws):
    pairs = _pairs(hb, 2, shape=(128, 160))
    p = hb.PIVParameters(window_size=32, overlap=16)

    def boom(k, planes, stats):
        raise RuntimeError("transport down")

    with pytest.raises(RuntimeError, match="transport down"):
        hb.run_piv_ensemble(pairs, p, workspace=ws, reducer=boom)
    with pytest.raises(hb.ArgumentError):
        hb.run_piv_ensemble(pairs, p, workspace=ws, reducer=boom, process_group=True)
    a = hb.run_piv_ensemble(pairs, p, workspace=ws)
    b = hb.run_piv_ensemble(pairs, p)
    for k in FIELDS:
        assert np.array_equal(getattr(a, k), getattr(b, k), equal_nan=True), k


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "hammerhead.jl_b200"))
    import datetime

    import torch.distributed as dist

    import hammerhead_b200 as hb

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        pairs = hb.shard_pairs(_pairs(hb, 12))
        passes = hb.multipass_parameters([32, 16], padding=True, uncertainty=True)
        e = hb.run_piv_ensemble(pairs, passes, process_group=True)
        q.put((rank, {k: getattr(e, k) for k in FIELDS + ("outliers",)}))
    except BaseException as ex:  # noqa: BLE001 - reported to the parent
        q.put((rank, repr(ex)))
    finally:
        dist.destroy_process_group()


def test_two_processes_match_one(hb, ws):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert isinstance(got[r], dict), got[r]
    # the reduced sums are the same on every rank, so are the fields
    for k in FIELDS + ("outliers",):
        assert np.array_equal(got[0][k], got[1][k], equal_nan=True), k
    whole = hb.run_piv_ensemble(_pairs(hb, 12), hb.multipass_parameters([32, 16], padding=True, uncertainty=True),
                                workspace=ws)

    class R:
        pass

    r0 = R()
    for k, v in got[0].items():
        setattr(r0, k, v)
    _close(r0, whole)


def _nccl_rank(port, q):
    sys.path.insert(0, os.path.join(ROOT, "hammerhead.jl_b200"))
    import datetime

    import torch
    import torch.distributed as dist

    import hammerhead_b200 as hb

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda", 0))
    try:
        pairs = _pairs(hb, 4)
        passes = hb.multipass_parameters([32, 16], padding=True, uncertainty=True)
        e = hb.run_piv_ensemble(pairs, passes, process_group=True)
        p = hb.run_piv_ensemble(pairs, passes)
        q.put({k: bool(np.array_equal(getattr(e, k), getattr(p, k), equal_nan=True)) for k in FIELDS})
    except BaseException as ex:  # noqa: BLE001 - reported to the parent
        q.put(repr(ex))
    finally:
        dist.destroy_process_group()


def test_nccl_group_of_one(hb):
    # the NCCL transport on the library stream: a group of one rank leaves
    # every sum as it is, so the result is the plain ensemble's bit for bit
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_rank, args=(_free_port(), q))
    p.start()
    got = q.get(timeout=600)
    p.join(timeout=60)
    assert p.exitcode == 0
    assert isinstance(got, dict) and all(got.values()), got
