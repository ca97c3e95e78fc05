"""Benchmark of the B200 planar-WIDIM path: final-pass vectors/s.

Workload (default): the mixed batch -- 64 synthetic pairs, 24 at 512x512,
24 at 768x1024 (rows x cols), 16 at 2048x2048, each with a seed-drawn
sinusoidal shear or uniform translation and its own pass schedule
([64,32,16] or [48,24]); every schedule is padded, Gaussian-apodized, the
final pass iterates up to 3 sweeps and estimates Wieneke uncertainty. A step
is one complete WIDIM run of every pair. Inputs (704 MB per rank) exceed the
126 MB L2, so no explicit flush is needed between steps.

value  = final-pass vectors of all pairs (all ranks) / max-over-ranks device
         time of the whole step (every pass, sweep, deformation, validation
         and uncertainty), images resident in HBM, in the batched form: every
         pass slot of all 64 pairs as one launch per kernel, convergence
         decided on the device, the launch sequence replayed as a CUDA graph.
         The plain per-pair form (run_piv per pair) is timed beside it
         ("plain_form") with --plain timing it as the headline instead.
e2e    = the same through the public streaming API (run_piv_batch_stream)
         with pinned host images: a stream of K batches (the 64 pairs each
         time), every batch's host->device copies and result read-back inside
         the timed region, the copies of batch k+1 overlapping the analysis of
         batch k; time per batch = total / K.

rms_px is the RMS error of all final-pass vectors against the synthetic
truth; fp64_oracle_error the device's deviation from the oracle's FP64 run
on the CPU baseline's sample pairs (vectors valid in both).

Before timing, the correlation kernel's CTA shape of every pass class is
chosen on the device by the autotuner (hammerhead_b200.autotune; the choices
and the per-shape times appear as "autotune"; --no-autotune keeps the
defaults).

--impl reference times the CPU restatement of the reference algorithm
(oracle/, all host threads) on a bounded sample of the same workload; the
reference itself is Julia, which neither this machine nor the GPU box has.

Multi-GPU: pairs are independent, so every rank runs its own batch (weak
scaling, no collective on the data path); only the timing max and the
vector counts are reduced.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hammerhead.jl_b200"))

METRIC = "final-pass vectors/s"
UNIT = "vectors/s"


# ---------------------------------------------------------------------------------
def schedule(hb, kind, uq=True):
    final = dict(max_iterations=3, uncertainty=uq)
    if kind == "64-32-16":
        return hb.multipass_parameters([64, 32, 16], padding=True, apodization="gauss", final=final)
    if kind == "48-24":
        return hb.multipass_parameters([48, 24], padding=True, apodization="gauss", final=final)
    if kind == "high":  # the reference's effort = :high preset (256 x 256 planes in its first pass)
        return hb.effort_schedule("high")
    raise ValueError(kind)


def make_workload(hb, name, rank=0, limit=None):
    syn = hb.synthetic
    if name == "batch64":
        specs = syn.config3_pairs(seed0=1003 + 100000 * rank)
    elif name == "vortex":
        specs = [dict(shape=(1024, 1024), flow=syn.lamb_oseen_flow((512.5, 512.5), 80.0, 8.0), kind=("vortex",),
                      schedule="64-32-16", seed=1001 + 100000 * rank)]
    elif name == "effort_high":
        specs = [dict(shape=(2048, 2048), flow=syn.lamb_oseen_flow((1024.5, 1024.5), 160.0, 8.0), kind=("vortex",),
                      schedule="high", seed=1005 + 100000 * rank + i) for i in range(4)]
    else:
        raise ValueError(name)
    if limit:
        specs = specs[:limit]
    pairs, scheds = [], {}
    for sp in specs:
        A, B = syn.particle_pair(sp["shape"], sp["flow"], seed=sp["seed"])
        if sp["schedule"] not in scheds:
            scheds[sp["schedule"]] = schedule(hb, sp["schedule"])
        pairs.append(dict(sp, A=A, B=B, passes=scheds[sp["schedule"]]))
    return pairs


def final_vectors(hb, p):
    x, y, gm, _ = hb.pass_grid(p["A"].shape, p["passes"][-1])
    return int(gm.size - gm.sum())


# --- clocks during the timed region -----------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, sm_max_default):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            if len(r) > 8:
                for n, v in zip(names, r[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else sm_max_default,
                "reasons": sorted(reasons), "samples": len(sm)}


# --- reference arm: the CPU restatement on the host cores -----------------------------
def _load_synthetic():
    """The synthetic-pair generator (pure numpy) without importing the device
    package, so that the CPU-only reference arm loads no device library."""
    import importlib.util

    path = os.path.join(ROOT, "hammerhead.jl_b200", "hammerhead_b200", "synthetic.py")
    spec = importlib.util.spec_from_file_location("_hh_synthetic", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def oracle_schedule(oracle, kind, uq=True):
    if kind == "high":
        return oracle.multipass([128, 64, 32], padding=True, apodization="gauss", max_iterations=2,
                                final=dict(uncertainty=uq))
    final = dict(max_iterations=3, uncertainty=uq)
    sizes = {"64-32-16": [64, 32, 16], "48-24": [48, 24]}[kind]
    return oracle.multipass(sizes, padding=True, apodization="gauss", final=final)


def size_sample(specs):
    """A bounded sample of the workload with its size mix: the first pair of
    each image size (512x512, 768x1024, 2048x2048), with its own schedule."""
    seen, idx = set(), []
    for i, sp in enumerate(specs):
        if tuple(sp["shape"]) not in seen:
            seen.add(tuple(sp["shape"]))
            idx.append(i)
    return idx


def run_reference(args):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    syn = _load_synthetic()
    threads = os.cpu_count() or 1
    if args.workload == "batch64":
        specs = syn.config3_pairs(seed0=1003)
    elif args.workload == "effort_high":
        specs = [dict(shape=(2048, 2048), flow=syn.lamb_oseen_flow((1024.5, 1024.5), 160.0, 8.0),
                      schedule="high", seed=1005)]
    else:
        specs = [dict(shape=(1024, 1024), flow=syn.lamb_oseen_flow((512.5, 512.5), 80.0, 8.0),
                      schedule="64-32-16", seed=1001)]
    sample = []
    for i in size_sample(specs):
        sp = specs[i]
        A, B = syn.particle_pair(sp["shape"], sp["flow"], seed=sp["seed"])
        sample.append(dict(sp, A=A, B=B, passes=oracle_schedule(oracle, sp["schedule"])))
    nvec = sum(oracle.final_vectors(p["A"].shape, p["passes"]) for p in sample)
    for _ in range(args.warmup):
        for p in sample:
            oracle.run_piv(p["A"], p["B"], p["passes"], nthreads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for p in sample:
            oracle.run_piv(p["A"], p["B"], p["passes"], nthreads=threads)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times))
    value = nvec / t
    desc = ", ".join(f"{p['shape'][0]}x{p['shape'][1]} {p['schedule']}" for p in sample)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args.workload),
                       "sample": f"one pair of each image size per step: {desc} ({nvec} final-pass vectors)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{len(sample)} pairs per step ({desc}), {nvec} final-pass vectors"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def workload_name(w):
    return {"batch64": "mixed batch: 64 pairs (24x 512x512, 24x 768x1024, 16x 2048x2048), shear/uniform, "
                       "[64,32,16] or [48,24] padded+gauss, final 3 sweeps + UQ",
            "vortex": "1024x1024 Lamb-Oseen vortex, [64,32,16] padded+gauss, final 3 sweeps + UQ",
            "effort_high": "4 pairs of 2048x2048 Lamb-Oseen vortex, effort=:high ([128,64,32] padded+gauss, "
                           "2 sweeps per pass, UQ)"}[w]


def cpu_baseline(hb, pairs, results=None, budget_s=20.0):
    """The oracle (CPU restatement, all host threads) on a bounded sample;
    with the device `results` of `pairs`, also the device's error against
    the oracle's FP64 run of the sample pairs (the checker, untimed)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    sample_idx = size_sample(pairs)
    sample = [pairs[i] for i in sample_idx]
    nvec, t_total, runs = 0, 0.0, 0
    t_start = time.perf_counter()
    f32 = {}
    while time.perf_counter() - t_start < budget_s or runs == 0:
        for i, p in zip(sample_idx, sample):
            t0 = time.perf_counter()
            f32[i] = oracle.run_piv(p["A"], p["B"], p["passes"], nthreads=threads)
            t_total += time.perf_counter() - t0
            nvec += oracle.final_vectors(p["A"].shape, p["passes"])
        runs += 1
        if runs >= 3:
            break
    desc = ", ".join(f"{p['shape'][0]}x{p['shape'][1]} {p['schedule']}" for p in sample)
    fp64 = None
    if results is not None:
        # the device against the oracle's FP64 run, and beside it the oracle's
        # own Float32 run against the same FP64 run: the Float32 algorithm's
        # own deviation, which bounds what a Float32 device path can reach
        diffs, own = [], []
        for i in sample_idx:
            p, r, o32 = pairs[i], results[i], f32[i]
            o = oracle.run_piv(p["A"], p["B"], p["passes"], nthreads=threads, dtype=np.float64)
            ok = ~(r.outliers | r.mask | o["outliers"] | o["mask"] | o32["outliers"])
            diffs += [np.abs(r.u - o["u"])[ok], np.abs(r.v - o["v"])[ok]]
            own += [np.abs(o32["u"] - o["u"])[ok], np.abs(o32["v"] - o["v"])[ok]]
        d = np.concatenate(diffs).astype(np.float64)
        e = np.concatenate(own).astype(np.float64)
        fp64 = {"sample": desc, "components": int(d.size), "max_abs_px": float(d.max()),
                "p999_abs_px": float(np.quantile(d, 0.999)), "rms_px": float(np.sqrt(np.mean(d * d))),
                "float32_oracle_max_abs_px": float(e.max()), "float32_oracle_rms_px": float(np.sqrt(np.mean(e * e)))}
    return {"value": nvec / t_total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{runs}x [{desc}] (oracle, float32, {threads} threads)", "fp64_oracle_error": fp64}


def adjoint_bench(hb, ws, torch, stream, dev_time, reps):
    """ms per pass of the correlation-loss adjoint on the differentiation case:
    the 1024 x 1024 vortex pair, P on the 127 x 127 grid of 16-px windows at
    50 % overlap (truth + N(0, 0.3 px)); one pass = loss and dL/dP over the
    whole field, predictor and gradient resident on the device."""
    A, B, _, P, grid = hb.synthetic.config2_case()
    loss = hb.NCCLoss(A, B, window=16, overlap=8, workspace=ws)
    gny, gnx = P.shape[:2]
    Pd = torch.from_numpy(hb.adjoint.to_planes(P)).cuda()
    gd = torch.empty_like(Pd)
    for _ in range(3):
        loss.device_value_and_grad(Pd, gny, gnx, grid, gd)
    ms = dev_time(lambda: loss.device_value_and_grad(Pd, gny, gnx, grid, gd), reps)
    ms_loss = dev_time(lambda: loss.device_value_and_grad(Pd, gny, gnx, grid, None), reps)
    return {"ms_per_pass": ms, "loss_only_ms": ms_loss, "unit": "ms",
            "config": "1024x1024 Lamb-Oseen pair, P 127x127x2 (truth + N(0, 0.3 px)), "
                      "L = -sum NCC0 over 16x16 windows at 50% overlap, loss + dL/dP per pass",
            "windows": int(((A.shape[0] - 16) // 8 + 1) * ((A.shape[1] - 16) // 8 + 1))}


def timeseries_leg(hb, ws, torch, dev_time, npairs=8, reps=3, cut_check=True):
    """The large-frame time series: chained 4096^2 frames (12-bit counts in
    UInt16, 0.01 ppp, noise 0.05, Poiseuille 6 px), passes [128, 64, 32, 16]
    with the final pass at 75 % overlap, three sweeps and uncertainty; a
    bounded run of `npairs` chained pairs (frames resident on the device,
    UInt16 converted on the device) in the batched and the plain per-pair
    form, final-pass vectors/s of each; the RMS error against the flow; and
    the device's deviation from the oracle's FP64 run on a 1024^2 cut.
    Beside it, the reference's effort = :high preset ([128, 64, 32] padded,
    2 sweeps, uncertainty) on one 4096^2 pair, ms per pair, the case the
    reference publishes for its own GPU path; and the sum-of-correlation
    ensemble (run_piv_ensemble) over the same pairs and schedule, ms per
    pair, with its deviation from the oracle's FP64 ensemble of two pairs
    on the 1024^2 cut."""
    syn = hb.synthetic
    frames, flow = syn.config4_frames(npairs + 1, seed=1004)
    passes = hb.multipass_parameters([128, 64, 32]) + [
        hb.PIVParameters(window_size=16, overlap=12, max_iterations=3, uncertainty=True)]
    dev16 = [torch.from_numpy(np.ascontiguousarray(f.T)).cuda().T for f in frames]
    dev32 = [(t.float() / 65535.0) for t in dev16]  # value / 65535, as the batched form converts UInt16
    pairs16 = [(dev16[k], dev16[k + 1]) for k in range(npairs)]
    runner = hb.BatchRunner(pairs16, passes, workspace=ws)
    runner.run(read=False)
    ms_b = dev_time(lambda: runner.run(read=False), reps)
    runner.run()
    res = runner.results(copy=True)
    runner.close()
    nvec = sum(int(r.u.size - r.mask.sum()) for r in res)

    def plain():
        for k in range(npairs):
            hb.run_piv(dev32[k], dev32[k + 1], passes, workspace=ws)
    plain()
    ms_p = dev_time(plain, 1)
    X, Y = np.meshgrid(res[0].x, res[0].y)
    ut, vt = flow(X, Y)
    ok = ~(res[0].outliers | res[0].mask)
    rms = float(np.sqrt(np.mean((res[0].u - ut)[ok] ** 2 + (res[0].v - vt)[ok] ** 2)))
    out = {"config": f"{npairs} chained 4096x4096 UInt16 pairs, [128,64,32] + 16 px at 75 % overlap, 3 sweeps + UQ",
           "final_pass_vectors": nvec,
           "batched": {"value": nvec / (ms_b / 1e3), "unit": UNIT, "ms_per_pair": ms_b / npairs},
           "plain": {"value": nvec / (ms_p / 1e3), "unit": UNIT, "ms_per_pair": ms_p / npairs},
           "batched_speedup": ms_p / ms_b, "rms_px_pair0": rms, "outlier_fraction_pair0": float(res[0].outliers.mean())}
    # effort = :high on one 4096^2 pair (the reference's published 4096^2 case)
    hi = hb.effort_schedule("high")
    A, B = dev32[0], dev32[1]
    hb.run_piv(A, B, hi, workspace=ws)
    ms_hi = dev_time(lambda: hb.run_piv(A, B, hi, workspace=ws), reps)
    out["effort_high_4096"] = {
        "ms_per_pair": ms_hi, "schedule": "[128,64,32] padded + gauss, 2 sweeps per pass, UQ in the final pass",
        "reference_published_s_per_pair": {"RTX 2000 Ada, Float32, batch 8192": 2.98,
                                           "RX 6800 XT, Float32, steady state": 3.29}}
    # the sum-of-correlation ensemble (run_piv_ensemble) over the same chained
    # UInt16 pairs and schedule: one field from all pairs' summed planes
    hb.run_piv_ensemble(pairs16, passes, workspace=ws)
    ms_e = dev_time(lambda: hb.run_piv_ensemble(pairs16, passes, workspace=ws), reps)
    e = hb.run_piv_ensemble(pairs16, passes, workspace=ws)
    X, Y = np.meshgrid(e.x, e.y)
    ut, vt = flow(X, Y)
    ok = ~(e.outliers | e.mask)
    out["ensemble"] = {
        "ms_per_pair": ms_e / npairs, "pairs_per_s": npairs / (ms_e / 1e3), "field_vectors": int(e.u.size - e.mask.sum()),
        "rms_px": float(np.sqrt(np.mean((e.u - ut)[ok] ** 2 + (e.v - vt)[ok] ** 2))),
        "outlier_fraction": float(e.outliers.mean())}
    if cut_check:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        a = np.asfortranarray(frames[0][:1024, :1024].astype(np.float32) / np.float32(65535))
        b = np.asfortranarray(frames[1][:1024, :1024].astype(np.float32) / np.float32(65535))
        r = hb.run_piv(a, b, passes, workspace=ws)
        o = oracle.run_piv(a, b, passes, nthreads=os.cpu_count() or 1, dtype=np.float64)
        ok = ~(r.outliers | r.mask | o["outliers"] | o["mask"])
        d = np.concatenate([np.abs(r.u - o["u"])[ok], np.abs(r.v - o["v"])[ok]]).astype(np.float64)
        out["fp64_oracle_error_1024_cut"] = {"components": int(d.size), "max_abs_px": float(d.max()),
                                             "rms_px": float(np.sqrt(np.mean(d * d)))}
        # the ensemble of the first two chained pairs on the same cut
        c2 = [np.asfortranarray(frames[k][:1024, :1024].astype(np.float32) / np.float32(65535)) for k in range(3)]
        cp = [(c2[0], c2[1]), (c2[1], c2[2])]
        re_ = hb.run_piv_ensemble(cp, passes, workspace=ws)
        oe = oracle.run_ensemble(cp, passes, nthreads=os.cpu_count() or 1, dtype=np.float64)
        ok = ~(re_.outliers | re_.mask | oe["outliers"] | oe["mask"])
        d = np.concatenate([np.abs(re_.u - oe["u"])[ok], np.abs(re_.v - oe["v"])[ok]]).astype(np.float64)
        out["ensemble"]["fp64_oracle_error_1024_cut_2_pairs"] = {
            "components": int(d.size), "max_abs_px": float(d.max()), "rms_px": float(np.sqrt(np.mean(d * d)))}
    return out


# ---------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="batch64", choices=["batch64", "vortex", "effort_high"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain", action="store_true", help="time the plain per-pair form instead of the batched one")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form comparison step")
    ap.add_argument("--limit", type=int, default=None, help="use only the first N pairs (debugging)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default correlation CTA shapes")
    ap.add_argument("--no-timeseries", action="store_true", help="skip the 4096^2 time-series leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        # CPU only: the reference algorithm (oracle/) on the host cores; the
        # device package is not imported
        if rank == 0:
            run_reference(args)
        return

    import hammerhead_b200 as hb

    local = int(os.environ.get("LOCAL_RANK", "0"))

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        peaks = json.load(open(pk_path))

    pairs = make_workload(hb, args.workload, rank=rank, limit=args.limit)
    ws = hb.piv_workspace(device=local)
    L = hb._lib.lib()
    stream = torch.cuda.ExternalStream(ws.stream())
    dev = [(torch.from_numpy(np.ascontiguousarray(p["A"].T)).cuda().T,
            torch.from_numpy(np.ascontiguousarray(p["B"].T)).cuda().T) for p in pairs]
    scheds = [p["passes"] for p in pairs]
    nvec_rank = sum(final_vectors(hb, p) for p in pairs)
    # the correlation kernel's CTA shape per pass class, timed on this device
    # (setup, outside every timed region)
    tuned = {} if args.no_autotune else hb.autotune(scheds, ws, reps=5)

    def dev_time(fn, steps):
        """Device time of `steps` calls of fn on the context stream (ms per call)."""
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    nv = torch.tensor([nvec_rank], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(nv, op=dist.ReduceOp.SUM)
    nvec_total = float(nv.item())

    # ---- batched form, images resident in HBM, results left on the device
    runner = hb.BatchRunner(dev, scheds, workspace=ws, graph=not args.plain)
    if args.plain:
        def step():
            for p, (dA, dB) in zip(pairs, dev):
                hb.run_piv(dA, dB, p["passes"], workspace=ws)
    else:
        def step():
            runner.run(read=False)
    for _ in range(args.warmup):
        step()
    runner.run()
    results = runner.results(copy=True)
    rms = [hb.rms_error(r, p["flow"]) for r, p in zip(results, pairs)]
    rms_all = float(np.sqrt(np.mean(np.square(rms))))
    launches0 = L.hh_launch_count(ws.ctx)
    with ClockSampler(local) as clk:
        ms = dev_time(step, args.steps)
    launches = (L.hh_launch_count(ws.ctx) - launches0) // args.steps
    ms_max = max_over_ranks(ms)
    value = nvec_total / (ms_max / 1e3)

    # ---- the plain per-pair form on the same pairs (one step), for the ratio
    plain_ms = None
    if not args.plain and not args.no_plain:
        def plain_step():
            for p, (dA, dB) in zip(pairs, dev):
                hb.run_piv(dA, dB, p["passes"], workspace=ws)
        plain_step()
        plain_ms = max_over_ranks(dev_time(plain_step, 1))
    # ---- the bound on batched / plain: the batched form of the largest pairs
    #      alone (they carry most of the windows and already fill the GPU in
    #      the plain form), so plain_ms / this is the most batching can give
    big_ms = None
    if not args.plain and not args.no_plain and args.workload == "batch64":
        big = max(p["A"].size for p in pairs)
        sel = [i for i, p in enumerate(pairs) if p["A"].size == big]
        if 0 < len(sel) < len(pairs):
            rb = hb.BatchRunner([dev[i] for i in sel], [scheds[i] for i in sel], workspace=ws)
            rb.run(read=False)
            big_ms = max_over_ranks(dev_time(lambda: rb.run(read=False), max(3, args.steps // 2)))
            rb.close()

    # ---- kernel classes: one profiled run (events around every launch, no graph)
    L.hh_set_profiling(ws.ctx, 1)
    hb._lib.profile_read(ws.ctx, reset=True)
    step()
    torch.cuda.synchronize()
    prof = hb._lib.profile_read(ws.ctx, reset=True)
    L.hh_set_profiling(ws.ctx, 0)

    # ---- end to end: pinned host images through the public API, results read back
    pinned = [(torch.from_numpy(np.ascontiguousarray(p["A"].T)).pin_memory().numpy().T,
               torch.from_numpy(np.ascontiguousarray(p["B"].T)).pin_memory().numpy().T) for p in pairs]
    h2d = sum(2 * p["A"].size * 4 for p in pairs)
    d2h = int(runner.offsets[-1]) * (6 * 4 + 1)
    if args.plain:
        def e2e_step():
            for p, (hA, hB) in zip(pairs, pinned):
                hb.run_piv(hA, hB, p["passes"], workspace=ws)
        e2e_step()
        e2e_ms = max_over_ranks(dev_time(e2e_step, max(1, min(args.steps, 3))))
    else:
        # a stream of K batches (the 64 pinned pairs each time) through the
        # public streaming call: every batch's frames are copied in and its
        # results read back inside the timed region, the copies of batch k+1
        # overlapping the analysis of batch k (the first copy and the last
        # read-back are not overlapped)
        nb = max(10, args.steps)
        hb.run_piv_batch_stream([pinned], scheds, workspace=ws)

        def e2e_stream():
            hb.run_piv_batch_stream([pinned] * nb, scheds, workspace=ws)
        e2e_ms = max_over_ranks(dev_time(e2e_stream, 1)) / nb
    e2e_value = nvec_total / (e2e_ms / 1e3)

    # ---- differentiation: loss + adjoint gradient over the full predictor field
    adj = adjoint_bench(hb, ws, torch, stream, dev_time, max(args.steps, 5))

    # ---- the large-frame time series (4096^2 UInt16 chained pairs)
    ts = None if args.no_timeseries else timeseries_leg(hb, ws, torch, dev_time, cut_check=rank == 0)

    # ---- roofline of the dominant kernel (the fused correlation)
    c = prof["correlate"]
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s, FMA = 2 FLOP
    achieved = (c["flops"] / (c["ms"] / 1e3)) / 1e12 if c["ms"] > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "correlate_traffic.txt")
    if os.path.exists(tpath) and c["units"] > 0:
        per_window = {ln.split()[0]: float(ln.split()[1]) for ln in open(tpath)
                      if ln.strip() and not ln.startswith("#")}["dram_bytes_per_window"]
        traffic = per_window * c["units"] / max(c["launches"], 1)
    general = any(not L.hh_corr_fused(ctypes.byref(p.to_desc())) for sc in scheds for p in sc)
    corr_label = ("correlate_kernel + correlate_general_kernel (window FFT correlation + peak analysis; "
                  "the general-shape kernel serves the passes without a fused kernel)" if general else
                  "correlate_kernel (fused window FFT correlation + peak analysis)")
    shares = {k: round(v["ms"] / max(sum(x["ms"] for x in prof.values()), 1e-9), 4) for k, v in prof.items()}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    d = prof["deform"]

    base = None
    if rank == 0 and not args.no_cpu_baseline:
        base = cpu_baseline(hb, pairs, results)

    if rank == 0:
        form = "plain (per-pair device schedule)" if args.plain else \
            "batched (one launch per kernel per pass slot for all pairs, CUDA graph replay)"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args.workload), "pairs_per_rank": len(pairs),
                       "final_pass_vectors_per_rank": nvec_rank, "form": form,
                       "l2": "inputs larger than L2 (704 MB per rank)", "parallelism": f"replicas x{world}"},
            "pairs_per_s": len(pairs) * world / (ms_max / 1e3),
            "plain_form": None if plain_ms is None else {
                "value": nvec_total / (plain_ms / 1e3), "unit": UNIT, "ms_per_step": plain_ms,
                "batched_speedup": plain_ms / ms_max,
                "largest_pairs_batched_ms": big_ms,
                "batched_speedup_bound": (plain_ms / big_ms) if big_ms else None},
            "rms_px": rms_all,
            "fp64_oracle_error": base.pop("fp64_oracle_error") if base else None,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": (achieved / fp32_peak) if achieved else None, "traffic": traffic,
                         "kernel": corr_label,
                         "peak_source": f"148 SMs x 128 FP32 lanes x 2 FLOP x {sm_max:.0f} MHz (no FP32 entry in "
                                        "MEASURED_PEAKS.json)",
                         "launches": c["launches"], "ms_per_launch": c["ms"] / max(c["launches"], 1)},
            "deform_roofline": {"bound": "hbm", "achieved": (d["bytes"] / (d["ms"] / 1e3) / 1e9) if d["ms"] else None,
                                "peak": hbm_peak, "unit": "GB/s"},
            "kernel_share": shares,
            "adjoint": adj,
            "timeseries_4096": ts,
            "autotune": {k.split("|", 1)[1]: {"variant": e["variant"], "ms": [round(m, 4) for m in e["ms"]]}
                         for k, e in tuned.items()},
            "clocks": clk.summary(sm_max),
            "cpu_baseline": base,
        }
        if line["roofline"]["frac"] is not None:
            line["roofline"]["frac"] = round(line["roofline"]["frac"], 4)
        print(json.dumps(line))
    runner.close()
    ws.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
