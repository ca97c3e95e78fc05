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
         and uncertainty), images resident in HBM.
e2e    = the same through run_piv with pinned host images: host->device
         copies and the result read-back inside the timed region.

--impl reference times the CPU restatement of the reference algorithm
(oracle/, all host threads) on a bounded sample of the same workload; the
reference itself is Julia, which neither this machine nor the GPU box has.

Multi-GPU: pairs are independent, so every rank runs its own batch (weak
scaling, no collective on the data path); only the timing max and the
vector counts are reduced.
"""
import argparse
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
    raise ValueError(kind)


def make_workload(hb, name, rank=0, limit=None):
    syn = hb.synthetic
    if name == "batch64":
        specs = syn.config3_pairs(seed0=1003 + 100000 * rank)
    elif name == "vortex":
        specs = [dict(shape=(1024, 1024), flow=syn.lamb_oseen_flow((512.5, 512.5), 80.0, 8.0), kind=("vortex",),
                      schedule="64-32-16", seed=1001 + 100000 * rank)]
    else:
        raise ValueError(name)
    if limit:
        specs = specs[:limit]
    pairs = []
    for sp in specs:
        A, B = syn.particle_pair(sp["shape"], sp["flow"], seed=sp["seed"])
        pairs.append(dict(sp, A=A, B=B, passes=schedule(hb, sp["schedule"])))
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
def run_reference(args, hb):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    pairs = make_workload(hb, args.workload, limit=None)
    # a bounded sample per step: one pair of each image size present
    seen, sample = set(), []
    for p in pairs:
        if p["shape"] not in seen and p["shape"][0] <= 1024:
            seen.add(p["shape"])
            sample.append(p)
    if not sample:
        sample = pairs[:1]
    nvec = sum(final_vectors(hb, p) for p in sample)
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
            "config": {"workload": workload_name(args.workload), "sample": desc},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{len(sample)} pairs per step ({desc}), {nvec} final-pass vectors"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def workload_name(w):
    return {"batch64": "mixed batch: 64 pairs (24x 512x512, 24x 768x1024, 16x 2048x2048), shear/uniform, "
                       "[64,32,16] or [48,24] padded+gauss, final 3 sweeps + UQ",
            "vortex": "1024x1024 Lamb-Oseen vortex, [64,32,16] padded+gauss, final 3 sweeps + UQ"}[w]


def cpu_baseline(hb, pairs, budget_s=20.0):
    """The oracle (CPU restatement, all host threads) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    threads = os.cpu_count() or 1
    sample = sorted(pairs, key=lambda p: p["A"].size)[:2]
    nvec, t_total, runs = 0, 0.0, 0
    t_start = time.perf_counter()
    while time.perf_counter() - t_start < budget_s or runs == 0:
        for p in sample:
            t0 = time.perf_counter()
            oracle.run_piv(p["A"], p["B"], p["passes"], nthreads=threads)
            t_total += time.perf_counter() - t0
            nvec += final_vectors(hb, p)
        runs += 1
        if runs >= 3:
            break
    desc = ", ".join(f"{p['shape'][0]}x{p['shape'][1]} {p['schedule']}" for p in sample)
    return {"value": nvec / t_total, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{runs}x [{desc}] (oracle, float32, {threads} threads)"}


# ---------------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="batch64", choices=["batch64", "vortex"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--limit", type=int, default=None, help="use only the first N pairs (debugging)")
    args = ap.parse_args()

    import hammerhead_b200 as hb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, hb)
        return

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
    dev = []
    for p in pairs:
        dev.append((torch.from_numpy(np.ascontiguousarray(p["A"].T)).cuda().T,
                    torch.from_numpy(np.ascontiguousarray(p["B"].T)).cuda().T))
    nvec_rank = sum(final_vectors(hb, p) for p in pairs)

    def step(timing=None):
        fin = 0.0
        out = []
        for p, (dA, dB) in zip(pairs, dev):
            r = hb.run_piv(dA, dB, p["passes"], workspace=ws)
            fin += float(r.pass_times_ms[-1])
            out.append(r)
        return out, fin

    for _ in range(args.warmup):
        results, _ = step()
    # accuracy of the last warm-up step against the known displacement
    rms = [hb.rms_error(r, p["flow"]) for r, p in zip(results, pairs)]
    rms_all = float(np.sqrt(np.mean(np.square(rms))))

    # ---- timed region: device-resident inputs
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    L.hh_set_profiling(ws.ctx, 1)
    hb._lib.profile_read(ws.ctx, reset=True)
    launches0 = L.hh_launch_count(ws.ctx)
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        fin_ms = 0.0
        for _ in range(args.steps):
            _, f = step()
            fin_ms += f
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = L.hh_launch_count(ws.ctx) - launches0
    prof = hb._lib.profile_read(ws.ctx, reset=True)
    L.hh_set_profiling(ws.ctx, 0)
    ms = ev0.elapsed_time(ev1) / args.steps
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    nv = torch.tensor([nvec_rank], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(nv, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    nvec_total = float(nv.item())
    value = nvec_total / (ms_max / 1e3)

    # ---- end to end: pinned host images through the public API
    pinned = [(torch.from_numpy(p["A"].T.copy()).pin_memory().numpy().T,
               torch.from_numpy(p["B"].T.copy()).pin_memory().numpy().T) for p in pairs]
    h2d = sum(2 * p["A"].size * 4 for p in pairs)
    d2h = 0
    for p in pairs:
        x, y, gm, _ = hb.pass_grid(p["A"].shape, p["passes"][-1])
        d2h += gm.size * (6 * 4 + 1)
    hb.run_piv(pinned[0][0], pinned[0][1], pairs[0]["passes"], workspace=ws)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for p, (hA, hB) in zip(pairs, pinned):
        hb.run_piv(hA, hB, p["passes"], workspace=ws)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_value = nvec_total / (float(e2e_ms.item()) / 1e3)

    # ---- roofline of the dominant kernel (the fused correlation)
    c = prof["correlate"]
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s, FMA = 2 FLOP
    achieved = (c["flops"] / (c["ms"] / 1e3)) / 1e12 if c["ms"] > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "correlate_traffic.json")
    if os.path.exists(tpath):
        tr = json.load(open(tpath))
        if c["units"] > 0:
            traffic = tr["dram_bytes_per_window"] * c["units"] / max(c["launches"], 1)
    shares = {k: round(v["ms"] / max(sum(x["ms"] for x in prof.values()), 1e-9), 4) for k, v in prof.items()}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    d = prof["deform"]

    base = None
    if rank == 0 and not args.no_cpu_baseline:
        base = cpu_baseline(hb, pairs)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_name(args.workload), "pairs_per_rank": len(pairs),
                       "final_pass_vectors_per_rank": nvec_rank, "form": "plain (per-pair device schedule)",
                       "l2": "inputs larger than L2 (704 MB per rank)", "parallelism": f"replicas x{world}"},
            "pairs_per_s": len(pairs) * world / (ms_max / 1e3),
            "final_pass_only_vectors_per_s": nvec_total / (fin_ms / args.steps / 1e3) if fin_ms > 0 else None,
            "rms_px": rms_all,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": (achieved / fp32_peak) if achieved else None, "traffic": traffic,
                         "kernel": "correlate_kernel (fused window FFT correlation + peak analysis)",
                         "peak_source": f"148 SMs x 128 FP32 lanes x 2 FLOP x {sm_max:.0f} MHz (no FP32 entry in "
                                        "MEASURED_PEAKS.json)",
                         "launches": c["launches"], "ms_per_launch": c["ms"] / max(c["launches"], 1)},
            "deform_roofline": {"bound": "hbm", "achieved": (d["bytes"] / (d["ms"] / 1e3) / 1e9) if d["ms"] else None,
                                "peak": hbm_peak, "unit": "GB/s"},
            "kernel_share": shares,
            "clocks": clk.summary(sm_max),
            "cpu_baseline": base,
        }
        if line["roofline"]["frac"] is not None:
            line["roofline"]["frac"] = round(line["roofline"]["frac"], 4)
        print(json.dumps(line))
    ws.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
