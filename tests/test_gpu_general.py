"""The general-shape correlation and uncertainty kernels against the oracle.

Shapes the fused kernels do not cover, all of which the reference's CPU path
accepts (src/correlators.jl:42-129, 188-355; src/types.jl:254-257;
src/uncertainty.jl:51-151): padded 128 px windows (256 x 256 planes, the
first pass of effort = :high, src/pipeline.jl:189-192), window sizes with
factors 3, 5 and 7, rectangular windows and search areas, and uncertainty
for rectangular windows and windows above 64 px. Parity rules as in
test_gpu_parity.py: planes within 2e-5 of their peak, integer peaks equal
except where the oracle plane holds a decision closer than twice the planes'
difference, subpixel u/v within 1e-3 px; end to end, flags identical and
every vector within 1e-3 px.
"""
import math

import numpy as np
import pytest

from helpers import plane_decision_margin

pytestmark = pytest.mark.gpu

TOL_PX = 1e-3

GENERAL_CASES = [
    dict(window_size=128, overlap=64, padding=True, apodization="gauss"),  # 256 x 256
    dict(window_size=40, overlap=20),  # 40 = 4 * 2 * 5
    dict(window_size=40, overlap=20, padding=True, apodization="gauss"),  # 80
    dict(window_size=20, overlap=10, padding=True),  # 40
    dict(window_size=36, overlap=18, padding=True, apodization="gauss"),  # 72 = 4 * 2 * 9
    dict(window_size=28, overlap=14, padding=True, correlation_method="phase"),  # 56 = 8 * 7
    dict(window_size=(24, 32), overlap=(12, 16), padding=True, apodization="gauss"),  # 48 x 64
    dict(window_size=(32, 20), overlap=(16, 10)),  # 32 x 20
    dict(window_size=(16, 24), search_area_size=(32, 40), overlap=(8, 12)),  # search area 32 x 40
    dict(window_size=(24, 16), search_area_size=(40, 24), overlap=(12, 8), padding=True),  # 80 x 48
    dict(window_size=40, overlap=20, peak_finder="exclusion", n_peaks=4, subpixel_method="gauss9"),
]


@pytest.fixture(scope="module")
def hooks():
    from hammerhead_b200 import hooks

    return hooks


@pytest.fixture(scope="module")
def pair384(hb):
    syn = hb.synthetic
    return syn.particle_pair((384, 352), syn.uniform_flow(3.3, -2.6), seed=177)


@pytest.mark.parametrize("kw", GENERAL_CASES, ids=lambda k: "-".join(f"{a}={b}" for a, b in k.items()))
def test_general_planes_and_peaks(ws, orc, hb, hooks, pair384, kw):
    A, B = pair384
    p = hb.PIVParameters(**kw)
    assert not hb._lib.lib().hh_corr_fused(__import__("ctypes").byref(p.to_desc()))
    sess = hooks.DeviceSession(ws)
    sess.stage_pair(A, B)
    _, _, _, jobs = hb.pass_grid(A.shape, p)
    jobs = jobs[:: max(1, len(jobs) // 40)]
    planes = sess.correlation_planes(p, jobs)
    out, locs, _ = sess.process_windows(p, jobs, want_locs=True)
    (wr, wc), (sr, sc) = p.window_size, p.search_area_size
    mr, mc = (sr - wr) // 2, (sc - wc) // 2
    f = 2 if p.padding else 1
    assert planes.shape[1:] == (f * sr, f * sc)
    ptol = 1e-4 if p.correlation_method == "phase" else 2e-5
    near = []
    for q, (gi, gj, rs, cs) in enumerate(jobs):
        sa = A[rs - 1:rs - 1 + wr, cs - 1:cs - 1 + wc]
        sb = B[rs - 1 - mr:rs - 1 + wr + mr, cs - 1 - mc:cs - 1 + wc + mc]
        R = orc.correlation_plane(sa, sb, p)
        scale = np.abs(R).max()
        err = float(np.abs(planes[q] - R).max())
        if p.correlation_method == "phase":
            # the phase method divides every bin by its magnitude, so the
            # round-off of weak bins reaches the plane at full weight (more so
            # through radix-7 stages): the device plane is held to twice the
            # Float32 oracle's own distance from the Float64 plane
            R64 = orc.correlation_plane(sa, sb, p, dtype=np.float64)
            own = float(np.abs(R - R64).max())
            assert float(np.abs(planes[q] - R64).max()) <= max(2 * own, 2e-5 * scale), (q, err / scale, own / scale)
        else:
            assert err <= ptol * scale + 1e-12, (q, err / scale)
        if (sr, sc) != (wr, wc):
            cr, cc = planes.shape[1] // 2, planes.shape[2] // 2
            keep = np.zeros(planes.shape[1:], bool)
            keep[cr - mr:cr + mr + 1, cc - mc:cc + mc + 1] = True
            assert not planes[q][~keep].any()
        ref, rl = orc.analyze_plane(R, p.n_peaks, p.peak_finder, p.subpixel_method)
        nf = int(ref[4])
        if int(out[q, 4]) != nf or not np.array_equal(locs[q, :2 * nf], rl[:2 * nf]):
            margin = plane_decision_margin(R, rl[:2 * nf], locs[q, :2 * int(out[q, 4])], p.n_peaks, p.peak_finder)
            assert margin <= 2 * err, (q, margin, err, out[q], ref)
            near.append((q, margin / scale))
            continue
        np.testing.assert_allclose(out[q, :2], ref[:2], atol=TOL_PX)
        np.testing.assert_allclose(out[q, 3], ref[3], rtol=1e-3, atol=1e-6, equal_nan=True)
    print(f"{len(jobs)} windows, {len(near)} near-tie peak differences {near}")
    assert len(near) <= max(1, len(jobs) // 50)


@pytest.mark.parametrize("w", [(24, 32), (40, 20), (80, 80), (128, 128)])
def test_general_uncertainty_statistics(ws, orc, hb, hooks, pair384, w):
    """Wieneke statistics of rectangular windows and windows above 64 px (the
    general form, its buffers in global scratch) against the oracle."""
    A, B = pair384
    p = hb.PIVParameters(window_size=w, overlap=(w[0] // 2, w[1] // 2), padding=True, apodization="gauss",
                         uncertainty=True)
    sess = hooks.DeviceSession(ws)
    sess.stage_pair(A, B)
    jobs = hb.pass_grid(A.shape, p)[3][:12]
    _, _, uq = sess.process_windows(p, jobs, want_uq=True)
    for q, (gi, gj, rs, cs) in enumerate(jobs):
        s = orc.uq_stats(A[rs - 1:rs - 1 + w[0], cs - 1:cs - 1 + w[1]], B[rs - 1:rs - 1 + w[0], cs - 1:cs - 1 + w[1]],
                         "gauss")
        for comp in (0, 1):
            c = slice(44 * comp, 44 * comp + 3)
            np.testing.assert_allclose(uq[q, c], s[c], rtol=0, atol=2e-5 * np.abs(s[c]).max())
        np.testing.assert_allclose(uq[q], s, rtol=1e-3, atol=1e-6 * max(abs(s[3]), abs(s[47])))
        # sigma is a ratio of logarithms of near-equal sums, so the few-ulp
        # difference of the window means (FP64 here, a Float32 fold in the
        # reference) is amplified: the device sigma is held to 1e-4 relative
        # or to twice the Float32 oracle's own distance from the FP64 oracle
        s64 = orc.uq_stats(A[rs - 1:rs - 1 + w[0], cs - 1:cs - 1 + w[1]].astype(np.float64),
                           B[rs - 1:rs - 1 + w[0], cs - 1:cs - 1 + w[1]].astype(np.float64), "gauss",
                           dtype=np.float64)
        for comp in (0, 1):
            a = orc.finalize_uncertainty(uq[q, 44 * comp:44 * comp + 44])
            b = orc.finalize_uncertainty(s[44 * comp:44 * comp + 44])
            c = orc.finalize_uncertainty(s64[44 * comp:44 * comp + 44])
            assert (math.isnan(a) and math.isnan(b)) or abs(a - b) <= max(1e-4 * abs(b), 2 * abs(b - c)) + 1e-7, \
                (q, comp, a, b, c)


def _compare_runs(r, o, tol=TOL_PX):
    assert np.array_equal(r.mask, o["mask"])
    flips = np.argwhere(r.outliers != o["outliers"])
    assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
    assert list(r.sweeps) == list(o["sweeps"])
    ok = ~o["mask"]
    du, dv = np.abs(r.u - o["u"])[ok], np.abs(r.v - o["v"])[ok]
    assert du.max() <= tol and dv.max() <= tol, (du.max(), dv.max())
    fin = np.isfinite(r.uncertainty_u)
    assert np.array_equal(fin, np.isfinite(o["uncertainty_u"]))
    if fin.any():
        assert np.quantile(np.abs(r.uncertainty_u - o["uncertainty_u"])[fin], 0.99) < 1e-3
    print(f"grid {r.u.shape}: flags identical, max |du| {du.max():.2e}, max |dv| {dv.max():.2e}")


def test_effort_high_1024_against_oracle(hb, orc, ws):
    """The reference's effort = :high preset ([128, 64, 32] padded, Gaussian,
    two sweeps per pass, uncertainty in the final pass) on the 1024^2 vortex
    pair, end to end against the oracle's Float32 run."""
    syn = hb.synthetic
    A, B, flow = syn.config1_pair()
    passes = hb.effort_schedule("high")
    assert [p.window_size[0] for p in passes] == [128, 64, 32] and passes[0].padding
    r = hb.run_piv(A, B, passes, workspace=ws)
    o = orc.run_piv(A, B, passes, nthreads=8)
    _compare_runs(r, o)
    assert hb.rms_error(r, flow) < 0.1


def test_rectangular_multipass_against_oracle(hb, orc, ws):
    """Rectangular windows through a whole schedule: [(48, 32), (24, 16)],
    padded, Gaussian, three sweeps, uncertainty (rectangular Wieneke
    statistics), on a 512 x 640 shear pair."""
    syn = hb.synthetic
    A, B = syn.particle_pair((512, 640), syn.sine_shear_flow(3.0, 256.0), seed=2024)
    passes = hb.multipass_parameters([(48, 32), (24, 16)], padding=True, apodization="gauss",
                                     final=dict(max_iterations=3, uncertainty=True))
    r = hb.run_piv(A, B, passes, workspace=ws)
    o = orc.run_piv(A, B, passes, nthreads=8)
    _compare_runs(r, o)


def test_general_batch_equals_single(hb, ws):
    """General-shape classes in the batched form (the plan's own scratch)
    equal the single-pair schedule bit for bit."""
    syn = hb.synthetic
    pairs = [syn.particle_pair((384, 384), syn.uniform_flow(2.1, 1.3), seed=510),
             syn.particle_pair((320, 448), syn.sine_shear_flow(2.5, 180.0), seed=511)]
    sched_a = hb.effort_schedule("high", final=dict(max_iterations=2))
    sched_b = hb.multipass_parameters([(40, 24), 20], padding=True, final=dict(uncertainty=True, max_iterations=2))
    scheds = [sched_a, sched_b]
    res = hb.run_piv_batch(pairs, scheds, workspace=ws)
    for (a, b), sc, got in zip(pairs, scheds, res):
        ref = hb.run_piv(a, b, sc, workspace=ws)
        for k in ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v"):
            assert np.array_equal(getattr(got, k), getattr(ref, k), equal_nan=True), k
        assert np.array_equal(got.outliers, ref.outliers)


def test_general_ensemble_against_oracle(hb, orc, ws):
    """Ensemble sums of 256 x 256 planes (padded 128 px windows) and of a
    rectangular pass, analysed from global memory, against the oracle."""
    syn = hb.synthetic
    flow = syn.uniform_flow(4.2, -3.1)
    pairs = [syn.particle_pair((384, 384), flow, seed=800 + i, ppp=0.01, noise=0.03) for i in range(4)]
    passes = [hb.PIVParameters(window_size=128, overlap=64, padding=True, apodization="gauss"),
              hb.PIVParameters(window_size=(48, 32), overlap=(24, 16), padding=True, uncertainty=True)]
    e = hb.run_piv_ensemble(pairs, passes, workspace=ws)
    o = orc.run_ensemble(pairs, passes, nthreads=8)
    flips = np.argwhere(e.outliers != o["outliers"])
    assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
    assert np.abs(e.u - o["u"]).max() <= TOL_PX and np.abs(e.v - o["v"]).max() <= TOL_PX


def test_hook_mask_matches_run_piv(hb, ws, hooks):
    """hh_stage_mask: the hook-level windows of a masked pair equal the
    single-pass schedule's residuals of the same pair and mask (validation
    off, so the schedule returns the raw correlation results)."""
    syn = hb.synthetic
    A, B = syn.particle_pair((256, 256), syn.uniform_flow(1.7, -2.2), seed=66)
    mask = np.zeros(A.shape, bool)
    mask[40:120, 30:90] = True
    mask[200:, 180:] = True
    p = hb.PIVParameters(window_size=32, overlap=16, padding=True, apodization="gauss", uod_enable=False,
                         replace_outliers=False)
    r = hb.run_piv(A, B, p, mask=mask, mask_threshold=0.9, workspace=ws)
    _, _, gm, jobs = hb.pass_grid(A.shape, p, mask=mask, mask_threshold=0.9)
    sess = hooks.DeviceSession(ws)
    sess.stage_pair(A, B)
    sess.stage_mask(mask)
    out, _, _ = sess.process_windows(p, jobs)
    gi, gj = jobs[:, 0] - 1, jobs[:, 1] - 1
    assert np.array_equal(out[:, 0], r.u[gi, gj]) and np.array_equal(out[:, 1], r.v[gi, gj])
    partly = [k for k, (a, b, rs, cs) in enumerate(jobs) if mask[rs - 1:rs + 31, cs - 1:cs + 31].any()]
    assert partly  # some windows are partly masked
    sess.stage_mask(None)
    out2, _, _ = sess.process_windows(p, jobs)
    assert not np.array_equal(out2[partly, 0], out[partly, 0])
