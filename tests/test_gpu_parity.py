"""Device parity: the sm_100a library against the CPU oracle, through the C ABI.

Integer peak locations and validation flags must match exactly; subpixel
displacements within 1e-3 px of the oracle's Float32 path (the tolerance of
the reference's own device-vs-CPU tests, test/test_ka.jl:22-26). Vector-grid
kernels given identical inputs must match bit for bit.
"""
import json
import math
import zlib
import os

import numpy as np
import pytest

from helpers import Grid, particle_pair, plane_decision_margin, random_positions, shear_pair

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_PX = 1e-3


@pytest.fixture(scope="module")
def hooks():
    from hammerhead_b200 import hooks

    return hooks


# --- plane analysis ---------------------------------------------------------------

@pytest.mark.parametrize("case", ["nearby", "plateau", "nonpositive", "allnan"])
def test_crafted_planes_device(ws, hooks, case):
    g = json.load(open(os.path.join(GOLDEN, "crafted_planes.json")))[case]
    R = np.array(g["plane"], np.float32)
    out, locs = hooks.analyze_planes(ws, R, n_peaks=g["k"])
    found = int(out[0, 4])
    assert found == len(g["values"])
    got = [[int(locs[0, 2 * m]), int(locs[0, 2 * m + 1])] for m in range(found)]
    assert got == g["locations"]


def _random_planes(rng, n, shape):
    nr, nc = shape
    planes = np.zeros((n, nr, nc), np.float32)
    ii = np.arange(1, nr + 1)[:, None]
    jj = np.arange(1, nc + 1)[None, :]
    for k in range(n):
        P = 0.02 * rng.uniform(size=shape)
        for _ in range(rng.integers(1, 5)):
            r0, c0 = rng.uniform(2, nr - 1), rng.uniform(2, nc - 1)
            s = rng.uniform(0.6, 2.0)
            P += rng.uniform(0.2, 1.0) * np.exp(-((ii - r0) ** 2 + (jj - c0) ** 2) / (2 * s * s))
        planes[k] = P
    return planes


@pytest.mark.parametrize("finder", ["regionalmax", "exclusion"])
@pytest.mark.parametrize("subpixel", ["gauss3", "gauss9", "none"])
@pytest.mark.parametrize("npeaks", [1, 3, 5])
def test_analyze_random_planes(ws, orc, hooks, finder, subpixel, npeaks):
    rng = np.random.default_rng(zlib.crc32(f"{finder}-{subpixel}-{npeaks}".encode()))
    planes = _random_planes(rng, 40, (32, 32))
    planes[3, 5:9, 5:9] = planes[3].max() + 1  # plateau
    out, locs = hooks.analyze_planes(ws, planes, n_peaks=npeaks, peak_finder=finder, subpixel_method=subpixel)
    K = max(npeaks, 2)
    for k in range(planes.shape[0]):
        ref, rlocs = orc.analyze_plane(planes[k], npeaks, finder, subpixel, dtype=np.float32)
        f = int(ref[4])
        assert int(out[k, 4]) == f
        assert np.array_equal(locs[k, : 2 * f], rlocs[: 2 * f])
        np.testing.assert_allclose(out[k, :2], ref[:2], atol=1e-5)
        assert out[k, 2] == ref[2] or (math.isnan(out[k, 2]) and math.isnan(ref[2]))
        np.testing.assert_allclose(out[k, 3], ref[3], rtol=1e-5, equal_nan=True)
        # alternative peaks on noise can be ill-conditioned fits (offsets of
        # hundreds of px); FP64 vs Float32 logarithms then differ relatively,
        # the more the further the fit lands outside the plane
        alt, ralt = out[k, 5:5 + 2 * (K - 1)], ref[5:5 + 2 * (K - 1)]
        inside = ~(np.abs(ralt) > 32)
        np.testing.assert_allclose(alt[inside], ralt[inside], rtol=2e-4, atol=1e-5, equal_nan=True)
        np.testing.assert_allclose(alt[~inside], ralt[~inside], rtol=1e-2, equal_nan=True)


# --- correlation planes and per-window outputs ------------------------------------

CORR_CASES = [
    dict(window_size=32, overlap=16),
    dict(window_size=16, overlap=8, padding=True, apodization="gauss"),
    dict(window_size=32, overlap=16, padding=True, apodization="gauss"),
    dict(window_size=64, overlap=32, padding=True, apodization="gauss"),
    dict(window_size=24, overlap=12, padding=True, apodization="gauss"),
    dict(window_size=48, overlap=24, padding=True, apodization="gauss"),
    dict(window_size=16, overlap=8, padding=True, apodization="none"),
    dict(window_size=24, overlap=12),
    dict(window_size=48, overlap=24),
    dict(window_size=64, overlap=32),
    dict(window_size=16, overlap=8),
    dict(window_size=32, overlap=16, correlation_method="phase", padding=True, apodization="gauss"),
    dict(window_size=32, overlap=16, peak_finder="exclusion", n_peaks=4),
    # 16 px padded windows run two per warp: the exclusion finder and the
    # other options through the half-warp groups as well
    dict(window_size=16, overlap=8, padding=True, peak_finder="exclusion", n_peaks=3),
    dict(window_size=16, overlap=8, padding=True, correlation_method="phase", n_peaks=3,
         subpixel_method="gauss9"),
]


@pytest.fixture(scope="module")
def pair256(hb):
    syn = hb.synthetic
    A, B = syn.particle_pair((256, 256), syn.uniform_flow(2.3, -1.7), seed=77)
    return A, B


@pytest.mark.parametrize("kw", CORR_CASES, ids=lambda k: "-".join(f"{a}={b}" for a, b in k.items()))
def test_correlation_planes_and_peaks(ws, orc, hb, hooks, pair256, kw):
    A, B = pair256
    p = hb.PIVParameters(**kw)
    sess = hooks.DeviceSession(ws)
    sess.stage_pair(A, B)
    x, y, _, jobs = hb.pass_grid(A.shape, p)
    jobs = jobs[:: max(1, len(jobs) // 60)]
    planes = sess.correlation_planes(p, jobs)
    out, locs, _ = sess.process_windows(p, jobs, want_locs=True)
    w = p.window_size[0]
    near_ties = []
    # the phase method divides every bin by its magnitude, so FFT round-off in
    # bins of small magnitude reaches the plane at full weight: 2.9e-5 of the
    # peak is seen for unapodized 16 px windows, against ~3e-7 for the cross
    # method
    ptol = 1e-4 if p.correlation_method == "phase" else 2e-5
    close = 0
    for q, (gi, gj, rs, cs) in enumerate(jobs):
        sa = A[rs - 1:rs - 1 + w, cs - 1:cs - 1 + w]
        sb = B[rs - 1:rs - 1 + w, cs - 1:cs - 1 + w]
        R = orc.correlation_plane(sa, sb, p)
        scale = np.abs(R).max()
        err = float(np.abs(planes[q] - R).max())
        assert err <= ptol * scale + 1e-12
        ref, rl = orc.analyze_plane(R, p.n_peaks, p.peak_finder, p.subpixel_method)
        f = int(ref[4])
        margin = plane_decision_margin(R, rl[:2 * f], locs[q, :2 * int(out[q, 4])], p.n_peaks, p.peak_finder)
        close += margin <= 1e-6 * scale
        if int(out[q, 4]) != f or not np.array_equal(locs[q, :2 * f], rl[:2 * f]):
            # admissible only where two values whose order decides the peaks
            # are closer than the two planes' own difference allows to resolve
            assert margin <= 2 * err, (q, margin, err, out[q], ref)
            near_ties.append((q, margin / scale, rl[:2 * f].tolist(), locs[q, :2 * f].tolist()))
            continue
        np.testing.assert_allclose(out[q, :2], ref[:2], atol=TOL_PX)
        np.testing.assert_allclose(out[q, 3], ref[3], rtol=1e-3, atol=1e-6, equal_nan=True)
    print(f"{len(jobs)} windows: {len(near_ties)} near-tie peak differences {near_ties}; "
          f"{close} windows with a decision margin below 1e-6 of the peak")
    assert len(near_ties) <= max(1, len(jobs) // 50)


# --- deformation ----------------------------------------------------------------------

def _deform_close(w, o):
    """The oracle solves each B-spline line in one Thomas sweep (the system
    Interpolations' Cubic(Line(OnGrid())) prefilter solves); the device cuts
    the sweeps into 64-unknown segments that start 32 unknowns early from
    zero. The neglected term is below 0.268^32 ~ 5e-19 of the value, so the
    two agree to float rounding: at most 4 ulp of the image scale (1 here),
    and in practice bit for bit at almost every pixel."""
    d = np.abs(w.astype(np.float64) - o)
    assert d.max() <= 4 * np.spacing(np.float32(1.0)), d.max()
    print(f"deformed pixels identical to the oracle: {np.mean(w == o):.6f}, max |diff| {d.max():.3g}")


@pytest.mark.parametrize("shape", [(96, 128), (300, 260)])
def test_deformation_matches_oracle(ws, orc, hooks, hb, shape):
    rng = np.random.default_rng(9)
    A = rng.uniform(size=shape).astype(np.float32)
    B = rng.uniform(size=shape).astype(np.float32)
    py = np.array([16.5, 48.5, 80.5], np.float32)
    px = np.array([16.5, 48.5, 80.5, 112.5], np.float32)
    pu = np.array([[0.8 * math.sin(0.05 * a) + 0.3 * math.cos(0.04 * b) for b in px] for a in py], np.float32)
    pv = np.array([[0.5 * math.cos(0.03 * a) - 0.4 * math.sin(0.06 * b) for b in px] for a in py], np.float32)
    gy = np.array([20.5, 50.5], np.float32)
    gx = np.array([20.5, 60.5, 100.5], np.float32)
    sess = hooks.DeviceSession(ws)
    sess.stage_pair(A, B)
    nu, nv, wA, wB = sess.apply_predictor(pu, pv, py, px, gy, gx, return_warped=True)
    cA = orc.prefilter(A)
    cB = orc.prefilter(B)
    oA, oB = orc.deform(cA, cB, A.shape, pu, pv, py, px)
    _deform_close(wA, oA)
    _deform_close(wB, oB)
    # FP64 oracle: the FP32 device deformation stays within float round-off
    dA, _ = orc.deform(orc.prefilter(A, np.float64), orc.prefilter(B, np.float64), A.shape, pu, pv, py, px,
                       dtype=np.float64)
    # FP32 rounding of the coefficients (the prefilter amplifies white noise
    # by about sqrt(3)) and of the 16-tap sums of each sample
    assert np.abs(wA - dA).max() < 4e-5
    for i, yy in enumerate(gy):
        for j, xx in enumerate(gx):
            import oracle as _o
            f = _o._fn("bilinear", "f32")
            import ctypes
            f.restype = ctypes.c_float
            f.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_float, ctypes.c_float]
            pf = np.asfortranarray(pu)
            ref = f(pf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 3, 4, float(py[0]), float(py[1] - py[0]),
                    float(px[0]), float(px[1] - px[0]), float(yy), float(xx))
            assert nu[i, j] == np.float32(ref)


# --- vector-grid kernels (identical inputs -> identical outputs) ----------------------

def _noisy_field(rng, ny, nx, nspikes=6):
    u = (2.0 + 0.1 * rng.standard_normal((ny, nx))).astype(np.float32)
    v = (-1.0 + 0.1 * rng.standard_normal((ny, nx))).astype(np.float32)
    for _ in range(nspikes):
        i, j = rng.integers(0, ny), rng.integers(0, nx)
        u[i, j] += rng.uniform(-8, 8)
        v[i, j] += rng.uniform(-8, 8)
    return u, v


@pytest.mark.parametrize("nans", [False, True])
@pytest.mark.parametrize("nb", [1, 2, 3])
def test_uod_bit_exact(ws, orc, hooks, nb, nans):
    """Neighbourhoods of 1 and 2 layers take the sorting-network path, 3 the
    general one; NaN neighbours make the median NaN (never flagged), zeros of
    either sign and ties exercise the median's order rules."""
    rng = np.random.default_rng(nb + 10 * nans)
    u, v = _noisy_field(rng, 41, 37)
    u[::7, ::5] = 0.0
    v[3::7, ::5] = -0.0
    u[10, 4:9] = u[10, 3]  # ties
    if nans:
        u[rng.uniform(size=u.shape) < 0.02] = np.nan
        v[rng.uniform(size=v.shape) < 0.02] = np.nan
    ex = rng.uniform(size=u.shape) < 0.05
    f = hooks.universal_outlier_detection(ws, u, v, 2.0, nb, 0.1, ex)
    g = orc.uod(u, v, 2.0, nb, 0.1, ex, dtype=np.float32)
    assert np.array_equal(f, g) and f.any()


def test_replace_smooth_bit_exact(ws, orc, hooks):
    rng = np.random.default_rng(4)
    u, v = _noisy_field(rng, 33, 29)
    inv = rng.uniform(size=u.shape) < 0.1
    inv[:12, :12] = True  # a large hole: the radius grows
    u1, v1 = hooks.replace_vectors(ws, u, v, inv)
    u2, v2 = orc.replace_vectors(u, v, inv, dtype=np.float32)
    assert np.array_equal(u1, u2) and np.array_equal(v1, v2)
    assert np.array_equal(hooks.smooth_field(ws, u), orc.smooth_field(u, dtype=np.float32))


def test_replace_large_neighbourhood(ws, orc, hooks):
    """More valid donors than the local buffer holds -> counting selection."""
    rng = np.random.default_rng(8)
    u, v = _noisy_field(rng, 40, 40, 0)
    inv = np.ones(u.shape, bool)
    inv[::3, 30] = False  # a sparse valid column far away
    inv[5, :] = False
    u1, v1 = hooks.replace_vectors(ws, u, v, inv)
    u2, v2 = orc.replace_vectors(u, v, inv, dtype=np.float32)
    assert np.array_equal(u1, u2) and np.array_equal(v1, v2)


@pytest.mark.parametrize("replace", [True, False])
def test_validate_with_substitution_bit_exact(ws, orc, hb, hooks, replace):
    rng = np.random.default_rng(11)
    u, v = _noisy_field(rng, 30, 34, 12)
    ratio = rng.uniform(1.0, 3.0, u.shape).astype(np.float32)
    mom = rng.uniform(0.3, 1.5, u.shape).astype(np.float32)
    nalt = 2
    au = np.full(u.shape + (nalt,), np.nan, np.float32)
    av = np.full(u.shape + (nalt,), np.nan, np.float32)
    au[..., 0] = 2.0 + 0.1 * rng.standard_normal(u.shape)
    av[..., 0] = -1.0 + 0.1 * rng.standard_normal(u.shape)
    au[::2, ::3, 1] = 5.0
    av[::2, ::3, 1] = 5.0
    mask = np.zeros(u.shape, bool)
    mask[:4, -5:] = True
    u[mask] = np.nan
    v[mask] = np.nan
    p = hb.PIVParameters(min_peak_ratio=1.2, replace_outliers=replace,
                         validation=(("correlation_moment", 1.3), ("velocity_magnitude", dict(min=0, max=9.0))))
    du, dv, do = hooks.validate(ws, p, u, v, ratio, mom, mask, au, av, force_replace=False)
    ou, ov, oo = orc.validate(p, u, v, ratio, mom, mask, au, av, force_replace=False)
    assert np.array_equal(do, oo)
    assert np.array_equal(du, ou, equal_nan=True) and np.array_equal(dv, ov, equal_nan=True)


def test_field_change_bit_exact(ws, orc, hooks):
    rng = np.random.default_rng(12)
    for n in (1, 2, 7, 1000, 16129):
        u = rng.standard_normal(n).astype(np.float32)
        v = rng.standard_normal(n).astype(np.float32)
        pu = u + 0.01 * rng.standard_normal(n).astype(np.float32)
        pv = v + 0.01 * rng.standard_normal(n).astype(np.float32)
        if n > 10:
            u[3] = np.nan
            pv[5] = np.nan
            u[7] = pu[7] = np.nan
        m = rng.uniform(size=n) < 0.1
        a = hooks.field_change(ws, u, v, pu, pv, m)
        b = orc.field_change(u, v, pu, pv, m)
        assert a == b or (math.isnan(a) and math.isnan(b)), (n, a, b)


# --- uncertainty -------------------------------------------------------------------------

@pytest.mark.parametrize("w", [16, 24, 32, 64])
def test_uq_statistics(ws, orc, hb, hooks, pair256, w):
    """Wieneke statistics of the device against the oracle. The device forms
    window means as one FP64 reduction (the oracle folds left to right in
    Float32, like the reference), so the sums agree to float round-off of
    the mean, and the final sigma to ~1e-5 relative."""
    A, B = pair256
    p = hb.PIVParameters(window_size=w, overlap=w // 2, padding=True, apodization="gauss", uncertainty=True)
    sess = hooks.DeviceSession(ws)
    sess.stage_pair(A, B)
    jobs = hb.pass_grid(A.shape, p)[3][:40]
    _, _, uq = sess.process_windows(p, jobs, want_uq=True)
    for q, (gi, gj, rs, cs) in enumerate(jobs):
        s = orc.uq_stats(A[rs - 1:rs - 1 + w, cs - 1:cs - 1 + w], B[rs - 1:rs - 1 + w, cs - 1:cs - 1 + w], "gauss")
        for comp in (0, 1):
            c = slice(44 * comp, 44 * comp + 3)
            np.testing.assert_allclose(uq[q, c], s[c], rtol=0, atol=2e-5 * np.abs(s[c]).max())
        np.testing.assert_allclose(uq[q], s, rtol=1e-3, atol=1e-6 * abs(s[3]))
        for comp in (0, 1):
            a = orc.finalize_uncertainty(uq[q, 44 * comp:44 * comp + 44])
            b = orc.finalize_uncertainty(s[44 * comp:44 * comp + 44])
            assert (math.isnan(a) and math.isnan(b)) or abs(a - b) <= 1e-4 * abs(b) + 1e-7


# --- end to end ---------------------------------------------------------------------------

def _compare_runs(r_dev, r_orc, tol=TOL_PX):
    """A device run against the oracle's Float32 run of the same schedule:
    grid masks, validation flags and sweep counts identical, and every vector
    valid in both within `tol` px (no quantile: the maximum)."""
    assert np.array_equal(r_dev.mask, r_orc["mask"])
    assert np.all(np.isnan(r_dev.u[r_dev.mask]))
    flips = np.argwhere(r_dev.outliers != r_orc["outliers"])
    assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
    assert list(r_dev.sweeps) == list(r_orc["sweeps"])
    valid = ~(r_orc["outliers"] | r_orc["mask"])
    du = np.abs(r_dev.u - r_orc["u"])[valid]
    dv = np.abs(r_dev.v - r_orc["v"])[valid]
    assert du.max() <= tol and dv.max() <= tol, (du.max(), dv.max())
    # replaced outliers are medians of valid neighbours: the same tolerance
    out = r_orc["outliers"] & ~r_orc["mask"]
    if out.any():
        assert np.abs(r_dev.u - r_orc["u"])[out].max() <= tol and np.abs(r_dev.v - r_orc["v"])[out].max() <= tol
    print(f"grid {r_dev.u.shape}: flags identical, max |du| {du.max():.2e}, max |dv| {dv.max():.2e}")
    return du, dv


def _compare_uncertainty(r_dev, r_orc, q=0.99, tol=1e-3):
    """Uncertainty: the same finite cells, and all but 1 % within `tol`.
    finalize_uncertainty (src/uncertainty.jl:162-179) takes a ring of the
    covariance sums only while its largest entry reaches 0.05 S00; where a
    ring sits at that threshold, float round-off of the sums decides whether
    it counts and sigma jumps, so the comparison is by quantile."""
    fin = np.isfinite(r_dev.uncertainty_u)
    assert np.array_equal(fin, np.isfinite(r_orc["uncertainty_u"]))
    assert np.array_equal(np.isfinite(r_dev.uncertainty_v), np.isfinite(r_orc["uncertainty_v"]))
    if fin.any():
        assert np.quantile(np.abs(r_dev.uncertainty_u - r_orc["uncertainty_u"])[fin], q) < tol
        fv = np.isfinite(r_dev.uncertainty_v)
        assert np.quantile(np.abs(r_dev.uncertainty_v - r_orc["uncertainty_v"])[fv], q) < tol


def test_run_piv_config0(hb, orc, ws):
    syn = hb.synthetic
    A, B, flow = syn.config0_pair()
    p = hb.PIVParameters(window_size=32, overlap=16)
    r = hb.run_piv(A, B, p, workspace=ws)
    o = orc.run_piv(A, B, p)
    _compare_runs(r, o)
    assert hb.rms_error(r, flow) < 0.1


def test_run_piv_config1(hb, orc, ws):
    syn = hb.synthetic
    A, B, flow = syn.config1_pair()
    passes = hb.multipass_parameters([64, 32, 16], padding=True, apodization="gauss",
                                     final=dict(max_iterations=3, uncertainty=True))
    r = hb.run_piv(A, B, passes, workspace=ws)
    o = orc.run_piv(A, B, passes, nthreads=8)
    _compare_runs(r, o)
    _compare_uncertainty(r, o)
    assert hb.rms_error(r, flow) <= 0.05


def test_run_piv_iterated_equals_repeated(hb, ws):
    A, B = shear_pair(17)
    a = hb.run_piv(A, B, hb.multipass_parameters([32, 16, 16, 16], uncertainty=True), workspace=ws)
    b = hb.run_piv(A, B, hb.multipass_parameters([32, 16], uncertainty=True,
                                                 final=dict(max_iterations=3, convergence_tol=0.0)), workspace=ws)
    for k in ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v"):
        assert np.array_equal(getattr(a, k), getattr(b, k), equal_nan=True), k
    assert np.array_equal(a.outliers, b.outliers)


def test_run_piv_mask_and_shear(hb, orc, ws):
    A, B = shear_pair(11)
    mask = np.zeros((128, 128), bool)
    mask[:48, :48] = True
    passes = hb.multipass_parameters([64, 32, 16, 16], padding=True, apodization="gauss")
    r = hb.run_piv(A, B, passes, mask=mask, workspace=ws)
    o = orc.run_piv(A, B, passes, mask=mask)
    _compare_runs(r, o)
    assert r.mask.any()


def test_run_piv_device_inputs(hb, ws):
    import torch

    syn = hb.synthetic
    A, B, _ = syn.config0_pair()
    p = hb.PIVParameters(window_size=32, overlap=16)
    r_host = hb.run_piv(A, B, p, workspace=ws)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda().T
    r_dev = hb.run_piv(dA, dB, p, workspace=ws)
    assert np.array_equal(r_host.u, r_dev.u) and np.array_equal(r_host.v, r_dev.v)


# --- the mixed batch's second schedule: [48, 24], padded, Gaussian, 3 sweeps, UQ ----------

def _cut(a, n=1024):
    return np.asfortranarray(a[:n, :n])


@pytest.mark.parametrize("shape", [(512, 512), (768, 1024), (2048, 2048)], ids=["512", "768x1024", "2048cut"])
def test_run_piv_48_24_against_oracle(hb, orc, ws, shape):
    """The [48, 24] schedule of the mixed batch (48- and 96-point transforms in
    the first pass, 48-point in the final one, up to three sweeps,
    uncertainty) end to end against the oracle's Float32 run, on the first
    pair of each image size of the batch (a 1024 x 1024 cut of the 2048^2
    pair). The device's deviation from the oracle's FP64 run is also the
    Float32 algorithm's own: it is bounded by the deviation of the oracle's
    Float32 run from its FP64 run (plus the 1e-3 px parity tolerance)."""
    syn = hb.synthetic
    sp = next(s for s in syn.config3_pairs() if s["shape"] == shape)
    A, B = syn.particle_pair(sp["shape"], sp["flow"], seed=sp["seed"])
    if shape[0] > 1024:
        A, B = _cut(A), _cut(B)
    passes = hb.multipass_parameters([48, 24], padding=True, apodization="gauss",
                                     final=dict(max_iterations=3, uncertainty=True))
    r = hb.run_piv(A, B, passes, workspace=ws)
    o = orc.run_piv(A, B, passes, nthreads=8)
    _compare_runs(r, o)
    _compare_uncertainty(r, o)
    o64 = orc.run_piv(A, B, passes, nthreads=8, dtype=np.float64)
    ok = ~(r.outliers | o64["outliers"] | r.mask)
    e_dev = np.maximum(np.abs(r.u - o64["u"]), np.abs(r.v - o64["v"]))[ok]
    e_f32 = np.maximum(np.abs(o["u"] - o64["u"]), np.abs(o["v"] - o64["v"]))[ok]
    print(f"deviation from FP64: device {e_dev.max():.3g} px, Float32 oracle {e_f32.max():.3g} px")
    assert e_dev.max() <= e_f32.max() + TOL_PX
