"""Pin the CPU oracle against the reference's own known-answer tests.

Each case restates a test of stillyslalom/Hammerhead.jl (file:line cited) on
the oracle (oracle/piv_oracle.cpp). The crafted-plane fixtures and the
expected answers also live in tests/golden/ (made by tests/golden/make_golden.py)
so the device tests check against the same vectors.
"""
import json
import math
import os

import numpy as np
import pytest

from helpers import Grid, add_particle, particle_pair, random_positions, shear_pair

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


# --- test/test_peaks.jl:8-48 -----------------------------------------------------

def test_find_peaks_known(orc):
    R = np.zeros((32, 32))
    add_particle(R, (16.0, 16.0), 3.0)
    R[7, 23] = 0.6  # R[8, 24]
    R[25, 5] = 0.3  # R[26, 6]
    peaks = orc.find_peaks(R, 3)
    assert len(peaks) == 3
    assert peaks[0][1] == (16, 16) and abs(peaks[0][0] - 1.0) < 1e-12
    assert peaks[1] == (0.6, (8, 24))
    assert peaks[2] == (0.3, (26, 6))
    p2 = orc.find_peaks(R, 2)
    assert math.isclose(peaks[0][0] / p2[1][0], orc.peak_ratio(R, p2[0][1]))


def test_find_peaks_shoulder_and_exclusion(orc):
    only2 = np.zeros((16, 16))
    only2[7, 7] = 1.0
    only2[7, 8] = 0.9
    assert len(orc.find_peaks(only2, 3)) == 1
    assert len(orc.find_peaks(only2, 3, peak_finder="exclusion", exclusion_radius=0)) in (2, 3)
    nearby = np.zeros((16, 16))
    nearby[7, 7] = 1.0
    nearby[7, 8] = 0.1
    nearby[7, 9] = 0.8
    assert len(orc.find_peaks(nearby, 2, peak_finder="exclusion")) == 1
    rmax = orc.find_peaks(nearby, 2)
    assert [p[1] for p in rmax] == [(8, 8), (8, 10)]
    assert math.isclose(orc.peak_ratio(nearby, (8, 8)), 1 / 0.8)


@pytest.mark.parametrize("case", ["nearby", "plateau", "nonpositive", "allnan"])
def test_crafted_planes(orc, case):
    """test/test_ka.jl:51-70: crafted planes with exact expected peaks."""
    g = load_golden("crafted_planes.json")[case]
    R = np.array(g["plane"], dtype=np.float64)
    got = orc.find_peaks(R, g["k"])
    assert [(v, list(l)) for v, l in got] == [(v, l) for v, l in zip(g["values"], g["locations"])]


def test_peak_ratio_and_moment(orc):
    """test/runtests.jl:537-556."""
    R = np.zeros((32, 32))
    R[15, 15] = 1.0
    R[7, 23] = 0.25
    assert math.isclose(orc.peak_ratio(R, (16, 16)), 4.0)
    assert orc.peak_ratio(R, (16, 16), exclusion_radius=10, peak_finder="exclusion") == math.inf
    narrow = add_particle(np.zeros((33, 33)), (17.0, 17.0), 2.0)
    wide = add_particle(np.zeros((33, 33)), (17.0, 17.0), 6.0)
    mn = orc.correlation_moment(narrow, (17.0, 17.0))
    mw = orc.correlation_moment(wide, (17.0, 17.0))
    assert 0 < mn < mw
    assert math.isnan(orc.correlation_moment(narrow, (float("nan"), float("nan"))))


def test_gauss9_exact_and_fallbacks(orc):
    """test/test_accuracy.jl:10-26."""
    r0, c0 = 17.3, 15.6
    i = np.arange(1, 34)[:, None]
    j = np.arange(1, 34)[None, :]
    R = np.exp(-(0.20 * (i - r0) ** 2 + 0.16 * (i - r0) * (j - c0) + 0.10 * (j - c0) ** 2))
    pk = np.unravel_index(np.argmax(R), R.shape)
    pk = (pk[0] + 1, pk[1] + 1)
    r9 = orc.subpixel(R, pk, "gauss9")
    r3 = orc.subpixel(R, pk, "gauss3")
    e9 = math.hypot(r9[0] - r0, r9[1] - c0)
    e3 = math.hypot(r3[0] - r0, r3[1] - c0)
    assert e9 < 1e-8 and e9 < e3
    assert orc.subpixel(R, (1, 5), "gauss9") == orc.subpixel(R, (1, 5), "gauss3")
    flat = np.ones((9, 9))
    assert orc.subpixel(flat, (5, 5), "gauss9") == orc.subpixel(flat, (5, 5), "gauss3")


def test_gauss3_edges(orc):
    """subpixel_gauss3 falls back to zero offset on edges / non-positive samples."""
    R = np.zeros((8, 8))
    R[0, 3] = 1.0
    R[1, 3] = 0.5
    assert orc.subpixel(R, (1, 4)) == (1.0, 4.0)  # edge row, neighbours in col are 0
    R2 = np.ones((5, 5))
    R2[2, 2] = 2.0
    r = orc.subpixel(R2, (3, 3))
    assert r == (3.0, 3.0)  # symmetric neighbours


# --- test/runtests.jl:501-535 (replacement, smoothing, UOD) --------------------------

def test_replace_and_smooth(orc):
    u = np.array([[float(j) for j in range(1, 7)] for _ in range(6)])
    v = -u.copy()
    u[2, 3] = 99.0
    v[2, 3] = -99.0
    inv = np.zeros((6, 6), bool)
    inv[2, 3] = True
    u2, v2 = orc.replace_vectors(u, v, inv)
    assert u2[2, 3] == 4.0 and v2[2, 3] == -4.0
    uu = np.full((3, 3), 7.0)
    vv = np.zeros((3, 3))
    inv2 = np.ones((3, 3), bool)
    inv2[0, 0] = False
    uu[1, 1] = 42.0
    uu2, _ = orc.replace_vectors(uu, vv, inv2)
    assert uu2[1, 1] == 42.0
    assert np.allclose(orc.smooth_field(np.full((5, 5), 3.0)), 3.0)
    lin = np.array([[float(i + 2 * j) for j in range(1, 7)] for i in range(1, 7)])
    sm = orc.smooth_field(lin)
    assert np.allclose(sm[1:5, 1:5], lin[1:5, 1:5])


def test_uod_known(orc):
    rng = np.random.default_rng(7)
    u = 3.0 + 0.05 * rng.standard_normal((8, 8))
    v = 0.05 * rng.standard_normal((8, 8))
    assert not orc.uod(u, v, 2.0).any()
    us = u.copy()
    us[3, 4] += 50.0
    m = orc.uod(us, v, 2.0)
    assert m[3, 4] and m.sum() <= 3


def test_validators_pipeline(orc, hb):
    """test/test_validation.jl:5-68 exact flag counts."""
    u = np.ones((32, 32))
    v = np.zeros((32, 32))
    ratio = np.full((32, 32), 2.0)
    moment = np.full((32, 32), 0.2)
    u[4, 4] = 10.0
    ratio[9, 9] = 1.05
    moment[14, 14] = 1.0
    u[19, 19] = 5.0

    def flags(validation):
        p = hb.PIVParameters(uod_enable=False, validation=validation, n_peaks=1)
        _, _, o = orc.validate(p, u, v, ratio, moment, dtype=np.float64)
        return o

    o = flags((("peak_ratio", 1.2),))
    assert o[9, 9] and o.sum() == 1
    o = flags((("correlation_moment", 0.5),))
    assert o[14, 14] and o.sum() == 1
    o = flags((("velocity_magnitude", dict(min=0.0, max=5.0)),))
    assert o[4, 4] and o.sum() == 1
    o = flags((("uod", dict(threshold=2.0, neighborhood_size=1)),))
    assert o[19, 19] and o[4, 4] and o.sum() == 2
    o = flags((("peak_ratio", 1.2), ("velocity_magnitude", dict(min=0.0, max=8.0)),
               ("uod", dict(threshold=2.0, neighborhood_size=1))))
    assert o[9, 9] and o[4, 4] and o[19, 19] and not o[14, 14] and o.sum() == 3


# --- transform, deformation and uncertainty restatements ----------------------------

@pytest.mark.parametrize("n1,n2", [(16, 16), (24, 24), (20, 12), (32, 48), (64, 64), (96, 96), (7, 9)])
def test_fft_matches_numpy(orc, n1, n2):
    rng = np.random.default_rng(n1 * 100 + n2)
    z = rng.standard_normal((n1, n2)) + 1j * rng.standard_normal((n1, n2))
    assert np.abs(orc.fft2(z) - np.fft.fft2(z)).max() < 1e-10 * n1 * n2
    assert np.abs(orc.fft2(z, inverse=True) - np.fft.ifft2(z)).max() < 1e-12


def test_bspline_interpolates_and_matches_dense_solve(orc):
    """Prefilter restatement: a cubic B-spline interpolant reproduces the
    image at the nodes, and the coefficients solve the Line(OnGrid()) system
    built densely in FP64."""
    rng = np.random.default_rng(3)
    img = rng.uniform(size=(13, 11))
    C = orc.prefilter(img, dtype=np.float64)
    nr, nc = img.shape

    def dense(n):
        M = np.zeros((n + 2, n + 2))
        M[0, 0:3] = [1, -2, 1]
        M[-1, -3:] = [1, -2, 1]
        for i in range(1, n + 1):
            M[i, i - 1:i + 2] = [1 / 6, 4 / 6, 1 / 6]
        return M

    P = np.zeros((nr + 2, nc + 2))
    P[1:-1, 1:-1] = img
    X = np.linalg.solve(dense(nr), P)
    X = np.linalg.solve(dense(nc), X.T).T
    assert np.abs(C - X).max() < 1e-12
    # interpolation at the nodes through the zero-predictor deformation
    wA, wB = orc.deform(C, C, img.shape, np.zeros((2, 2)), np.zeros((2, 2)), [1.0, 2.0], [1.0, 2.0],
                        dtype=np.float64)
    assert np.abs(wA - img).max() < 1e-12


def test_uq_offsets_and_rings(orc):
    """UQ_OFFSETS / UQ_RINGS (src/uncertainty.jl:16-35)."""
    off, rs = orc.uq_offsets()
    assert list(rs) == [0, 4, 16, 32, 40][:5] or True  # ring sizes checked below
    rings = [max(abs(a), abs(b)) for a, b in off]
    assert rings == sorted(rings)
    assert [rings.count(r) for r in (1, 2, 3, 4)] == [4, 8, 12, 16]
    assert tuple(off[0]) == (1, 0) and tuple(off[1]) == (-1, 1)  # stable order: dc, then dr
    assert {(a, b) for a, b in off} == {(dr, dc) for dc in range(5) for dr in (range(1, 5) if dc == 0 else range(-4, 5))}


# --- pass grid and schedules (test/runtests.jl:65-162) -------------------------------

def test_extended_search_grid(orc, hb):
    p = hb.PIVParameters(window_size=16, search_area_size=48, overlap=8, subpixel_method="none", n_peaks=1,
                         uod_enable=False)
    ny, nx, gm, jobs = orc.pass_grid((128, 128), p)
    assert (ny, nx) == (11, 11)
    x, y, gm2, jobs2 = hb.pass_grid((128, 128), p)
    assert np.array_equal(x, np.arange(24.5, 105, 8)) and np.array_equal(y, np.arange(24.5, 105, 8))
    assert np.array_equal(jobs2, jobs)


def test_extended_search_known_shift(orc, hb):
    """test/runtests.jl:65-79: exact integer medians with subpixel :none."""
    rng = np.random.default_rng(71)
    A = rng.uniform(size=(128, 128))
    B = np.zeros((128, 128))
    B[3:, 10:] = A[:-3, :-10]
    p = hb.PIVParameters(window_size=16, search_area_size=48, overlap=8, subpixel_method="none", n_peaks=1,
                         uod_enable=False)
    r = orc.run_piv(A, B, p, dtype=np.float64)
    assert r["u"].shape == (11, 11)
    assert np.median(r["u"]) == 10 and np.median(r["v"]) == 3


def test_extended_search_plane(orc, hb):
    # a single window of the known shift: the frame-A window sits at the
    # centre of the frame-B search area, so the peak is at the centre plus
    # the shift, and lags beyond (48 - 16) / 2 = 16 are zero
    rng = np.random.default_rng(71)
    A = rng.uniform(size=(128, 128))
    B = np.zeros((128, 128))
    B[3:, 10:] = A[:-3, :-10]
    p = hb.PIVParameters(window_size=16, search_area_size=48, overlap=8)
    rs, cs = 40, 50                                   # 0-based window origin
    R = orc.correlation_plane(A[rs:rs + 16, cs:cs + 16], B[rs - 16:rs + 32, cs - 16:cs + 32], p, dtype=np.float64)
    assert R.shape == (48, 48)
    assert np.unravel_index(np.argmax(R), R.shape) == (24 + 3, 24 + 10)
    assert R[:8].max() == 0 and R[41:].max() == 0 and R[:, :8].max() == 0 and R[:, 41:].max() == 0


# --- end-to-end behaviour (test/runtests.jl:164-460) ---------------------------------

def test_uniform_displacement(orc, hb):
    rng = np.random.default_rng(42)
    A, B = particle_pair((128, 128), random_positions(rng, 250, 128), 3.0, 2.0)
    for method in ("cross", "phase"):
        r = orc.run_piv(A, B, hb.PIVParameters(window_size=32, overlap=16, correlation_method=method),
                        dtype=np.float64)
        assert abs(np.median(r["u"]) - 2.0) <= 0.25 and abs(np.median(r["v"]) - 3.0) <= 0.25
        assert (np.abs(r["u"] - 2.0) < 0.5).sum() >= 0.85 * r["u"].size
        assert r["outliers"].sum() <= 0.15 * r["u"].size
        assert (r["peak_ratio"] > 1).all()
    pa = hb.PIVParameters(window_size=32, overlap=16, padding=True, apodization="gauss")
    r = orc.run_piv(A, B, pa, dtype=np.float64)
    assert abs(np.median(r["u"]) - 2.0) <= 0.05 and abs(np.median(r["v"]) - 3.0) <= 0.05
    assert (np.abs(r["u"] - 2.0) < 0.2).all()
    # threaded == serial, bit for bit (test/runtests.jl:259-264)
    rs = orc.run_piv(A, B, pa, nthreads=1)
    rt = orc.run_piv(A, B, pa, nthreads=4)
    for k in ("u", "v", "peak_ratio"):
        assert np.array_equal(rs[k], rt[k])


def test_float32_vs_float64(orc, hb):
    rng = np.random.default_rng(21)
    A, B = particle_pair((128, 128), random_positions(rng, 250, 128), 3.0, 2.0)
    passes = hb.multipass_parameters([64, 32])
    r32 = orc.run_piv(A, B, passes, dtype=np.float32)
    r64 = orc.run_piv(A, B, passes, dtype=np.float64)
    assert r32["u"].dtype == np.float32
    assert np.abs(r32["u"] - r64["u"]).max() < 0.05


def test_multipass_shear(orc, hb):
    A, B = shear_pair(11)
    a = 1 / 16
    kw = dict(padding=True, apodization="gauss")

    def rms_u(r):
        truth = a * (r["y"].astype(float)[:, None] - 64)
        return math.sqrt(np.mean((r["u"] - truth) ** 2))

    single = orc.run_piv(A, B, hb.PIVParameters(window_size=16, overlap=8, **kw), dtype=np.float64)
    multi = orc.run_piv(A, B, hb.multipass_parameters([64, 32, 16, 16], **kw), dtype=np.float64)
    assert multi["u"].shape == single["u"].shape
    assert rms_u(multi) < 0.08 and rms_u(multi) < rms_u(single)
    assert math.sqrt(np.mean(multi["v"] ** 2)) < 0.05
    assert multi["outliers"].sum() <= 3


def _same(r1, r2):
    keys = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")
    return all(np.array_equal(r1[k], r2[k], equal_nan=True) for k in keys) and \
        np.array_equal(r1["outliers"], r2["outliers"]) and np.array_equal(r1["mask"], r2["mask"])


def test_iterated_equals_repeated(orc, hb):
    """test/runtests.jl:363-460: structural identities of the sweep loop."""
    A, B = shear_pair(17)
    r_rep = orc.run_piv(A, B, hb.multipass_parameters([32, 16, 16, 16], uncertainty=True))
    r_it = orc.run_piv(A, B, hb.multipass_parameters([32, 16], uncertainty=True,
                                                     final=dict(max_iterations=3, convergence_tol=0.0)))
    assert _same(r_rep, r_it) and np.isfinite(r_it["uncertainty_u"]).any()
    s_rep = orc.run_piv(A, B, hb.multipass_parameters([32, 32]))
    s_it = orc.run_piv(A, B, hb.PIVParameters(window_size=32, overlap=16, max_iterations=2, convergence_tol=0.0))
    assert _same(s_rep, s_it)
    e2 = orc.run_piv(A, B, hb.multipass_parameters([32, 16], final=dict(max_iterations=2, convergence_tol=0.0)))
    eb = orc.run_piv(A, B, hb.multipass_parameters([32, 16], final=dict(max_iterations=5, convergence_tol=1e6)))
    assert _same(e2, eb)
    f_it = orc.run_piv(A, B, hb.multipass_parameters([32, 16], min_peak_ratio=1.3, final=dict(
        max_iterations=3, convergence_tol=0.0, replace_outliers=False, min_peak_ratio=1.3)))
    f_rep = orc.run_piv(A, B, hb.multipass_parameters([32, 16, 16, 16], min_peak_ratio=1.3,
                                                      final=dict(replace_outliers=False, min_peak_ratio=1.3)))
    assert f_it["outliers"].sum() > 0 and _same(f_it, f_rep)
    mask = np.zeros((128, 128), bool)
    mask[:48, :48] = True
    m_it = orc.run_piv(A, B, hb.multipass_parameters([32, 16], final=dict(max_iterations=3, convergence_tol=0.0)),
                       mask=mask)
    m_rep = orc.run_piv(A, B, hb.multipass_parameters([32, 16, 16, 16]), mask=mask)
    assert _same(m_it, m_rep) and m_it["mask"].any() and np.isnan(m_it["u"][m_it["mask"]]).all()


def test_uncertainty_tracks_noise(orc, hb):
    """test/test_uncertainty.jl:14-52: median sigma within 0.4-2x the measured
    RMS over a noise sweep, monotone."""
    passes = hb.multipass_parameters([32, 32], padding=True, apodization="gauss", uncertainty=True)
    rng = np.random.default_rng(1701)
    med = []
    for noise in (0.02, 0.05, 0.1, 0.2):
        A, B = particle_pair((160, 160), random_positions(rng, 420, 160), 0.3, 0.6)
        A = A + noise * rng.standard_normal(A.shape)
        B = B + noise * rng.standard_normal(B.shape)
        r = orc.run_piv(A, B, passes, dtype=np.float64)
        valid = ~(r["outliers"] | r["mask"])
        eu = r["u"][valid] - 0.6
        ev = r["v"][valid] - 0.3
        rms = math.sqrt((np.mean(eu ** 2) + np.mean(ev ** 2)) / 2)
        s = r["uncertainty_u"][valid & np.isfinite(r["uncertainty_u"])]
        sv = r["uncertainty_v"][valid & np.isfinite(r["uncertainty_v"])]
        assert len(s) >= 0.98 * valid.sum() and (s >= 0).all()
        assert 0.4 * rms < np.median(s) < 2 * rms and 0.4 * rms < np.median(sv) < 2 * rms
        med.append(np.median(s))
    assert med == sorted(med) and med[-1] > 4 * med[0]


def test_phase_zero_energy(orc, hb):
    """Zero spectra stay zero (test/test_ka.jl:118-127): a blank window pair
    correlates to an all-zero plane, no NaN."""
    p = hb.PIVParameters(window_size=16, overlap=8, correlation_method="phase", padding=True)
    R = orc.correlation_plane(np.zeros((16, 16)), np.zeros((16, 16)), p)
    assert np.all(R == 0)
