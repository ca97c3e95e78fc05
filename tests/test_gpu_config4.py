"""The large-frame time series: chained 4096 x 4096 frames with 12-bit counts
in UInt16, Poiseuille channel flow (6 px peak), 0.01 ppp, noise 0.05;
passes [128, 64, 32, 16] at 50 % overlap with the final pass at 75 %, three
sweeps and uncertainty; per-pair WIDIM and the sum-of-correlation ensemble.

A 1024 x 1024 cut of the same case is checked against the CPU restatement
(the oracle would take minutes per 4096^2 pair); the full size is checked
through properties that do not depend on it: the batched form equals the
single-pair schedule bit for bit, UInt16 frames converted on the device equal
the host conversion, and the fields match the analytic profile.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_PX = 1e-3


def _passes(hb):
    return hb.multipass_parameters([128, 64, 32]) + [
        hb.PIVParameters(window_size=16, overlap=12, max_iterations=3, uncertainty=True)]


def _f32(f16):
    # the device's conversion of a UInt16 pixel: value / 65535, correctly rounded
    return np.asfortranarray(f16.astype(np.float32) / np.float32(65535))


def _truth_rms(r, flow):
    X, Y = np.meshgrid(r.x, r.y)
    ut, vt = flow(X, Y)
    ok = ~(r.outliers | r.mask)
    return float(np.sqrt(np.mean((r.u - ut)[ok] ** 2 + (r.v - vt)[ok] ** 2)))


def test_config4_cut_against_oracle(hb, orc, ws):
    frames, flow = hb.synthetic.config4_frames(3, shape=(1024, 1024), seed=1104)
    passes = _passes(hb)
    assert [p.window_size[0] for p in passes] == [128, 64, 32, 16] and passes[-1].overlap == (12, 12)
    for k in range(2):
        A, B = _f32(frames[k]), _f32(frames[k + 1])
        r = hb.run_piv(A, B, passes, workspace=ws)
        o = orc.run_piv(A, B, passes, nthreads=8)
        # flags identical, every vector within the parity tolerance
        assert np.array_equal(r.mask, o["mask"])
        flips = np.argwhere(r.outliers != o["outliers"])
        assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
        ok = ~o["mask"]
        du, dv = np.abs(r.u - o["u"])[ok], np.abs(r.v - o["v"])[ok]
        assert du.max() <= TOL_PX and dv.max() <= TOL_PX, (du.max(), dv.max())
        assert list(r.sweeps) == list(o["sweeps"])
        both = np.isfinite(r.uncertainty_u) & np.isfinite(o["uncertainty_u"])
        assert both.mean() > 0.9
        assert np.quantile(np.abs(r.uncertainty_u - o["uncertainty_u"])[both], 0.99) < 1e-3
        # 0.01 ppp puts 2.6 particles in a 16 px window: 0.18 px RMS and 6 %
        # outliers are what the case gives (the oracle's fields are the same)
        assert _truth_rms(r, flow) < 0.3 and r.outliers.mean() < 0.1
    # sum-of-correlation ensemble of the two chained pairs, UInt16 frames
    # converted on the device
    e = hb.run_piv_ensemble([(frames[0], frames[1]), (frames[1], frames[2])], passes, workspace=ws)
    oe = orc.run_ensemble([(_f32(frames[0]), _f32(frames[1])), (_f32(frames[1]), _f32(frames[2]))], passes,
                          nthreads=8)
    flips = np.argwhere(e.outliers != oe["outliers"])
    assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
    assert np.abs(e.u - oe["u"]).max() <= TOL_PX and np.abs(e.v - oe["v"]).max() <= TOL_PX
    assert _truth_rms(e, flow) < 0.3


def test_config4_full_size(hb, ws):
    frames, flow = hb.synthetic.config4_frames(3, seed=1004)
    assert frames[0].shape == (4096, 4096) and frames[0].dtype == np.uint16
    passes = _passes(hb)
    pairs16 = [(frames[0], frames[1]), (frames[1], frames[2])]
    batch = hb.run_piv_batch(pairs16, passes, workspace=ws)
    for (a, b), rb in zip(pairs16, batch):
        rs = hb.run_piv(_f32(a), _f32(b), passes, workspace=ws)
        for k in ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v"):
            assert np.array_equal(getattr(rs, k), getattr(rb, k), equal_nan=True), k
        assert np.array_equal(rs.outliers, rb.outliers)
        assert rb.u.shape == (1021, 1021)
        assert _truth_rms(rb, flow) < 0.3 and rb.outliers.mean() < 0.1
    # summing the two pairs' planes doubles the particle images per window
    e = hb.run_piv_ensemble(pairs16, passes, workspace=ws)
    assert e.u.shape == (1021, 1021)
    assert _truth_rms(e, flow) < _truth_rms(batch[0], flow) and e.outliers.mean() < batch[0].outliers.mean()
