"""Ensemble PIV on the device (hh_run_ensemble) against the CPU restatement
of run_piv_ensemble (src/ensemble.jl:51-343)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")


def test_ensemble_of_one_pair_is_run_piv(hb, ws):
    # one summed plane is the plane itself, so the ensemble of one pair is
    # the single-sweep schedule of that pair, bit for bit
    syn = hb.synthetic
    A, B = syn.particle_pair((256, 288), syn.sine_shear_flow(2.5, 150.0), seed=41)
    passes = hb.multipass_parameters([32, 16], padding=True, apodization="gauss", uncertainty=True)
    e = hb.run_piv_ensemble([(A, B)], passes, workspace=ws)
    r = hb.run_piv(A, B, passes, workspace=ws)
    for k in FIELDS:
        assert np.array_equal(getattr(e, k), getattr(r, k), equal_nan=True), k
    assert np.array_equal(e.outliers, r.outliers)


def test_ensemble_matches_oracle(hb, orc, ws):
    syn = hb.synthetic
    flow = syn.sine_shear_flow(2.0, 200.0)
    pairs = [syn.particle_pair((192, 256), flow, seed=700 + i, ppp=0.01, noise=0.03) for i in range(12)]
    passes = hb.multipass_parameters([32, 16], padding=True, uncertainty=True)
    e = hb.run_piv_ensemble(pairs, passes, workspace=ws)
    o = orc.run_ensemble(pairs, passes, nthreads=8)
    # the planes of every pair are summed in pair order on both sides: flags
    # identical and every vector within the parity tolerance
    flips = np.argwhere(e.outliers != o["outliers"])
    assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
    assert np.abs(e.u - o["u"]).max() <= 1e-3 and np.abs(e.v - o["v"]).max() <= 1e-3
    fin = np.isfinite(e.uncertainty_u)
    assert np.array_equal(fin, np.isfinite(o["uncertainty_u"])) and fin.mean() > 0.9
    assert np.quantile(np.abs(e.uncertainty_u - o["uncertainty_u"])[fin], 0.99) < 1e-3


def test_ensemble_low_snr_and_inputs(hb, ws):
    import torch

    syn = hb.synthetic
    flow = syn.uniform_flow(2.3, -1.4)
    pairs = [syn.particle_pair((128, 160), flow, seed=900 + i, ppp=0.002, noise=0.05) for i in range(24)]
    p = hb.PIVParameters(window_size=32, overlap=16)
    e = hb.run_piv_ensemble(pairs, p, workspace=ws)
    assert np.nanmax(np.hypot(e.u - 2.3, e.v + 1.4)) < 0.1 and not e.outliers.any()
    dev = [(torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T, torch.from_numpy(np.ascontiguousarray(B.T)).cuda().T)
           for A, B in pairs]
    ed = hb.run_piv_ensemble(dev, p, workspace=ws)
    for k in FIELDS:
        assert np.array_equal(getattr(e, k), getattr(ed, k), equal_nan=True), k
    with pytest.raises(hb.DimensionMismatch):
        hb.run_piv_ensemble([pairs[0], (pairs[1][0][:100], pairs[1][1][:100])], p, workspace=ws)
