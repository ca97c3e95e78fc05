"""The CPU restatement of run_piv_ensemble (src/ensemble.jl:51-343).

Known answers: the ensemble of a single pair is the single-sweep run_piv of
that pair (one summed plane = the plane; pooled statistics = the pair's);
and on pairs too noisy for a single-pair peak the summed planes recover the
common displacement (test/test_ensemble.jl's premise)."""
import numpy as np


def test_ensemble_of_one_pair_is_run_piv(orc, hb):
    syn = hb.synthetic
    A, B = syn.particle_pair((192, 224), syn.sine_shear_flow(2.5, 150.0), seed=41)
    passes = hb.multipass_parameters([32, 16], padding=True, uncertainty=True)
    e = orc.run_ensemble([(A, B)], passes)
    r = orc.run_piv(A, B, passes)
    for k in ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v"):
        assert np.array_equal(e[k], r[k], equal_nan=True), k
    assert np.array_equal(e["outliers"], r["outliers"])


def test_ensemble_recovers_low_snr_displacement(orc, hb):
    syn = hb.synthetic
    flow = syn.uniform_flow(2.3, -1.4)
    pairs = [syn.particle_pair((128, 128), flow, seed=500 + i, ppp=0.002, noise=0.05) for i in range(24)]
    p = hb.PIVParameters(window_size=32, overlap=16)
    e = orc.run_ensemble(pairs, p)
    single = orc.run_piv(pairs[0][0], pairs[0][1], p)
    err_e = np.hypot(e["u"] - 2.3, e["v"] + 1.4)
    assert np.nanmax(err_e) < 0.1
    # the summed planes have cleaner peaks: no outliers, higher peak ratios
    assert e["outliers"].sum() == 0 < single["outliers"].sum()
    assert np.nanmedian(e["peak_ratio"]) > 2 * np.nanmedian(single["peak_ratio"])
