"""Autotuning of the correlation kernel's CTA shape and FFT split on the device.

Variants 0-3 run the same arithmetic on another thread mapping (the FP64
window sums are exact, so their order does not matter), so their results
must not depend on the choice. Variant 4 splits the DFTs differently, so it
is held to the oracle like the default. The tuner times the variants,
applies the fastest and keeps it in its cache.
"""
import json

import numpy as np
import pytest

from helpers import compare_runs

pytestmark = pytest.mark.gpu

SAME_ARITHMETIC = 4  # variants 0..3; variant 4 is the alternative FFT split

FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")

SCHEDULES = [
    lambda hb: hb.multipass_parameters([64, 32, 16], padding=True, apodization="gauss",
                                       final=dict(max_iterations=2, uncertainty=True)),
    lambda hb: hb.multipass_parameters([48, 24], padding=True, apodization="gauss", n_peaks=3),
    lambda hb: [hb.PIVParameters(window_size=w, overlap=w // 2, peak_finder=f)
                for w, f in ((96, "regionalmax"), (48, "exclusion"), (32, "regionalmax"), (24, "regionalmax"),
                             (16, "exclusion"))],
    lambda hb: [hb.PIVParameters(window_size=w, overlap=w // 2, padding=True) for w in (8, 12)],
]


@pytest.mark.parametrize("k", range(len(SCHEDULES)))
def test_every_shape_gives_the_same_results(hb, ws, k):
    syn = hb.synthetic
    A, B = syn.particle_pair((384, 448), syn.sine_shear_flow(3.0, 200.0), seed=51 + k)
    passes = SCHEDULES[k](hb)
    classes = hb.tuning.pass_classes(passes)
    res = []
    for v in range(SAME_ARITHMETIC):
        for n, w, _ in classes:
            hb.tuning.set_variant(ws, n, w, v)
        res.append((hb.run_piv(A, B, passes, workspace=ws), hb.run_piv_batch([(A, B)], passes, workspace=ws)[0]))
    for n, w, _ in classes:
        hb.tuning.set_variant(ws, n, w, 0)
    for a, b in res[1:]:
        for x, y in ((a, res[0][0]), (b, res[0][1])):
            for f in FIELDS:
                assert np.array_equal(getattr(x, f), getattr(y, f), equal_nan=True), f
            assert np.array_equal(x.outliers, y.outliers)


@pytest.mark.parametrize("k", range(len(SCHEDULES)))
def test_alternative_split_against_oracle(hb, orc, ws, k):
    """The alternative FFT split (variant 4) in the single-pair schedule and
    the batched form, each against the oracle's Float32 run."""
    syn = hb.synthetic
    A, B = syn.particle_pair((384, 448), syn.sine_shear_flow(3.0, 200.0), seed=51 + k)
    passes = SCHEDULES[k](hb)
    classes = hb.tuning.pass_classes(passes)
    o = orc.run_piv(A, B, passes, nthreads=8)
    try:
        for n, w, _ in classes:
            hb.tuning.set_variant(ws, n, w, 4)
        single = hb.run_piv(A, B, passes, workspace=ws)
        batched = hb.run_piv_batch([(A, B)], passes, workspace=ws)[0]
    finally:
        for n, w, _ in classes:
            hb.tuning.set_variant(ws, n, w, 0)
    for r, form in ((single, "single"), (batched, "batched")):
        du, dv = compare_runs(r, o, all_sweeps=form == "single")
        print(f"schedule {k} {form}: flags identical, max |du| {du:.2e}, max |dv| {dv:.2e}")


def test_autotune_times_applies_and_caches(hb, orc, ws, tmp_path):
    passes = hb.multipass_parameters([64, 32, 16], padding=True, apodization="gauss")
    cache = str(tmp_path / "tune.json")
    got = hb.autotune(passes, ws, cache=cache, reps=3, image_size=(768, 768))
    assert len(got) == 3
    for key, e in got.items():
        assert e["source"] == "timed" and len(e["ms"]) == hb.tuning.VARIANTS and all(m > 0 for m in e["ms"])
        assert e["variant"] == int(np.argmin(e["ms"]))
    data = json.load(open(cache))
    assert set(data) == set(got)
    again = hb.autotune(passes, ws, cache=cache)
    assert all(e["source"] == "cache" for e in again.values())
    assert {k: e["variant"] for k, e in again.items()} == {k: e["variant"] for k, e in got.items()}
    # the schedule runs with the tuned choices: exactly as with the defaults
    # when no class chose the alternative split, else within the oracle bar
    syn = hb.synthetic
    A, B = syn.particle_pair((256, 320), syn.uniform_flow(1.7, -2.2), seed=3)
    tuned = hb.run_piv(A, B, passes, workspace=ws)
    for n, w, _ in hb.tuning.pass_classes(passes):
        hb.tuning.set_variant(ws, n, w, 0)
    plain = hb.run_piv(A, B, passes, workspace=ws)
    if all(e["variant"] < SAME_ARITHMETIC for e in got.values()):
        for f in FIELDS:
            assert np.array_equal(getattr(tuned, f), getattr(plain, f), equal_nan=True), f
    else:
        compare_runs(tuned, orc.run_piv(A, B, passes))


def test_autotune_argument_errors(hb, ws):
    import ctypes

    from hammerhead_b200 import _lib

    with pytest.raises(hb.ArgumentError):
        hb.tuning.set_variant(ws, 32, 16, hb.tuning.VARIANTS)
    with pytest.raises(hb.ArgumentError):
        hb.tuning.set_variant(ws, 40, 20, 0)
    syn = hb.synthetic
    A, B = syn.particle_pair((128, 128), syn.uniform_flow(1.0, 1.0), seed=1)
    A, B = _lib.as_f32_colmajor(A), _lib.as_f32_colmajor(B)
    _lib.check(_lib.lib().hh_stage_pair(ws.ctx, _lib.fptr(A), _lib.fptr(B), 128, 128), ws.ctx)
    d = hb.PIVParameters(window_size=16, search_area_size=32, overlap=8).to_desc()
    ms = (ctypes.c_float * hb.tuning.VARIANTS)()
    best = ctypes.c_int32()
    st = _lib.lib().hh_autotune_correlation(ws.ctx, ctypes.byref(d), 2, ms, ctypes.byref(best))
    assert st == _lib.HH_ERR_ARG
    d = hb.PIVParameters(window_size=16, overlap=8).to_desc()
    assert _lib.lib().hh_autotune_correlation(ws.ctx, ctypes.byref(d), 0, ms, ctypes.byref(best)) == _lib.HH_ERR_ARG
