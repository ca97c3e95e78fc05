"""Host side of the correlation autotuner (no GPU): the pass classes a
schedule tunes, the cache keys, and the JSON cache round trip."""


def test_pass_classes(hb):
    s1 = hb.multipass_parameters([64, 32, 16], padding=True, n_peaks=3)
    s2 = [hb.PIVParameters(window_size=48, overlap=24), hb.PIVParameters(window_size=16, search_area_size=32, overlap=8)]
    cl = hb.tuning.pass_classes([s1, s2, s1])
    assert cl == [(128, 64, 3), (64, 32, 3), (32, 16, 3), (48, 48, 3)]  # enlarged search areas have one shape
    assert hb.tuning.pass_classes(hb.PIVParameters(window_size=24, padding=True)) == [(48, 24, 3)]


def test_cache_round_trip(hb, tmp_path):
    path = str(tmp_path / "sub" / "tune.json")
    assert hb.tuning.load_cache(path) == {}
    key = hb.tuning.tune_key("NVIDIA B200", 32, 16, 3)
    assert key == "NVIDIA B200|N=32|W=16|K=3"
    hb.tuning.save_cache(path, {key: {"variant": 1, "ms": [0.5, 0.4]}})
    assert hb.tuning.load_cache(path) == {key: {"variant": 1, "ms": [0.5, 0.4]}}
    (tmp_path / "bad.json").write_text("[1, 2]")
    import pytest

    with pytest.raises(hb.ArgumentError):
        hb.tuning.load_cache(str(tmp_path / "bad.json"))
    with pytest.raises(hb.ArgumentError):
        hb.autotune([hb.PIVParameters()], None, reps=0)
