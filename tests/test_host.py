"""Host-side tests (no GPU): the C ABI library loads and exports every symbol
of include/hammerhead_b200.h, parameter validation mirrors PIVParameters
(test/runtests.jl:38-63), schedules mirror multipass_parameters /
effort_schedule (test/runtests.jl:105-162), the device scope check rejects
what the path does not implement, and the host-only entry points agree with
the oracle."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "hammerhead_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hh_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_header(hb):
    from hammerhead_b200 import _lib

    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), f"{s} declared in the header but not exported"
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(syms) == bound, set(syms) ^ bound
    assert L.hh_version().startswith(b"hammerhead_b200")


def header_constants():
    """Integer constants of the header: #define NAME value and enum members."""
    txt = open(os.path.join(ROOT, "include", "hammerhead_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    out = {k: int(v) for k, v in re.findall(r"#define\s+(HH_[A-Z0-9_]+)\s+(\d+)\b", txt)}
    for body in re.findall(r"enum\s*\{(.*?)\}", txt, flags=re.S):
        out.update({k: int(v) for k, v in re.findall(r"\b(HH_[A-Z0-9_]+)\s*=\s*(\d+)", body)})
    return out


def test_python_constants_match_header(hb):
    # the host layer mirrors the header's status codes, flags and pixel
    # formats by value: each HH_* integer it defines equals the header's
    from hammerhead_b200 import _lib

    hdr = header_constants()
    mirrored = {k: v for k, v in vars(_lib).items() if k.startswith("HH_") and isinstance(v, int)}
    assert {"HH_OK", "HH_ERR_OOM", "HH_BATCH_ASYNC", "HH_PIX_U16"} <= set(mirrored)
    for k, v in mirrored.items():
        assert k in hdr, f"{k} is not in the header"
        assert hdr[k] == v, (k, hdr[k], v)


def test_struct_layout(hb):
    from hammerhead_b200 import _lib
    import oracle

    assert ctypes.sizeof(_lib.hh_pass_desc) == ctypes.sizeof(oracle.Pass) == 104 + 8 * 40


def test_parameters_validation(hb):
    P = hb.PIVParameters
    p = P()
    assert p.window_size == (32, 32) and p.search_area_size == p.window_size and p.overlap == (16, 16)
    assert P(window_size=64).window_size == (64, 64)
    assert P(window_size=16, search_area_size=32, overlap=8).search_area_size == (32, 32)
    assert P(overlap=0).overlap == (0, 0)
    bad = [dict(window_size=2), dict(window_size=16, search_area_size=14), dict(window_size=16, search_area_size=31),
           dict(overlap=(32, 16)), dict(overlap=-1), dict(correlation_method="fancy"), dict(apodization="hann"),
           dict(subpixel_method="spline"), dict(peak_finder="watershed"), dict(uod_threshold=0),
           dict(uod_neighborhood=0), dict(min_peak_ratio=-1), dict(n_peaks=0), dict(max_iterations=0),
           dict(convergence_tol=-0.1)]
    for kw in bad:
        with pytest.raises(hb.ArgumentError):
            P(**kw)
    assert P().peak_finder == "regionalmax" and P(peak_finder="exclusion").peak_finder == "exclusion"
    assert "peak_finder" not in str(P()) and "peak_finder=:exclusion" in str(P(peak_finder="exclusion"))
    assert "max_iterations=3" in str(P(max_iterations=3)) and "max_iterations" not in str(P())
    with pytest.raises(hb.ArgumentError, match="window_size must be at least 4"):
        P(window_size=3)
    with pytest.raises(hb.ArgumentError, match="overlap must satisfy"):
        P(overlap=32)


def test_multipass_parameters(hb):
    mp = hb.multipass_parameters
    passes = mp([64, 32, 16], padding=True, apodization="gauss")
    assert len(passes) == 3
    assert passes[0].window_size == (64, 64) and passes[0].overlap == (32, 32)
    assert passes[2].window_size == (16, 16) and passes[2].overlap == (8, 8)
    assert all(p.padding and p.apodization == "gauss" for p in passes)
    assert mp([(64, 32)])[0].window_size == (64, 32)
    assert mp([32], overlap_fraction=0.75)[0].overlap == (24, 24)
    with pytest.raises(hb.ArgumentError):
        mp([32], overlap_fraction=1.0)
    with pytest.raises(hb.ArgumentError):
        mp([])
    fp = mp([64, 32, 16], padding=True, final=dict(n_peaks=2, keep_correlation_planes=True))
    assert all(p.padding for p in fp)
    assert fp[0].n_peaks == 3 and fp[1].n_peaks == 3 and fp[2].n_peaks == 2 and fp[2].keep_correlation_planes


def test_effort_schedule(hb):
    lo = hb.effort_schedule("low")
    assert [p.window_size for p in lo] == [(32, 32)]
    hi = hb.effort_schedule("high")
    assert [p.window_size for p in hi] == [(128, 128), (64, 64), (32, 32)]
    assert all(p.padding and p.apodization == "gauss" and p.max_iterations == 2 for p in hi)
    assert hi[-1].uncertainty and not hi[0].uncertainty
    assert [p.window_size for p in hb.effort_schedule("high", window_size=16)] == [(64, 64), (32, 32), (16, 16)]
    assert [p.window_size for p in hb.effort_schedule("medium", image_size=(48, 48))] == [(48, 48), (32, 32)]
    with pytest.raises(hb.ArgumentError):
        hb.effort_schedule("extreme")


def test_backend_scope_check(hb):
    ok = hb.multipass_parameters([64, 32, 16], padding=True, apodization="gauss", final=dict(uncertainty=True))
    hb.check_backend_params(ok)
    hb.check_backend_params([hb.PIVParameters(window_size=16, search_area_size=48, overlap=8)])
    # the reference's effort=:high preset (128 px padded windows, 256 x 256
    # planes) and any other window or search-area shape whose FFT lengths
    # factor into primes up to 61: the general-shape kernel
    hb.check_backend_params(hb.effort_schedule("high"))
    for kw in [dict(window_size=16, search_area_size=40, overlap=8),
               dict(window_size=16, search_area_size=(48, 32), overlap=8),
               dict(window_size=(32, 16), overlap=(8, 8), padding=True, uncertainty=True),
               dict(window_size=20, overlap=10, uncertainty=True),
               dict(window_size=128, overlap=64, padding=True, apodization="gauss", uncertainty=True),
               dict(window_size=(56, 44), overlap=(28, 22), correlation_method="phase")]:
        hb.check_backend_params([hb.PIVParameters(**kw)])
    for kw, msg in [(dict(subpixel_method="gauss2d"), "gauss2d"),
                    (dict(keep_correlation_planes=True), "keep_correlation_planes"),
                    (dict(window_size=67, overlap=10), "prime factors of at most 61"),
                    (dict(window_size=(1200, 1200), overlap=(600, 600), padding=True), "FFT plane of 2400 x 2400"),
                    (dict(n_peaks=9), "at most 8"),
                    (dict(uod_neighborhood=5), "uod_neighborhood")]:
        with pytest.raises(hb.ArgumentError, match=msg):
            hb.check_backend_params([hb.PIVParameters(**kw)])
    with pytest.raises(hb.ArgumentError, match="unsupported Hammerhead backend"):
        hb.run_piv(np.zeros((64, 64)), np.zeros((64, 64)), backend="cpu")
    with pytest.raises(hb.ArgumentError, match="effort cannot be combined"):
        hb.run_piv(np.zeros((64, 64)), np.zeros((64, 64)), hb.PIVParameters(), effort="low")


def test_dimension_checks(hb):
    with pytest.raises(hb.DimensionMismatch):
        hb.run_piv(np.zeros((64, 64)), np.zeros((32, 32)))
    with pytest.raises(hb.DimensionMismatch):
        hb.run_piv(np.zeros((64, 64)), np.zeros((64, 64)), mask=np.zeros((8, 8), bool))
    with pytest.raises(hb.ArgumentError):
        hb.run_piv(np.zeros((64, 64)), np.zeros((64, 64)), mask_threshold=0.0)


@pytest.mark.parametrize("shape,kw", [((128, 128), dict(window_size=32, overlap=16)),
                                      ((96, 200), dict(window_size=16, overlap=8)),
                                      ((512, 512), dict(window_size=32, overlap=24)),
                                      ((768, 1024), dict(window_size=24, overlap=12))])
def test_pass_grid_matches_oracle(hb, orc, shape, kw):
    p = hb.PIVParameters(**kw)
    x, y, gm, jobs = hb.pass_grid(shape, p)
    ny, nx, gm2, jobs2 = orc.pass_grid(shape, p)
    assert (len(y), len(x)) == (ny, nx)
    assert np.array_equal(jobs, jobs2)
    ws = p.window_size[0]
    assert x[0] == 1 + (ws - 1) / 2 and np.all(np.diff(x) == ws - p.overlap[0])


def test_pass_grid_mask(hb, orc):
    p = hb.PIVParameters(window_size=32, overlap=16)
    mask = np.zeros((128, 128), bool)
    mask[:40, :40] = True
    x, y, gm, jobs = hb.pass_grid((128, 128), p, mask, 0.5)
    ny, nx, gm2, jobs2 = orc.pass_grid((128, 128), p, mask, 0.5)
    assert np.array_equal(gm, gm2) and gm.any() and np.array_equal(jobs, jobs2)


def test_finalize_uncertainty_host(hb, orc):
    from hammerhead_b200 import _lib

    rng = np.random.default_rng(5)
    stats = np.zeros((6, 88))
    for j in range(6):
        s = np.zeros(44)
        s[0] = rng.uniform(5, 10)
        s[1] = s[2] = s[0] * rng.uniform(0.5, 0.9)
        s[3] = rng.uniform(0.01, 0.2)
        s[4:] = rng.uniform(-0.01, 0.05, 40) * s[3]
        stats[j, :44] = s
        stats[j, 44:] = s
    stats[5, 0] = -1  # C0 <= 0 -> NaN
    su = np.empty(6, np.float32)
    sv = np.empty(6, np.float32)
    _lib.check(_lib.lib().hh_finalize_uncertainty(_lib.dptr(stats), 6, _lib.fptr(su), _lib.fptr(sv)))
    for j in range(6):
        ref = orc.finalize_uncertainty(stats[j, :44], dtype=np.float32)
        assert (math.isnan(ref) and math.isnan(su[j])) or su[j] == np.float32(ref)


def test_synthetic_generator(hb):
    """The generator follows src/synthetic_data.jl: seeded, clamped >= 0,
    uniform flow moves the pattern by (u, v)."""
    syn = hb.synthetic
    A, B = syn.particle_pair((128, 128), syn.uniform_flow(2.0, -1.0), seed=5, noise=0.0)
    A2, _ = syn.particle_pair((128, 128), syn.uniform_flow(2.0, -1.0), seed=5, noise=0.0)
    assert np.array_equal(A, A2) and A.flags.f_contiguous and A.dtype == np.float32
    assert (A >= 0).all() and A.max() > 0.3
    # shifted content: B[r, c] == A[r + 1, c - 2] in the interior
    assert np.abs(B[20:100, 20:100] - A[21:101, 18:98]).max() < 1e-5
    flow = syn.lamb_oseen_flow((512.5, 512.5), 80.0, 8.0)
    r = np.linspace(1, 400, 4000)
    u, v = flow(512.5 + r, 512.5 + 0 * r)
    assert abs(np.hypot(u, v).max() - 8.0) < 1e-3


def test_batch_grid_host(hb):
    """hh_batch_grid: final grids and compact result offsets of a mixed batch,
    equal to pass_grid of each pair's final pass (host-only, no GPU)."""
    import ctypes

    from hammerhead_b200 import _lib

    s1 = hb.multipass_parameters([64, 32, 16], padding=True)
    s2 = hb.multipass_parameters([48, 24], padding=True)
    shapes = [(512, 512), (768, 1024), (200, 333)]
    scheds = [s1, s2]
    pairs = (_lib.hh_batch_pair * 3)()
    for p, sh in enumerate(shapes):
        pairs[p] = _lib.hh_batch_pair(1, 1, None, sh[0], sh[1], p % 2, 0)
    flat = s1 + s2
    descs = (_lib.hh_pass_desc * len(flat))(*[q.to_desc() for q in flat])
    so = np.array([0, len(s1), len(s1) + len(s2)], np.int32)
    ny, nx, off = np.zeros(3, np.int32), np.zeros(3, np.int32), np.zeros(4, np.int64)
    L = _lib.lib()
    _lib.check(L.hh_batch_grid(pairs, 3, descs, _lib.i32ptr(so), 2, _lib.i32ptr(ny), _lib.i32ptr(nx),
                               off.ctypes.data_as(_lib._I64)))
    tot = 0
    for p, sh in enumerate(shapes):
        x, y, _, _ = hb.pass_grid(sh, scheds[p % 2][-1])
        assert (ny[p], nx[p]) == (len(y), len(x))
        assert off[p] == tot
        tot += len(x) * len(y)
    assert off[3] == tot
    # argument errors carry messages
    bad = (_lib.hh_batch_pair * 1)(_lib.hh_batch_pair(1, 1, None, 64, 64, 5, 0))
    with pytest.raises(hb.ArgumentError, match="schedule index"):
        _lib.check(L.hh_batch_grid(bad, 1, descs, _lib.i32ptr(so), 2, None, None, None))
    with pytest.raises(hb.ArgumentError, match="must not be empty"):
        _lib.check(L.hh_batch_grid(bad, 0, descs, _lib.i32ptr(so), 2, None, None, None))
    small = (_lib.hh_batch_pair * 1)(_lib.hh_batch_pair(1, 1, None, 40, 40, 0, 0))
    with pytest.raises(hb.ArgumentError, match="exceeds image size"):
        _lib.check(L.hh_batch_grid(small, 1, descs, _lib.i32ptr(so), 2, None, None, None))
