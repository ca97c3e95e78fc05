"""ctypes access to the CPU oracle (liborc_piv.so).

TEST INFRASTRUCTURE ONLY: the checker for the device library and the CPU
baseline of bench.py. Product code never imports this module.

Pass descriptors are built from any object with PIVParameters attributes
(window_size, overlap, correlation_method, ...), so tests hand the same
PIVParameters to the device path and to the oracle.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "liborc_piv.so")


def build():
    """Compile the oracle (make) if the library is missing or stale."""
    src = os.path.join(HERE, "piv_oracle.cpp")
    if not os.path.exists(LIBPATH) or os.path.getmtime(src) > os.path.getmtime(LIBPATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIBPATH


class Validator(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("neighborhood", ctypes.c_int32), ("threshold", ctypes.c_double),
                ("vmin", ctypes.c_double), ("vmax", ctypes.c_double), ("epsilon", ctypes.c_double)]


class Pass(ctypes.Structure):
    _fields_ = [("window", ctypes.c_int32 * 2), ("search", ctypes.c_int32 * 2), ("overlap", ctypes.c_int32 * 2),
                ("method", ctypes.c_int32), ("padding", ctypes.c_int32), ("apod", ctypes.c_int32),
                ("subpixel", ctypes.c_int32), ("n_peaks", ctypes.c_int32), ("finder", ctypes.c_int32),
                ("uncertainty", ctypes.c_int32), ("uod_enable", ctypes.c_int32), ("uod_threshold", ctypes.c_double),
                ("uod_neighborhood", ctypes.c_int32), ("replace_outliers", ctypes.c_int32),
                ("min_peak_ratio", ctypes.c_double), ("max_iterations", ctypes.c_int32),
                ("keep_planes", ctypes.c_int32), ("convergence_tol", ctypes.c_double),
                ("n_validators", ctypes.c_int32), ("_pad", ctypes.c_int32), ("validators", Validator * 8)]


_METHODS = {"cross": 0, "phase": 1}
_APOD = {"none": 0, "gauss": 1}
_SUBPIXEL = {"gauss3": 0, "gauss9": 1, "gauss2d": 2, "none": 3}
_FINDERS = {"regionalmax": 0, "exclusion": 1}


def to_pass(p):
    d = Pass()
    d.window[0], d.window[1] = p.window_size
    d.search[0], d.search[1] = p.search_area_size
    d.overlap[0], d.overlap[1] = p.overlap
    d.method = _METHODS[p.correlation_method]
    d.padding = int(p.padding)
    d.apod = _APOD[p.apodization]
    d.subpixel = _SUBPIXEL[p.subpixel_method]
    d.n_peaks = p.n_peaks
    d.finder = _FINDERS[p.peak_finder]
    d.uncertainty = int(p.uncertainty)
    d.uod_enable = int(p.uod_enable)
    d.uod_threshold = p.uod_threshold
    d.uod_neighborhood = p.uod_neighborhood
    d.replace_outliers = int(p.replace_outliers)
    d.min_peak_ratio = p.min_peak_ratio
    d.max_iterations = p.max_iterations
    d.keep_planes = int(p.keep_correlation_planes)
    d.convergence_tol = p.convergence_tol
    d.n_validators = len(p.validation)
    for i, v in enumerate(p.validation):
        e = d.validators[i]
        e.kind = v.kind
        e.neighborhood = getattr(v, "neighborhood_size", 0)
        e.threshold = getattr(v, "threshold", 0.0)
        e.vmin = getattr(v, "min", 0.0)
        e.vmax = getattr(v, "max", 0.0)
        e.epsilon = getattr(v, "epsilon", 0.0)
    return d


_L = None


def lib():
    global _L
    if _L is None:
        build()
        L = ctypes.CDLL(LIBPATH)
        assert L.orc_sizeof_pass() == ctypes.sizeof(Pass), "oracle Pass layout mismatch"
        _L = L
    return _L


def _T(dtype):
    return (np.float32, ctypes.c_float, "f32") if np.dtype(dtype) == np.float32 else (np.float64, ctypes.c_double, "f64")


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ct))


def _u8(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _i32(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _fn(name, suf):
    return getattr(lib(), f"orc_{name}_{suf}")


def pass_grid(shape, params, mask=None, thr=0.5):
    d = to_pass(params)
    ny, nx = ctypes.c_int32(), ctypes.c_int32()
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    nj = lib().orc_pass_grid(ctypes.c_int64(shape[0]), ctypes.c_int64(shape[1]), ctypes.byref(d), _u8(m), ctypes.c_double(thr), ctypes.byref(ny),
                             ctypes.byref(nx), None, None)
    gm = np.empty((ny.value, nx.value), np.uint8, order="F")
    jobs = np.empty((max(nj, 1), 4), np.int32)
    lib().orc_pass_grid(ctypes.c_int64(shape[0]), ctypes.c_int64(shape[1]), ctypes.byref(d), _u8(m), ctypes.c_double(thr), ctypes.byref(ny), ctypes.byref(nx),
                        _u8(gm), _i32(jobs))
    jobs = jobs[:nj].copy()
    jobs[:, 0] += 1  # 1-based gi, gj like the reference
    jobs[:, 1] += 1
    return ny.value, nx.value, gm.astype(bool), jobs


def run_piv(A, B, passes, mask=None, mask_threshold=0.5, predictor_smoothing=True, nthreads=1, dtype=np.float32):
    """The reference run_piv pass loop on the CPU; returns a dict of grids
    (ny, nx) in Fortran order plus per-bucket timings and sweep counts."""
    T, ct, suf = _T(dtype)
    if not isinstance(passes, (list, tuple)):
        passes = [passes]
    A = np.asfortranarray(A, T)
    B = np.asfortranarray(B, T)
    nr, nc = A.shape
    ny, nx, _, _ = pass_grid((nr, nc), passes[-1], mask, mask_threshold)
    out = {k: np.empty((ny, nx), T, order="F") for k in
           ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")}
    out["x"] = np.empty(nx, T)
    out["y"] = np.empty(ny, T)
    outl = np.empty((ny, nx), np.uint8, order="F")
    gm = np.empty((ny, nx), np.uint8, order="F")

    class Res(ctypes.Structure):
        _fields_ = [("ny", ctypes.c_int32), ("nx", ctypes.c_int32)] + [
            (k, ctypes.POINTER(ct)) for k in ("x", "y", "u", "v", "peak_ratio", "moment", "unc_u", "unc_v")] + [
            ("outliers", ctypes.POINTER(ctypes.c_uint8)), ("mask", ctypes.POINTER(ctypes.c_uint8))]

    res = Res(0, 0, _p(out["x"], ct), _p(out["y"], ct), _p(out["u"], ct), _p(out["v"], ct),
              _p(out["peak_ratio"], ct), _p(out["correlation_moment"], ct), _p(out["uncertainty_u"], ct),
              _p(out["uncertainty_v"], ct), _u8(outl), _u8(gm))
    descs = (Pass * len(passes))(*[to_pass(p) for p in passes])
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    timing = np.zeros(6, np.float64)
    sweeps = np.zeros(len(passes), np.int32)
    st = _fn("run_piv", suf)(_p(A, ct), _p(B, ct), ctypes.c_int64(nr), ctypes.c_int64(nc), descs, len(passes), _u8(m), ctypes.c_double(mask_threshold),
                             int(bool(predictor_smoothing)), int(nthreads), ctypes.byref(res), _p(timing, ctypes.c_double),
                             _i32(sweeps))
    if st != 0:
        raise ValueError("oracle run_piv rejected the arguments")
    out["outliers"] = outl.astype(bool)
    out["mask"] = gm.astype(bool)
    out["timing"] = dict(zip(("deform", "correlate", "validate", "uq", "total", "final_pass"), timing))
    out["sweeps"] = sweeps
    return out


def find_peaks(R, k, peak_finder="regionalmax", exclusion_radius=2, dtype=np.float64):
    """find_peaks (src/correlators.jl:368-377): [(value, (row, col)), ...] 1-based."""
    T, ct, suf = _T(dtype)
    R = np.asfortranarray(R, T)
    vals = np.empty(k, T)
    locs = np.empty(2 * k, np.int32)
    f = _fn("find_peaks", suf)(_p(R, ct), R.shape[0], R.shape[1], k, _FINDERS[peak_finder], exclusion_radius,
                               _p(vals, ct), _i32(locs))
    return [(vals[m].item(), (int(locs[2 * m]), int(locs[2 * m + 1]))) for m in range(f)]


def subpixel(R, peakloc, method="gauss3", dtype=np.float64):
    T, ct, suf = _T(dtype)
    R = np.asfortranarray(R, T)
    out = np.empty(2, T)
    _fn(method, suf)(_p(R, ct), R.shape[0], R.shape[1], int(peakloc[0]), int(peakloc[1]), _p(out, ct))
    return float(out[0]), float(out[1])


def correlation_moment(R, peakloc, dtype=np.float64):
    T, ct, suf = _T(dtype)
    R = np.asfortranarray(R, T)
    f = _fn("moment", suf)
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.POINTER(ct), ctypes.c_int, ctypes.c_int, ct, ct]
    return f(_p(R, ct), R.shape[0], R.shape[1], peakloc[0], peakloc[1])


def peak_ratio(R, peakloc, exclusion_radius=2, peak_finder="regionalmax", dtype=np.float64):
    T, ct, suf = _T(dtype)
    R = np.asfortranarray(R, T)
    f = _fn("peak_ratio", suf)
    f.restype = ct
    return f(_p(R, ct), R.shape[0], R.shape[1], int(peakloc[0]), int(peakloc[1]), exclusion_radius,
             _FINDERS[peak_finder])


def analyze_plane(R, n_peaks=3, peak_finder="regionalmax", subpixel_method="gauss3", dtype=np.float32):
    T, ct, suf = _T(dtype)
    R = np.asfortranarray(R, T)
    K = max(n_peaks, 2)
    out = np.empty(5 + 2 * (K - 1), T)
    locs = np.empty(2 * K, np.int32)
    _fn("analyze_plane", suf)(_p(R, ct), R.shape[0], R.shape[1], n_peaks, _FINDERS[peak_finder],
                              _SUBPIXEL[subpixel_method], _p(out, ct), _i32(locs))
    return out, locs


def uod(u, v, threshold, neighborhood_size=1, epsilon=0.1, exclude=None, dtype=np.float64):
    T, ct, suf = _T(dtype)
    u = np.asfortranarray(u, T)
    v = np.asfortranarray(v, T)
    ex = None if exclude is None else np.asfortranarray(exclude, np.uint8)
    out = np.zeros(u.shape, np.uint8, order="F")
    _fn("uod", suf)(_p(u, ct), _p(v, ct), u.shape[0], u.shape[1], ctypes.c_double(threshold), neighborhood_size,
                    ctypes.c_double(epsilon), _u8(ex), _u8(out))
    return out.astype(bool)


def replace_vectors(u, v, invalid, dtype=np.float64):
    T, ct, suf = _T(dtype)
    u = np.array(u, T, order="F")
    v = np.array(v, T, order="F")
    inv = np.asfortranarray(invalid, np.uint8)
    _fn("replace_vectors", suf)(_p(u, ct), _p(v, ct), u.shape[0], u.shape[1], _u8(inv))
    return u, v


def smooth_field(f, dtype=np.float64):
    T, ct, suf = _T(dtype)
    f = np.asfortranarray(f, T)
    out = np.empty_like(f, order="F")
    _fn("smooth_field", suf)(_p(f, ct), f.shape[0], f.shape[1], _p(out, ct))
    return out


def validate(params, u, v, peak_ratio=None, moment=None, mask=None, alt_u=None, alt_v=None, force_replace=False,
             dtype=np.float32):
    """validate_and_replace! (src/pipeline.jl:617-645); returns (u, v, outliers)."""
    T, ct, suf = _T(dtype)
    u = np.array(u, T, order="F")
    v = np.array(v, T, order="F")
    ny, nx = u.shape
    pr = np.asfortranarray(np.full((ny, nx), 2.0) if peak_ratio is None else peak_ratio, T)
    mo = np.asfortranarray(np.zeros((ny, nx)) if moment is None else moment, T)
    outl = np.zeros((ny, nx), np.uint8, order="F")
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    nalt = 0
    au = av = None
    if alt_u is not None:
        au = np.asfortranarray(alt_u, T)
        av = np.asfortranarray(alt_v, T)
        nalt = au.shape[2]
    d = to_pass(params)
    _fn("validate", suf)(_p(u, ct), _p(v, ct), _p(pr, ct), _p(mo, ct), _u8(outl), _u8(m), ny, nx, ctypes.byref(d),
                         int(force_replace), _p(au, ct), _p(av, ct), nalt)
    return u, v, outl.astype(bool)


def fft2(z, inverse=False, dtype=np.float64):
    T, ct, suf = _T(dtype)
    z = np.asfortranarray(z, np.complex64 if T == np.float32 else np.complex128)
    buf = z.copy(order="F")
    _fn("fft2", suf)(buf.ctypes.data_as(ctypes.POINTER(ct)), z.shape[0], z.shape[1], int(inverse))
    return buf


def correlation_plane(subA, subB, params, dtype=np.float32):
    """correlation_plane! (src/correlators.jl:326-341) of the frame-A window
    subA and the frame-B search area subB (the window itself unless
    search_area_size is larger)."""
    T, ct, suf = _T(dtype)
    B = np.asfortranarray(subB, T)
    if subA.shape == subB.shape:
        A = np.asfortranarray(subA, T)
        pa = _p(A, ct)
    else:
        # the C restatement reads both frames with one leading dimension:
        # place the window at its offset inside a search-area-sized array
        sr, sc = B.shape
        wr, wc = subA.shape
        orr, oc = (sr - wr) // 2, (sc - wc) // 2
        A = np.zeros((sr, sc), T, order="F")
        A[orr:orr + wr, oc:oc + wc] = subA
        pa = ctypes.cast(A.ctypes.data + (orr + oc * sr) * A.itemsize, ctypes.POINTER(ct))
    f = 2 if params.padding else 1
    R = np.empty((f * params.search_area_size[0], f * params.search_area_size[1]), T, order="F")
    d = to_pass(params)
    _fn("correlation_plane", suf)(pa, _p(B, ct), ctypes.c_int64(B.shape[0]), ctypes.byref(d), _p(R, ct))
    return R


def apodization(w, apod="gauss", dtype=np.float64):
    T, ct, suf = _T(dtype)
    out = np.empty((w, w), T, order="F")
    _fn("apodization", suf)(w, w, _APOD[apod], _p(out, ct))
    return out


def overlap_gain(w, apod="gauss", dtype=np.float64):
    T, ct, suf = _T(dtype)
    out = np.empty((2 * w, 2 * w), T, order="F")
    _fn("overlap_gain", suf)(w, w, _APOD[apod], _p(out, ct))
    return out


def prefilter(img, dtype=np.float32):
    T, ct, suf = _T(dtype)
    img = np.asfortranarray(img, T)
    nr, nc = img.shape
    coef = np.empty((nr + 2, nc + 2), T, order="F")
    _fn("prefilter", suf)(_p(img, ct), ctypes.c_int64(nr), ctypes.c_int64(nc), _p(coef, ct))
    return coef


def deform(coefA, coefB, shape, pu, pv, py, px, nthreads=1, dtype=np.float32):
    T, ct, suf = _T(dtype)
    nr, nc = shape
    pu = np.asfortranarray(pu, T)
    pv = np.asfortranarray(pv, T)
    gny, gnx = pu.shape
    py = np.asarray(py, T)
    px = np.asarray(px, T)
    ysp = float(T(py[1] - py[0])) if gny > 1 else 1.0
    xsp = float(T(px[1] - px[0])) if gnx > 1 else 1.0
    wA = np.empty((nr, nc), T, order="F")
    wB = np.empty((nr, nc), T, order="F")
    f = _fn("deform", suf)
    f(_p(np.asfortranarray(coefA, T), ct), _p(np.asfortranarray(coefB, T), ct), ctypes.c_int64(nr), ctypes.c_int64(nc), _p(pu, ct), _p(pv, ct), gny,
      gnx, ctypes.c_double(float(py[0])), ctypes.c_double(ysp), ctypes.c_double(float(px[0])), ctypes.c_double(xsp),
      _p(wA, ct), _p(wB, ct), int(nthreads))
    return wA, wB


def uq_stats(subA, subB, apod="gauss", mask=None, dtype=np.float32):
    T, ct, suf = _T(dtype)
    A = np.asfortranarray(subA, T)
    B = np.asfortranarray(subB, T)
    s = np.zeros(88, np.float64)
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    _fn("uq_stats", suf)(_p(A, ct), _p(B, ct), ctypes.c_int64(A.shape[0]), A.shape[0], A.shape[1], _APOD[apod], _u8(m),
                         _p(s, ctypes.c_double))
    return s


def finalize_uncertainty(s, dtype=np.float64):
    T, ct, suf = _T(dtype)
    s = np.ascontiguousarray(s, np.float64)
    f = _fn("finalize_uq", suf)
    f.restype = ct
    return f(_p(s, ctypes.c_double))


def field_change(u, v, pu, pv, mask=None, dtype=np.float32):
    T, ct, suf = _T(dtype)
    arrs = [np.asfortranarray(a, T) for a in (u, v, pu, pv)]
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    f = _fn("field_change", suf)
    f.restype = ct
    return f(*[_p(a, ct) for a in arrs], _u8(m), ctypes.c_int64(arrs[0].size))


def uq_offsets():
    out = np.empty(80, np.int32)
    rs = np.empty(5, np.int32)
    lib().orc_uq_offsets(_i32(out), _i32(rs))
    return out.reshape(40, 2), rs


def ncc_windows(shape, window, overlap):
    """0-based origins (2 x n, column-major window order) of the loss windows."""
    nr, nc = shape
    step = window - overlap
    wy = (nr - window) // step + 1
    wx = (nc - window) // step + 1
    jr, jc = np.meshgrid(np.arange(wy), np.arange(wx), indexing="ij")
    w = np.stack([jr.ravel(order="F") * step, jc.ravel(order="F") * step], axis=1)
    return np.ascontiguousarray(w, np.int32)


def ncc_loss_grad(coefA, coefB, shape, P, grid, window=16, overlap=8, windows=None, grad=True, nthreads=8,
                  dtype=np.float64):
    """Correlation loss L = -sum NCC0 over the windows (all, or the given
    0-based origins) of the pair deformed by P (gny, gnx, 2) on nodes
    grid = (y0, ysp, x0, xsp); returns (L, dL/dP shaped like P or None)."""
    T, ct, suf = _T(dtype)
    nr, nc = shape
    P = np.asarray(P)
    gny, gnx = P.shape[0], P.shape[1]
    flat = np.concatenate([P[..., 0].ravel(order="F"), P[..., 1].ravel(order="F")]).astype(T)
    wins = ncc_windows(shape, window, overlap) if windows is None else np.ascontiguousarray(windows, np.int32)
    g = np.zeros(2 * gny * gnx, T) if grad else None
    f = _fn("ncc_loss_grad", suf)
    f.restype = ctypes.c_double
    y0, ysp, x0, xsp = grid
    L = f(_p(np.asfortranarray(coefA, T), ct), _p(np.asfortranarray(coefB, T), ct), ctypes.c_int64(nr),
          ctypes.c_int64(nc), _p(flat, ct), gny, gnx, ctypes.c_double(y0), ctypes.c_double(ysp), ctypes.c_double(x0),
          ctypes.c_double(xsp), window, wins.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
          ctypes.c_int64(len(wins)), _p(g, ct) if grad else None, nthreads)
    if not grad:
        return L, None
    G = gny * gnx
    out = np.empty((gny, gnx, 2), T)
    out[..., 0] = np.reshape(g[:G], (gny, gnx), order="F")
    out[..., 1] = np.reshape(g[G:], (gny, gnx), order="F")
    return L, out


def run_ensemble(pairs, passes, mask=None, mask_threshold=0.5, predictor_smoothing=True, nthreads=1,
                 dtype=np.float32):
    """run_piv_ensemble on the CPU: pairs is a list of (A, B) of one size;
    returns the final pass as a dict of grids like run_piv."""
    T, ct, suf = _T(dtype)
    if not isinstance(passes, (list, tuple)):
        passes = [passes]
    imgs = [(np.asfortranarray(A, T), np.asfortranarray(B, T)) for A, B in pairs]
    nr, nc = imgs[0][0].shape
    ny, nx, _, _ = pass_grid((nr, nc), passes[-1], mask, mask_threshold)
    out = {k: np.empty((ny, nx), T, order="F") for k in
           ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")}
    out["x"] = np.empty(nx, T)
    out["y"] = np.empty(ny, T)
    outl = np.empty((ny, nx), np.uint8, order="F")
    gm = np.empty((ny, nx), np.uint8, order="F")

    class Res(ctypes.Structure):
        _fields_ = [("ny", ctypes.c_int32), ("nx", ctypes.c_int32)] + [
            (k, ctypes.POINTER(ct)) for k in ("x", "y", "u", "v", "peak_ratio", "moment", "unc_u", "unc_v")] + [
            ("outliers", ctypes.POINTER(ctypes.c_uint8)), ("mask", ctypes.POINTER(ctypes.c_uint8))]

    res = Res(0, 0, _p(out["x"], ct), _p(out["y"], ct), _p(out["u"], ct), _p(out["v"], ct),
              _p(out["peak_ratio"], ct), _p(out["correlation_moment"], ct), _p(out["uncertainty_u"], ct),
              _p(out["uncertainty_v"], ct), _u8(outl), _u8(gm))
    PT = ctypes.POINTER(ct)
    As = (PT * len(imgs))(*[_p(a, ct) for a, _ in imgs])
    Bs = (PT * len(imgs))(*[_p(b, ct) for _, b in imgs])
    descs = (Pass * len(passes))(*[to_pass(p) for p in passes])
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    st = _fn("run_ensemble", suf)(As, Bs, len(imgs), ctypes.c_int64(nr), ctypes.c_int64(nc), descs, len(passes),
                                  _u8(m), ctypes.c_double(mask_threshold), int(bool(predictor_smoothing)),
                                  int(nthreads), ctypes.byref(res))
    if st != 0:
        raise ValueError("oracle run_ensemble rejected the arguments")
    out["outliers"] = outl.astype(bool)
    out["mask"] = gm.astype(bool)
    return out


class Params:
    """A pass configuration with the fields and defaults of the reference's
    PIVParameters (src/types.jl:212-291), for callers of the oracle that do
    not load the device library (the CPU legs of the benchmark). No
    validation beyond what the C restatement does."""

    def __init__(self, window_size=(32, 32), search_area_size=None, overlap=(16, 16), correlation_method="cross",
                 padding=False, apodization="none", subpixel_method="gauss3", n_peaks=3, peak_finder="regionalmax",
                 uncertainty=False, uod_enable=True, uod_threshold=2.0, uod_neighborhood=2, min_peak_ratio=1.0,
                 validation=(), replace_outliers=True, max_iterations=1, convergence_tol=0.05,
                 keep_correlation_planes=False):
        pair = lambda v: (int(v), int(v)) if np.isscalar(v) else (int(v[0]), int(v[1]))  # noqa: E731
        self.window_size = pair(window_size)
        self.search_area_size = self.window_size if search_area_size is None else pair(search_area_size)
        self.overlap = pair(overlap)
        self.correlation_method = correlation_method
        self.padding = bool(padding)
        self.apodization = apodization
        self.subpixel_method = subpixel_method
        self.n_peaks = int(n_peaks)
        self.peak_finder = peak_finder
        self.uncertainty = bool(uncertainty)
        self.uod_enable = bool(uod_enable)
        self.uod_threshold = float(uod_threshold)
        self.uod_neighborhood = int(uod_neighborhood)
        self.min_peak_ratio = float(min_peak_ratio)
        self.validation = tuple(validation)
        self.replace_outliers = bool(replace_outliers)
        self.max_iterations = int(max_iterations)
        self.convergence_tol = float(convergence_tol)
        self.keep_correlation_planes = bool(keep_correlation_planes)


def multipass(window_sizes, overlap_fraction=0.5, final=None, **kw):
    """multipass_parameters (src/pipeline.jl:509-524): one pass per window
    size, overlap floor(w * fraction), `final` merged into the last pass."""
    out = []
    for i, w in enumerate(window_sizes):
        extra = dict(kw)
        if i == len(window_sizes) - 1:
            extra.update(final or {})
        w = (w, w) if np.isscalar(w) else tuple(w)
        out.append(Params(window_size=w, overlap=(int(w[0] * overlap_fraction), int(w[1] * overlap_fraction)),
                          **extra))
    return out


def final_vectors(shape, passes, mask=None, thr=0.5):
    """Unmasked cells of the final pass grid (pass_grid, src/pipeline.jl:529-555)."""
    ny, nx, gm, _ = pass_grid(shape, passes[-1], mask, thr)
    return int(gm.size - gm.sum())
