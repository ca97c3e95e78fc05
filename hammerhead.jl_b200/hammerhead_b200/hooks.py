"""Backend-hook level access to the device path.

These wrap the C-ABI entry points that replace the reference's private
backend hooks (docs/src/reference/backends.md:40-71): _deform_context /
apply_predictor (stage + deform), process_windows! (packed per-window
scalars), the device plane analysis (_ka_analyze!), and the vector-grid
validation kernels. They are what a host-side pass loop -- such as the
Julia extension's, or a parity test -- drives one step at a time.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError
from .params import PIVParameters


def packed_rows(n_peaks):
    k = max(n_peaks, 2)
    return 5 + 2 * (k - 1)


class DeviceSession:
    """A staged image pair on one library context (a PIVWorkspace)."""

    def __init__(self, workspace):
        self.ws = workspace
        self.shape = None

    def stage_pair(self, A, B):
        A = _lib.as_f32_colmajor(A)
        B = _lib.as_f32_colmajor(B)
        self.shape = A.shape
        _lib.check(_lib.lib().hh_stage_pair(self.ws.ctx, _lib.fptr(A), _lib.fptr(B), A.shape[0], A.shape[1]),
                   self.ws.ctx)

    def stage_mask(self, mask):
        """Image mask of the following process_windows / correlation_planes
        calls (None clears it): masked pixels leave the window means."""
        m = None if mask is None else np.asfortranarray(mask, np.uint8)
        if m is not None and m.shape != tuple(self.shape):
            raise ArgumentError(f"mask must have the staged image size {tuple(self.shape)}, got {m.shape}")
        _lib.check(_lib.lib().hh_stage_mask(self.ws.ctx, _lib.u8ptr(m)), self.ws.ctx)

    def apply_predictor(self, pu, pv, py, px, y, x, return_warped=False):
        """Deform the staged pair by predictor (pu, pv) on knots (py, px);
        returns node values at grid (y, x) and optionally the warped pair."""
        ny, nx = len(y), len(x)
        nu = np.empty((ny, nx), np.float32, order="F")
        nv = np.empty((ny, nx), np.float32, order="F")
        wA = wB = None
        if return_warped:
            wA = np.empty(self.shape, np.float32, order="F")
            wB = np.empty(self.shape, np.float32, order="F")
        y = np.ascontiguousarray(y, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        if pu is None:
            st = _lib.lib().hh_apply_predictor(self.ws.ctx, None, None, 0, 0, 0, 1, 0, 1, _lib.fptr(y), ny,
                                               _lib.fptr(x), nx, _lib.fptr(nu), _lib.fptr(nv), _lib.fptr(wA),
                                               _lib.fptr(wB))
        else:
            pu = _lib.as_f32_colmajor(pu)
            pv = _lib.as_f32_colmajor(pv)
            py = np.asarray(py, np.float32)
            px = np.asarray(px, np.float32)
            gny, gnx = pu.shape
            ysp = float(py[1] - py[0]) if gny > 1 else 1.0
            xsp = float(px[1] - px[0]) if gnx > 1 else 1.0
            st = _lib.lib().hh_apply_predictor(self.ws.ctx, _lib.fptr(pu), _lib.fptr(pv), gny, gnx, float(py[0]), ysp,
                                               float(px[0]), xsp, _lib.fptr(y), ny, _lib.fptr(x), nx, _lib.fptr(nu),
                                               _lib.fptr(nv), _lib.fptr(wA), _lib.fptr(wB))
        _lib.check(st, self.ws.ctx)
        return nu, nv, wA, wB

    def process_windows(self, params: PIVParameters, jobs, want_locs=False, want_uq=False):
        """Packed scalars [(5 + 2(K-1)) x njobs] for 1-based jobs (gi, gj, rs, cs)."""
        jobs = np.ascontiguousarray(jobs, np.int32)
        nj = jobs.shape[0]
        K = max(params.n_peaks, 2)
        out = np.empty((nj, packed_rows(params.n_peaks)), np.float32)
        locs = np.empty((nj, 2 * K), np.int32) if want_locs else None
        uq = np.empty((nj, 88), np.float64) if want_uq else None
        d = params.to_desc()
        st = _lib.lib().hh_process_windows(self.ws.ctx, ctypes.byref(d), _lib.i32ptr(jobs), nj, _lib.fptr(out),
                                           _lib.i32ptr(locs), _lib.dptr(uq))
        _lib.check(st, self.ws.ctx)
        return out, locs, uq

    def correlation_planes(self, params: PIVParameters, jobs):
        jobs = np.ascontiguousarray(jobs, np.int32)
        nj = jobs.shape[0]
        f = 2 if params.padding else 1
        nr, nc = f * params.search_area_size[0], f * params.search_area_size[1]
        planes = np.empty((nj, nr * nc), np.float32)
        d = params.to_desc()
        _lib.check(_lib.lib().hh_correlation_planes(self.ws.ctx, ctypes.byref(d), _lib.i32ptr(jobs), nj,
                                                    _lib.fptr(planes)), self.ws.ctx)
        return planes.reshape(nj, nc, nr).transpose(0, 2, 1)  # planes[j] indexed [row, col]


_FINDER = {"regionalmax": 0, "exclusion": 1}
_SUBPIXEL = {"gauss3": 0, "gauss9": 1, "gauss2d": 2, "none": 3}


def analyze_planes(ws, planes, n_peaks=3, peak_finder="regionalmax", subpixel_method="gauss3"):
    """Device plane analysis of a stack of planes [n, rows, cols]; returns
    (packed [n, 5+2(K-1)], locs [n, 2K] 1-based (row, col))."""
    planes = np.asarray(planes, np.float32)
    if planes.ndim == 2:
        planes = planes[None]
    n, nr, nc = planes.shape
    colmajor = np.ascontiguousarray(planes.transpose(0, 2, 1))  # column-major per plane
    K = max(n_peaks, 2)
    out = np.empty((n, packed_rows(n_peaks)), np.float32)
    locs = np.empty((n, 2 * K), np.int32)
    st = _lib.lib().hh_analyze_planes(ws.ctx, _lib.fptr(colmajor), n, nr, nc, n_peaks, _FINDER[peak_finder],
                                      _SUBPIXEL[subpixel_method], _lib.fptr(out), _lib.i32ptr(locs))
    _lib.check(st, ws.ctx)
    return out, locs


def validate(ws, params, u, v, peak_ratio=None, moment=None, mask=None, alt_u=None, alt_v=None, force_replace=False):
    """validate_and_replace! on the device; returns (u, v, outliers)."""
    u = np.array(u, np.float32, order="F")
    v = np.array(v, np.float32, order="F")
    ny, nx = u.shape
    pr = None if peak_ratio is None else np.asfortranarray(peak_ratio, np.float32)
    mo = None if moment is None else np.asfortranarray(moment, np.float32)
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    outl = np.zeros((ny, nx), np.uint8, order="F")
    nalt = 0
    au = av = None
    if alt_u is not None:
        au = np.asfortranarray(alt_u, np.float32)
        av = np.asfortranarray(alt_v, np.float32)
        nalt = au.shape[2]
    d = params.to_desc()
    st = _lib.lib().hh_validate(ws.ctx, ctypes.byref(d), ny, nx, _lib.fptr(u), _lib.fptr(v), _lib.fptr(pr),
                                _lib.fptr(mo), _lib.u8ptr(outl), _lib.u8ptr(m), _lib.fptr(au), _lib.fptr(av), nalt,
                                int(force_replace))
    _lib.check(st, ws.ctx)
    return u, v, outl.astype(bool)


def universal_outlier_detection(ws, u, v, threshold, neighborhood_size=1, epsilon=0.1, exclude=None):
    u = np.asfortranarray(u, np.float32)
    v = np.asfortranarray(v, np.float32)
    ny, nx = u.shape
    ex = None if exclude is None else np.asfortranarray(exclude, np.uint8)
    flags = np.zeros((ny, nx), np.uint8, order="F")
    st = _lib.lib().hh_uod(ws.ctx, _lib.fptr(u), _lib.fptr(v), ny, nx, float(threshold), int(neighborhood_size),
                           float(epsilon), _lib.u8ptr(ex), _lib.u8ptr(flags))
    _lib.check(st, ws.ctx)
    return flags.astype(bool)


def replace_vectors(ws, u, v, invalid):
    u = np.array(u, np.float32, order="F")
    v = np.array(v, np.float32, order="F")
    inv = np.asfortranarray(invalid, np.uint8)
    ny, nx = u.shape
    _lib.check(_lib.lib().hh_replace_vectors(ws.ctx, _lib.fptr(u), _lib.fptr(v), ny, nx, _lib.u8ptr(inv)), ws.ctx)
    return u, v


def smooth_field(ws, f):
    f = np.asfortranarray(f, np.float32)
    out = np.empty_like(f, order="F")
    ny, nx = f.shape
    _lib.check(_lib.lib().hh_smooth_field(ws.ctx, _lib.fptr(f), ny, nx, _lib.fptr(out)), ws.ctx)
    return out


def field_change(ws, u, v, pu, pv, mask=None):
    arrs = [np.asfortranarray(a, np.float32) for a in (u, v, pu, pv)]
    m = None if mask is None else np.asfortranarray(mask, np.uint8)
    out = ctypes.c_float()
    st = _lib.lib().hh_field_change(ws.ctx, *[_lib.fptr(a) for a in arrs], _lib.u8ptr(m), arrs[0].size,
                                    ctypes.byref(out))
    _lib.check(st, ws.ctx)
    return out.value
