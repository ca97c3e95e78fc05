"""run_piv on the B200 backend: PIVResult, PIVWorkspace, run_piv.

Mirrors the reference driver (src/pipeline.jl:361-449) and result type
(src/types.jl:359-373). The whole pass schedule -- deformation, correlation,
validation, substitution, replacement, convergence checks and uncertainty --
runs inside the library (hh_run_piv); this module only validates arguments,
converts arrays to the column-major float32 layout of the C ABI, and wraps
the returned grids. Grids are numpy arrays of shape (ny, nx) in Fortran
order, indexed like Julia: ``result.u[gi, gj]``.
"""
import ctypes
from dataclasses import dataclass, field, replace
from typing import Any, Optional

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch
from .params import PIVParameters, effort_schedule

BACKENDS = ("b200",)


@dataclass
class PhysicalScale:
    """Metadata attached to a result (src/types.jl:24-42); arrays stay in pixels."""
    pixel_size: float = 1.0
    dt: float = 1.0
    length_unit: str = "px"
    time_unit: str = "frame"

    def __post_init__(self):
        if not (np.isfinite(self.pixel_size) and self.pixel_size > 0):
            raise ArgumentError(f"pixel_size must be positive and finite, got {self.pixel_size}")
        if not (np.isfinite(self.dt) and self.dt > 0):
            raise ArgumentError(f"dt must be positive and finite, got {self.dt}")


@dataclass
class PIVResult:
    """Result of run_piv: the final pass's vector grid (PIVResult{Float32})."""
    x: np.ndarray
    y: np.ndarray
    u: np.ndarray
    v: np.ndarray
    peak_ratio: np.ndarray
    correlation_moment: np.ndarray
    uncertainty_u: np.ndarray
    uncertainty_v: np.ndarray
    outliers: np.ndarray
    mask: np.ndarray
    parameters: PIVParameters
    correlation_planes: Optional[Any] = None
    scale: Optional[PhysicalScale] = None
    pass_times_ms: Optional[np.ndarray] = field(default=None, repr=False)
    sweeps: Optional[np.ndarray] = field(default=None, repr=False)

    def __repr__(self):
        ny, nx = self.u.shape
        s = f"PIVResult{{Float32}}({nx}×{ny} grid, {int(self.outliers.sum())} outliers"
        return s + (f", {int(self.mask.sum())} masked)" if self.mask.any() else ")")


class PIVWorkspace:
    """Reusable device scratch for run_piv (src/pipeline.jl:21-44): one
    library context (stream, growable device arena, cached window tables).
    Not thread-safe; do not share across concurrent run_piv calls."""

    def __init__(self, backend="b200", device=0):
        backend = backend[1:] if backend.startswith(":") else backend
        _resolve_backend(backend)
        self.backend = backend
        self.device = int(device)
        h = ctypes.c_void_p()
        st = _lib.lib().hh_ctx_create(self.device, ctypes.byref(h))
        _lib.check(st)
        self._ctx = h

    @property
    def ctx(self):
        if self._ctx is None:
            raise _lib.HammerheadError(_lib.HH_ERR_STATE, "workspace has been released")
        return self._ctx

    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return _lib.lib().hh_ctx_stream(self.ctx)

    def close(self):
        self.__dict__.pop("_stream_sessions", None)  # device frames and runners of run_piv_batch_stream
        if getattr(self, "_ctx", None) is not None:
            _lib.lib().hh_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def piv_workspace(*, backend="b200", device=0):
    """Construct a PIVWorkspace (src/pipeline.jl:33-44)."""
    return PIVWorkspace(backend=backend, device=device)


def _resolve_backend(backend):
    if backend not in BACKENDS:
        raise ArgumentError(f"unsupported Hammerhead backend :{backend}; this package provides backend = :b200")
    return backend


def check_backend_params(passes):
    """_check_backend_params for :b200 -- reject options the device path does
    not implement before any work (src/ka_backend.jl:13-29)."""
    descs = (_lib.hh_pass_desc * len(passes))(*[p.to_desc() for p in passes])
    _lib.check(_lib.lib().hh_check_backend_params(descs, len(passes)))


def pass_grid(imgsize, params, mask=None, mask_threshold=0.5):
    """pass_grid (src/pipeline.jl:529-555): x, y, grid mask and 1-based jobs."""
    nr, nc = int(imgsize[0]), int(imgsize[1])
    d = params.to_desc()
    ny, nx, nj = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
    m = None if mask is None else np.asfortranarray(mask, dtype=np.uint8)
    L = _lib.lib()
    _lib.check(L.hh_pass_grid(nr, nc, ctypes.byref(d), _lib.u8ptr(m), float(mask_threshold), ctypes.byref(ny),
                              ctypes.byref(nx), None, None, None, None, ctypes.byref(nj)))
    x = np.empty(nx.value, np.float32)
    y = np.empty(ny.value, np.float32)
    gm = np.empty((ny.value, nx.value), np.uint8, order="F")
    jobs = np.empty((max(nj.value, 1), 4), np.int32)
    _lib.check(L.hh_pass_grid(nr, nc, ctypes.byref(d), _lib.u8ptr(m), float(mask_threshold), ctypes.byref(ny),
                              ctypes.byref(nx), _lib.fptr(x), _lib.fptr(y), _lib.u8ptr(gm), _lib.i32ptr(jobs),
                              ctypes.byref(nj)))
    return x, y, gm.astype(bool), jobs[: nj.value]


def _is_device_tensor(a):
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def run_piv(imgA, imgB, passes=None, *, effort=None, backend="b200", uncertainty_backend="same", threaded=None,
            predictor_smoothing=True, mask=None, mask_threshold=0.5, workspace=None, scale=None):
    """Run a (multi-pass) planar WIDIM analysis of one image pair on the B200.

    Same semantics as the reference run_piv (src/pipeline.jl:361-449):
    `passes` is a PIVParameters or a list of them (or None with `effort`);
    returns the PIVResult of the final pass. Images are (rows, cols) arrays
    (numpy, or torch CUDA tensors already resident on the device in
    column-major storage); they are analysed in float32.
    """
    backend = backend[1:] if isinstance(backend, str) and backend.startswith(":") else backend
    if passes is None:
        if effort is None:
            passes = [PIVParameters()]
        else:
            shape = tuple(imgA.shape)
            passes = effort_schedule(effort, image_size=shape)
    else:
        if effort is not None:
            raise ArgumentError("effort cannot be combined with explicit PIVParameters or pass schedules")
        if isinstance(passes, PIVParameters):
            passes = [passes]
        passes = list(passes)
    _resolve_backend(backend)
    if uncertainty_backend not in ("same", ":same"):
        raise ArgumentError(f"uncertainty_backend must be :same on backend :b200, got :{uncertainty_backend}")
    if workspace is not None and workspace.backend != backend:
        raise ArgumentError(f"workspace backend :{workspace.backend} does not match run backend :{backend}; "
                            "build the workspace with the same `backend`")
    if not passes:
        raise ArgumentError("at least one pass is required")
    check_backend_params(passes)
    if tuple(imgA.shape) != tuple(imgB.shape):
        raise DimensionMismatch(f"images must have the same size, got {tuple(imgA.shape)} and {tuple(imgB.shape)}")
    if len(imgA.shape) != 2:
        raise DimensionMismatch("images must be matrices")
    if mask is not None and tuple(mask.shape) != tuple(imgA.shape):
        raise DimensionMismatch(f"mask must have the same size as the images, got {tuple(mask.shape)}")
    if not (0 < mask_threshold <= 1):
        raise ArgumentError(f"mask_threshold must be in (0, 1], got {mask_threshold}")

    ws = workspace if workspace is not None else PIVWorkspace(backend=backend)
    try:
        nr, nc = int(imgA.shape[0]), int(imgA.shape[1])
        final = passes[-1]
        x, y, _, _ = pass_grid((nr, nc), final, None, mask_threshold)
        ny, nx = len(y), len(x)
        out = {k: np.empty((ny, nx), np.float32, order="F") for k in
               ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")}
        outl = np.empty((ny, nx), np.uint8, order="F")
        gm = np.empty((ny, nx), np.uint8, order="F")
        xs = np.empty(nx, np.float32)
        ys = np.empty(ny, np.float32)
        res = _lib.hh_result(0, 0, _lib.fptr(xs), _lib.fptr(ys), _lib.fptr(out["u"]), _lib.fptr(out["v"]),
                             _lib.fptr(out["peak_ratio"]), _lib.fptr(out["correlation_moment"]),
                             _lib.fptr(out["uncertainty_u"]), _lib.fptr(out["uncertainty_v"]), _lib.u8ptr(outl),
                             _lib.u8ptr(gm))
        descs = (_lib.hh_pass_desc * len(passes))(*[p.to_desc() for p in passes])
        L = _lib.lib()
        if _is_device_tensor(imgA):
            for t in (imgA, imgB) + ((mask,) if mask is not None else ()):
                if t.stride(0) != 1 or t.stride(1) != nr:
                    raise ArgumentError("device images must be column-major (stride (1, nrows)), "
                                        "e.g. torch.empty((ncols, nrows)).T")
            st = L.hh_run_piv_device(ws.ctx, ctypes.c_void_p(imgA.data_ptr()), ctypes.c_void_p(imgB.data_ptr()), nr,
                                     nc, descs, len(passes),
                                     ctypes.c_void_p(mask.data_ptr()) if mask is not None else None,
                                     float(mask_threshold), int(bool(predictor_smoothing)), ctypes.byref(res))
        else:
            A = _lib.as_f32_colmajor(imgA)
            B = _lib.as_f32_colmajor(imgB)
            m = None if mask is None else np.asfortranarray(mask, dtype=np.uint8)
            st = L.hh_run_piv(ws.ctx, _lib.fptr(A), _lib.fptr(B), nr, nc, descs, len(passes), _lib.u8ptr(m),
                              float(mask_threshold), int(bool(predictor_smoothing)), ctypes.byref(res))
        _lib.check(st, ws.ctx)
        ms = np.zeros(len(passes), np.float32)
        sw = np.zeros(len(passes), np.int32)
        L.hh_last_pass_times(ws.ctx, len(passes), _lib.fptr(ms), _lib.i32ptr(sw))
        result = PIVResult(xs, ys, out["u"], out["v"], out["peak_ratio"], out["correlation_moment"],
                           out["uncertainty_u"], out["uncertainty_v"], outl.astype(bool), gm.astype(bool), final,
                           None, scale, ms, sw)
        return result
    finally:
        if workspace is None:
            ws.close()


def with_scale(result, scale):
    """Attach a PhysicalScale (metadata only)."""
    return replace(result, scale=scale)
