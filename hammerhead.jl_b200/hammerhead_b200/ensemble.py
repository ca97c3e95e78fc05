"""run_piv_ensemble on the B200 (hh_run_ensemble).

Sum-of-correlation PIV (src/ensemble.jl:51-205): per pass every pair is
deformed by the shared predictor, each window's correlation planes are summed
over the pairs on the device and analysed once; uncertainty statistics pool
by summation. Pairs share one image size."""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch
from .params import PIVParameters, effort_schedule
from .batch import _pixel_format
from .pipeline import PIVResult, PIVWorkspace, _is_device_tensor, check_backend_params, pass_grid

_FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")


def run_piv_ensemble(pairs, params=None, *, effort=None, predictor_smoothing=True, mask=None, mask_threshold=0.5,
                     preprocess=None, workspace=None, scale=None, u16="normalised"):
    """Ensemble PIV over `pairs` (a list of (A, B) images: numpy (rows, cols)
    arrays, or column-major torch CUDA tensors); `params` is a
    PIVParameters or a pass schedule. Returns the PIVResult of the final
    pass (the ensemble-mean displacement field)."""
    if not pairs:
        raise ArgumentError("pairs must not be empty")
    if params is None:
        if effort is None:
            passes = [PIVParameters()]
        else:
            passes = effort_schedule(effort, image_size=tuple(pairs[0][0].shape))
    else:
        if effort is not None:
            raise ArgumentError("effort cannot be combined with explicit PIVParameters or pass schedules")
        passes = [params] if isinstance(params, PIVParameters) else list(params)
    if not passes:
        raise ArgumentError("at least one pass is required")
    check_backend_params(passes)
    if not (0 < mask_threshold <= 1):
        raise ArgumentError(f"mask_threshold must be in (0, 1], got {mask_threshold}")
    device = _is_device_tensor(pairs[0][0])
    keep = []
    arr = (_lib.hh_batch_pair * len(pairs))()
    shape = None
    for q, (A, B) in enumerate(pairs):
        if preprocess is not None:
            A, B = preprocess(A), preprocess(B)
        if tuple(A.shape) != tuple(B.shape):
            raise DimensionMismatch(f"images must have the same size, got {tuple(A.shape)} and {tuple(B.shape)}")
        if shape is None:
            shape = tuple(A.shape)
        elif tuple(A.shape) != shape:
            raise DimensionMismatch(f"all pairs must share the image size {shape}, got {tuple(A.shape)}")
        nr, nc = shape
        fmt = _pixel_format(A, B, u16)
        if device:
            for t in (A, B):
                if not _is_device_tensor(t) or t.stride(0) != 1 or t.stride(1) != nr:
                    raise ArgumentError("device images must be column-major CUDA tensors (stride (1, nrows))")
            ptrs = (A.data_ptr(), B.data_ptr())
            keep.append((A, B))
        else:
            if fmt == _lib.HH_PIX_F32:
                a, b = _lib.as_f32_colmajor(A), _lib.as_f32_colmajor(B)
            else:
                a, b = np.asfortranarray(A, np.uint16), np.asfortranarray(B, np.uint16)
            keep.append((a, b))
            ptrs = (a.ctypes.data, b.ctypes.data)
        arr[q] = _lib.hh_batch_pair(ptrs[0], ptrs[1], None, nr, nc, 0, fmt)
    if mask is not None and tuple(mask.shape) != shape:
        raise DimensionMismatch(f"mask must have the same size as the images, got {tuple(mask.shape)}")
    m = None if mask is None else np.asfortranarray(mask, dtype=np.uint8)
    x, y, _, _ = pass_grid(shape, passes[-1], None, mask_threshold)
    ny, nx = len(y), len(x)
    out = {k: np.empty((ny, nx), np.float32, order="F") for k in _FIELDS}
    outl = np.empty((ny, nx), np.uint8, order="F")
    gm = np.empty((ny, nx), np.uint8, order="F")
    xs, ys = np.empty(nx, np.float32), np.empty(ny, np.float32)
    res = _lib.hh_result(0, 0, _lib.fptr(xs), _lib.fptr(ys), *[_lib.fptr(out[k]) for k in _FIELDS], _lib.u8ptr(outl),
                         _lib.u8ptr(gm))
    descs = (_lib.hh_pass_desc * len(passes))(*[p.to_desc() for p in passes])
    ws = workspace if workspace is not None else PIVWorkspace()
    try:
        st = _lib.lib().hh_run_ensemble(ws.ctx, arr, len(pairs), descs, len(passes), _lib.u8ptr(m),
                                        float(mask_threshold), int(bool(predictor_smoothing)),
                                        _lib.HH_BATCH_DEVICE_INPUTS if device else 0, ctypes.byref(res))
        _lib.check(st, ws.ctx)
        ms = np.zeros(len(passes), np.float32)
        sw = np.zeros(len(passes), np.int32)
        _lib.lib().hh_last_pass_times(ws.ctx, len(passes), _lib.fptr(ms), _lib.i32ptr(sw))
    finally:
        if workspace is None:
            ws.close()
    return PIVResult(xs, ys, out["u"], out["v"], out["peak_ratio"], out["correlation_moment"], out["uncertainty_u"],
                     out["uncertainty_v"], outl.astype(bool), gm.astype(bool), passes[-1], None, scale, ms, sw)
