"""run_piv_ensemble on the B200 (hh_run_ensemble).

Sum-of-correlation PIV (src/ensemble.jl:51-205): per pass every pair is
deformed by the shared predictor, each window's correlation planes are summed
over the pairs on the device and analysed once; uncertainty statistics pool
by summation. Pairs share one image size.

Multi-GPU: the pairs of one ensemble can be split over processes (one per
GPU). Each process sums its own pairs on its device, and once per pass the
partial plane sums and uncertainty sums are all-reduced over a
torch.distributed process group (NCCL between GPUs) before the analysis, so
every process returns the field of the whole ensemble."""
import ctypes
import zlib

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch
from .params import PIVParameters, effort_schedule
from .batch import _pixel_format
from .pipeline import PIVResult, PIVWorkspace, _is_device_tensor, check_backend_params, pass_grid

_FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")


def shard_pairs(pairs, rank=None, world_size=None):
    """This process's contiguous share of `pairs` (rank r of w takes
    pairs[r*n//w:(r+1)*n//w]), so that the ranks' partial sums follow the
    pair order. rank / world_size default to the torch.distributed ones."""
    if rank is None or world_size is None:
        import torch.distributed as dist

        rank = dist.get_rank() if rank is None else rank
        world_size = dist.get_world_size() if world_size is None else world_size
    if not (0 <= rank < world_size):
        raise ArgumentError(f"rank must be in [0, {world_size}), got {rank}")
    n = len(pairs)
    return list(pairs[rank * n // world_size:(rank + 1) * n // world_size])


class _DeviceArray:
    """A borrowed 1-d device array (CUDA array interface, no stream key) for
    torch.as_tensor; the library keeps ownership."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None}


def collective_reducer(group=None):
    """Reducer over a torch.distributed process group: planes and stats are
    replaced by their sums over the group (dist.all_reduce, SUM)."""
    import torch.distributed as dist

    def reduce(k, planes, stats):
        dist.all_reduce(planes, op=dist.ReduceOp.SUM, group=group)
        if stats is not None:
            dist.all_reduce(stats, op=dist.ReduceOp.SUM, group=group)

    return reduce


def _agree(group, key, err):
    """Every rank learns whether all ranks prepared the same ensemble (same
    image size, passes, mask and options, at least one local pair); all raise
    together, so that no rank is left waiting in a collective."""
    import torch.distributed as dist

    got = [None] * dist.get_world_size(group)
    dist.all_gather_object(got, (key, None if err is None else f"{type(err).__name__}: {err}"), group=group)
    for r, (k, e) in enumerate(got):
        if e is not None:
            if err is not None:
                raise err
            raise ArgumentError(f"rank {r} rejected its share of the ensemble ({e})")
    for r, (k, e) in enumerate(got):
        if k != got[0][0]:
            what = [n for n, a, b in zip(("image size", "passes", "mask", "mask_threshold", "predictor_smoothing",
                                          "u16"), k, got[0][0]) if a != b]
            raise ArgumentError(f"rank {r} differs from rank 0 in {', '.join(what)}")


def _make_trampoline(fn, device, errors):
    import torch

    def cb(user, k, planes, nplanes, stats, nstats, stream):
        try:
            dev = torch.device("cuda", device)
            with torch.cuda.device(dev), torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev)):
                tp = torch.as_tensor(_DeviceArray(planes, nplanes, "<f4"), device=dev)
                ts = torch.as_tensor(_DeviceArray(stats, nstats, "<f8"), device=dev) if nstats > 0 else None
                fn(int(k), tp, ts)
            return 0
        except BaseException as e:  # noqa: BLE001 - reported through the library status
            errors.append(e)
            return 1

    return _lib.ENSEMBLE_REDUCER(cb)


def run_piv_ensemble(pairs, params=None, *, effort=None, predictor_smoothing=True, mask=None, mask_threshold=0.5,
                     preprocess=None, workspace=None, scale=None, u16="normalised", process_group=None,
                     reducer=None):
    """Ensemble PIV over `pairs` (a list of (A, B) images: numpy (rows, cols)
    arrays, or column-major torch CUDA tensors); `params` is a
    PIVParameters or a pass schedule. Returns the PIVResult of the final
    pass (the ensemble-mean displacement field).

    process_group: a torch.distributed process group, or True for the
    default one. `pairs` is then this process's share of the ensemble (see
    shard_pairs); the sums are all-reduced over the group once per pass and
    every process returns the field of all pairs. All processes must pass the
    same image size, passes, mask and options.
    reducer: instead of a process group, a callable (pass_index, planes,
    stats) that replaces the CUDA tensors planes (float32) and stats
    (float64, or None) in place by their sums over the processes; it runs
    with the library stream as the current torch stream."""
    if process_group is not None and reducer is not None:
        raise ArgumentError("process_group and reducer cannot be combined")
    if process_group is not None:
        group = None if process_group is True else process_group
        try:
            prep = _prepare(pairs, params, effort, predictor_smoothing, mask, mask_threshold, preprocess, u16)
            err = None
        except Exception as e:  # noqa: BLE001 - every rank raises together in _agree
            prep, err = None, e
        _agree(group, None if prep is None else prep["key"], err)
        return _run(prep, workspace, scale, collective_reducer(group))
    prep = _prepare(pairs, params, effort, predictor_smoothing, mask, mask_threshold, preprocess, u16)
    return _run(prep, workspace, scale, reducer)


def _prepare(pairs, params, effort, predictor_smoothing, mask, mask_threshold, preprocess, u16):
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
    descs = (_lib.hh_pass_desc * len(passes))(*[p.to_desc() for p in passes])
    key = (shape, zlib.crc32(bytes(descs)), None if m is None else zlib.crc32(m.tobytes(order="F")),
           float(mask_threshold), bool(predictor_smoothing), u16)
    return dict(pairs=arr, npairs=len(pairs), keep=keep, shape=shape, passes=passes, descs=descs, mask=m,
                mask_threshold=mask_threshold, smoothing=predictor_smoothing, device=device, key=key)


def _run(prep, workspace, scale, reducer):
    shape, passes, descs, m = prep["shape"], prep["passes"], prep["descs"], prep["mask"]
    mask_threshold, device = prep["mask_threshold"], prep["device"]
    x, y, _, _ = pass_grid(shape, passes[-1], None, mask_threshold)
    ny, nx = len(y), len(x)
    out = {k: np.empty((ny, nx), np.float32, order="F") for k in _FIELDS}
    outl = np.empty((ny, nx), np.uint8, order="F")
    gm = np.empty((ny, nx), np.uint8, order="F")
    xs, ys = np.empty(nx, np.float32), np.empty(ny, np.float32)
    res = _lib.hh_result(0, 0, _lib.fptr(xs), _lib.fptr(ys), *[_lib.fptr(out[k]) for k in _FIELDS], _lib.u8ptr(outl),
                         _lib.u8ptr(gm))
    ws = workspace if workspace is not None else PIVWorkspace()
    errors = []
    cb = None if reducer is None else _make_trampoline(reducer, ws.device, errors)
    try:
        if cb is not None:
            _lib.check(_lib.lib().hh_set_ensemble_reducer(ws.ctx, ctypes.cast(cb, ctypes.c_void_p), None), ws.ctx)
        try:
            st = _lib.lib().hh_run_ensemble(ws.ctx, prep["pairs"], prep["npairs"], descs, len(passes), _lib.u8ptr(m),
                                            float(mask_threshold), int(bool(prep["smoothing"])),
                                            _lib.HH_BATCH_DEVICE_INPUTS if device else 0, ctypes.byref(res))
        finally:
            if cb is not None:
                _lib.lib().hh_set_ensemble_reducer(ws.ctx, None, None)
        if errors:
            raise errors[0]
        _lib.check(st, ws.ctx)
        ms = np.zeros(len(passes), np.float32)
        sw = np.zeros(len(passes), np.int32)
        _lib.lib().hh_last_pass_times(ws.ctx, len(passes), _lib.fptr(ms), _lib.i32ptr(sw))
    finally:
        if workspace is None:
            ws.close()
    return PIVResult(xs, ys, out["u"], out["v"], out["peak_ratio"], out["correlation_moment"], out["uncertainty_u"],
                     out["uncertainty_v"], outl.astype(bool), gm.astype(bool), passes[-1], None, scale, ms, sw)
