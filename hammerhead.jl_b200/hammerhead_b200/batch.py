"""Batched planar WIDIM: many image pairs of uneven size and schedule at once.

The reference analyses a stream of pairs with run_piv_sequence
(src/io.jl:229-361), one run_piv per pair, results identical to separate
calls. Here the whole batch runs as one device schedule (hh_run_batched):
every pass slot is one launch per kernel for all pairs, convergence is
decided on the device, and the launch sequence of a batch shape is captured
in a CUDA graph once and replayed. Results equal run_piv on each pair.
"""
import ctypes
import zlib

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch
from .params import PIVParameters
from .pipeline import PIVResult, PIVWorkspace, _is_device_tensor, check_backend_params, pass_grid

_FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")


def _schedules(passes, npairs):
    """One pass list per pair, deduplicated: (unique schedules, index per pair)."""
    if isinstance(passes, PIVParameters):
        per_pair = [[passes]] * npairs
    elif passes and all(isinstance(p, PIVParameters) for p in passes):
        per_pair = [list(passes)] * npairs
    else:
        per_pair = [[s] if isinstance(s, PIVParameters) else list(s) for s in passes]
        if len(per_pair) != npairs:
            raise DimensionMismatch(f"got {len(per_pair)} pass schedules for {npairs} pairs")
    uniq, index = [], []
    for s in per_pair:
        if not s:
            raise ArgumentError("at least one pass is required")
        for k, u in enumerate(uniq):
            if len(u) == len(s) and all(a is b or a == b for a, b in zip(u, s)):
                index.append(k)
                break
        else:
            uniq.append(s)
            index.append(len(uniq) - 1)
    return uniq, index


def _is_u16(a):
    dt = getattr(a, "dtype", None)
    return dt is not None and str(dt) in ("uint16", "torch.uint16")


def _pixel_format(A, B, u16):
    """HH_PIX_* of a pair: UInt16 frames (12/16-bit camera counts) are sent
    as they are and converted on the device -- "normalised" to value/65535
    like load_image's Float32 of a 16-bit image, or "raw" counts."""
    if _is_u16(A) != _is_u16(B):
        raise ArgumentError("both frames of a pair must have the same pixel type")
    if not _is_u16(A):
        return _lib.HH_PIX_F32
    if u16 not in ("normalised", "raw"):
        raise ArgumentError(f"u16 must be 'normalised' or 'raw', got {u16!r}")
    return _lib.HH_PIX_U16 if u16 == "normalised" else _lib.HH_PIX_U16_RAW


class BatchRunner:
    """A prepared batch: pair descriptors, pass tables and (page-locked)
    result buffers built once; `run()` is one library call. Keep the images
    (and masks) alive and unchanged in shape while the runner is used;
    their contents may change between runs."""

    def __init__(self, pairs, passes, *, masks=None, predictor_smoothing=True, mask_threshold=0.5, workspace=None,
                 graph=True, pinned=True, u16="normalised"):
        if not pairs:
            raise ArgumentError("pairs must not be empty")
        if not (0 < mask_threshold <= 1):
            raise ArgumentError(f"mask_threshold must be in (0, 1], got {mask_threshold}")
        n = len(pairs)
        masks = [None] * n if masks is None else list(masks)
        if len(masks) != n:
            raise DimensionMismatch(f"got {len(masks)} masks for {n} pairs")
        self.schedules, self.index = _schedules(passes, n)
        for s in self.schedules:
            check_backend_params(s)
        self.device = _is_device_tensor(pairs[0][0])
        self._keep = []
        self.pairs = (_lib.hh_batch_pair * n)()
        for p, ((A, B), M) in enumerate(zip(pairs, masks)):
            if tuple(A.shape) != tuple(B.shape):
                raise DimensionMismatch(f"images must have the same size, got {tuple(A.shape)} and {tuple(B.shape)}")
            if len(A.shape) != 2:
                raise DimensionMismatch("images must be matrices")
            if M is not None and tuple(M.shape) != tuple(A.shape):
                raise DimensionMismatch(f"mask must have the same size as the images, got {tuple(M.shape)}")
            nr, nc = int(A.shape[0]), int(A.shape[1])
            if self.device != _is_device_tensor(A) or self.device != _is_device_tensor(B):
                raise ArgumentError("all images of a batch must be host arrays or all device tensors")
            fmt = _pixel_format(A, B, u16)
            if self.device:
                for t in (A, B) + ((M,) if M is not None else ()):
                    if t.stride(0) != 1 or t.stride(1) != nr:
                        raise ArgumentError("device images must be column-major (stride (1, nrows))")
                ptrs = [t.data_ptr() if t is not None else None for t in (A, B, M)]
                self._keep.append((A, B, M))
            else:
                if fmt == _lib.HH_PIX_F32:
                    a = _lib.as_f32_colmajor(A)
                    b = _lib.as_f32_colmajor(B)
                else:
                    a = np.asfortranarray(A, np.uint16)
                    b = np.asfortranarray(B, np.uint16)
                m = None if M is None else np.asfortranarray(M, dtype=np.uint8)
                self._keep.append((a, b, m))
                ptrs = [x.ctypes.data if x is not None else None for x in (a, b, m)]
            self.pairs[p] = _lib.hh_batch_pair(ptrs[0], ptrs[1], ptrs[2], nr, nc, self.index[p], fmt)
        flat = [p for s in self.schedules for p in s]
        self.descs = (_lib.hh_pass_desc * len(flat))(*[p.to_desc() for p in flat])
        offs = np.cumsum([0] + [len(s) for s in self.schedules]).astype(np.int32)
        self.offsets_in = np.ascontiguousarray(offs)
        self.ny = np.zeros(n, np.int32)
        self.nx = np.zeros(n, np.int32)
        self.offsets = np.zeros(n + 1, np.int64)
        L = _lib.lib()
        _lib.check(L.hh_batch_grid(self.pairs, n, self.descs, _lib.i32ptr(self.offsets_in), len(self.schedules),
                                   _lib.i32ptr(self.ny), _lib.i32ptr(self.nx),
                                   self.offsets.ctypes.data_as(_lib._I64)))
        R = int(self.offsets[-1])
        self.out = {k: self._buffer(R, np.float32, pinned) for k in _FIELDS}
        self.outliers = self._buffer(R, np.uint8, pinned)
        self.gmask = np.zeros(R, np.uint8)
        self.sweeps = self._buffer(n, np.int32, pinned)
        self.sweeps[...] = 0
        self.result = _lib.hh_batch_result(
            _lib.i32ptr(self.ny), _lib.i32ptr(self.nx), self.offsets.ctypes.data_as(_lib._I64),
            *[_lib.fptr(self.out[k]) for k in _FIELDS], _lib.u8ptr(self.outliers), _lib.u8ptr(self.gmask),
            _lib.i32ptr(self.sweeps))
        self.smoothing = int(bool(predictor_smoothing))
        self.mask_threshold = float(mask_threshold)
        self.flags = (_lib.HH_BATCH_DEVICE_INPUTS if self.device else 0) | (0 if graph else _lib.HH_BATCH_NO_GRAPH)
        self._own_ws = workspace is None
        self.ws = workspace if workspace is not None else PIVWorkspace()
        self.npairs = n
        self._grids = {}

    def _buffer(self, n, dtype, pinned):
        """Host result buffer; page-locked (through torch) when available so
        the read-back is one asynchronous copy per field."""
        if pinned:
            try:
                import torch
                if torch.cuda.is_available():
                    t = torch.empty(max(n, 1), dtype={np.float32: torch.float32, np.uint8: torch.uint8,
                                                      np.int32: torch.int32}[dtype], pin_memory=True)
                    self._keep.append(t)
                    return t.numpy()[:n]
            except Exception:  # noqa: BLE001 -- no CUDA torch: pageable buffers
                pass
        return np.empty(n, dtype)

    @property
    def final_vectors(self):
        """Final-pass vectors of the batch (grid cells not masked)."""
        return int(self.offsets[-1] - self.gmask.sum())

    def run(self, read=True, wait=True):
        """Analyse the whole batch once; results land in the runner's buffers
        (read=False leaves them on the device, for timing the device work).
        wait=False returns once the run and its read-back are queued on the
        workspace's stream (HH_BATCH_ASYNC): wait on that stream (for example
        through an event recorded on it, see `stream`) before reading the
        results or changing the images."""
        L = _lib.lib()
        flags = self.flags | (0 if wait else _lib.HH_BATCH_ASYNC)
        st = L.hh_run_batched(self.ws.ctx, self.pairs, self.npairs, self.descs, _lib.i32ptr(self.offsets_in),
                              len(self.schedules), self.mask_threshold, self.smoothing, flags,
                              ctypes.byref(self.result) if read else None)
        _lib.check(st, self.ws.ctx)
        return self

    def results(self, copy=True):
        """PIVResult per pair (views into the runner's buffers unless copy;
        with copy, views into one private copy of each buffer)."""
        R = int(self.offsets[-1])
        if copy:
            fields = {k: self.out[k][:R].copy() for k in _FIELDS}
            outl, gmask = self.outliers[:R].astype(bool), self.gmask[:R].astype(bool)
        else:
            fields = self.out
            outl, gmask = self.outliers, self.gmask
        res = []
        for p in range(self.npairs):
            a, b = int(self.offsets[p]), int(self.offsets[p + 1])
            ny, nx = int(self.ny[p]), int(self.nx[p])
            sched = self.schedules[self.index[p]]
            nr, nc = int(self.pairs[p].nr), int(self.pairs[p].nc)
            key = (nr, nc, self.index[p])
            if key not in self._grids:
                x, y, _, _ = pass_grid((nr, nc), sched[-1])
                self._grids[key] = (x, y)
            x, y = self._grids[key]

            def f(arr):
                return arr[a:b].reshape((ny, nx), order="F")

            sweeps = np.zeros(len(sched), np.int32)
            sweeps[-1] = self.sweeps[p]
            res.append(PIVResult(x.copy(), y.copy(), *[f(fields[k]) for k in _FIELDS],
                                 f(outl) if copy else f(outl).astype(bool), f(gmask) if copy else f(gmask).astype(bool),
                                 sched[-1], None, None, None, sweeps))
        return res

    def close(self):
        if self._own_ws and self.ws is not None:
            self.ws.close()
        self.ws = None


def run_piv_batch(pairs, passes, *, masks=None, predictor_smoothing=True, mask_threshold=0.5, workspace=None,
                  graph=True):
    """Analyse many pairs at once; returns one PIVResult per pair, equal to
    run_piv(A, B, schedule) of each pair.

    `pairs`: list of (A, B) images (numpy (rows, cols) arrays, or column-major
    torch CUDA tensors); `passes`: one schedule (a PIVParameters or a list of
    them) for every pair, or one schedule per pair; `masks`: None or one mask
    (or None) per pair.

    A batch whose device storage does not fit (the library reports
    HH_ERR_OOM and releases what it had allocated) is split in halves that run
    one after the other, down to single pairs; the results are the same, as
    every pair's result is independent of its batch. This is the bounded
    sub-batch of the reference's device backends (the memory-aware batch cap,
    ext/HammerheadCUDAExt.jl:147-164) taken on demand."""
    if not pairs:
        raise ArgumentError("pairs must not be empty")
    n = len(pairs)
    try:
        runner = BatchRunner(pairs, passes, masks=masks, predictor_smoothing=predictor_smoothing,
                             mask_threshold=mask_threshold, workspace=workspace, graph=graph, pinned=False)
        try:
            return runner.run().results(copy=True)
        finally:
            runner.close()
    except _lib.HammerheadError as e:
        if e.status != _lib.HH_ERR_OOM or n == 1:
            raise
    uniq, index = _schedules(passes, n)
    per_pair = [uniq[k] for k in index]
    masks = [None] * n if masks is None else list(masks)
    h = n // 2
    kw = dict(predictor_smoothing=predictor_smoothing, mask_threshold=mask_threshold, workspace=workspace,
              graph=graph)
    return (run_piv_batch(pairs[:h], per_pair[:h], masks=masks[:h], **kw) +
            run_piv_batch(pairs[h:], per_pair[h:], masks=masks[h:], **kw))


def run_piv_sequence(pairs, params=None, *, preprocess=None, progress=False, on_result=None, mask=None,
                     batch_size=16, predictor_smoothing=True, mask_threshold=0.5, workspace=None, u16="normalised",
                     pipeline=True):
    """run_piv_sequence (src/io.jl:229-247) for in-memory pairs.

    Pairs are analysed in batches of `batch_size` with the batched schedule;
    `on_result(i, r)` and `progress(i, n)` are called per pair in order
    (1-based i), as each batch completes. `mask` is None, one mask for every
    pair, or a function (i, pair) -> mask. Frames may be float32 or UInt16
    (converted on the device, see BatchRunner).

    With `pipeline` (CUDA available, every pair of one shape and pixel type,
    no mask or one mask for every pair), the frames of batch k+1 are copied
    to the device through
    page-locked double buffers on a copy stream while batch k is analysed,
    so ingestion overlaps the analysis (the reference prefetches the next
    pair's frames on a background task, src/io.jl:296-306)."""
    if not pairs:
        raise ArgumentError("pairs must not be empty")
    if params is None:
        params = [PIVParameters()]
    n = len(pairs)
    if preprocess is not None:
        pairs = [(preprocess(a), preprocess(b)) for a, b in pairs]
    same = len({(tuple(a.shape), str(a.dtype), tuple(b.shape), str(b.dtype)) for a, b in pairs}) == 1
    if pipeline and not callable(mask) and same and not _is_device(pairs[0][0]):
        try:
            import torch
            ok = torch.cuda.is_available()
        except Exception:  # noqa: BLE001 -- no torch: unpipelined path
            ok = False
        if ok:
            return _sequence_pipelined(pairs, params, on_result, progress, batch_size, predictor_smoothing,
                                       mask_threshold, workspace, u16, mask)
    out = []
    for start in range(0, n, batch_size):
        chunk = pairs[start:start + batch_size]
        if mask is None:
            ms = None
        elif callable(mask):
            ms = [mask(start + j + 1, chunk[j]) for j in range(len(chunk))]
        else:
            ms = [mask] * len(chunk)
        runner = BatchRunner(chunk, params, masks=ms, predictor_smoothing=predictor_smoothing,
                             mask_threshold=mask_threshold, workspace=workspace, pinned=False, u16=u16)
        try:
            res = runner.run().results(copy=True)
        finally:
            runner.close()
        for j, r in enumerate(res):
            i = start + j + 1
            out.append(r)
            if on_result is not None:
                on_result(i, r)
            if callable(progress):
                progress(i, n)
    return out


def _is_device(a):
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def _device_mask(m, shape):
    """A host mask as a column-major uint8 CUDA tensor (stride (1, nrows))."""
    import torch

    m = np.asarray(m)
    if tuple(m.shape) != tuple(shape):
        raise DimensionMismatch(f"mask must have the same size as the images, got {tuple(m.shape)}")
    return torch.from_numpy(np.ascontiguousarray(m.T != 0).astype(np.uint8)).cuda().T


def _sequence_pipelined(pairs, params, on_result, progress, batch_size, smoothing, thr, workspace, u16, mask=None):
    import concurrent.futures as cf

    import torch

    n = len(pairs)
    nr, nc = pairs[0][0].shape
    dmask = None if mask is None else _device_mask(mask, (nr, nc))
    tdt = torch.uint16 if _is_u16(pairs[0][0]) else torch.float32
    ndt = np.uint16 if tdt == torch.uint16 else np.float32
    B = min(batch_size, n)
    own = workspace is None
    ws = workspace if workspace is not None else PIVWorkspace()
    copy_stream = torch.cuda.Stream()
    # two sets of (pinned host, device) frame buffers, column-major (stride (1, nr))
    host = [torch.empty((2 * B, nc, nr), dtype=tdt, pin_memory=True) for _ in range(2)]
    dev = [torch.empty((2 * B, nc, nr), dtype=tdt, device="cuda") for _ in range(2)]
    events = [torch.cuda.Event(), torch.cuda.Event()]
    runners = {}

    def stage(k, slot):
        """Host -> page-locked -> device copy of batch k into buffer set `slot`."""
        chunk = pairs[k * B:(k + 1) * B]
        hv = host[slot].numpy()
        for j, (a, b) in enumerate(chunk):
            hv[2 * j] = np.asarray(a, ndt).T
            hv[2 * j + 1] = np.asarray(b, ndt).T
        with torch.cuda.stream(copy_stream):
            dev[slot][:2 * len(chunk)].copy_(host[slot][:2 * len(chunk)], non_blocking=True)
            events[slot].record(copy_stream)
        return len(chunk)

    def runner_for(slot, m):
        key = (slot, m)
        if key not in runners:
            frames = [(dev[slot][2 * j].T, dev[slot][2 * j + 1].T) for j in range(m)]
            runners[key] = BatchRunner(frames, params, masks=None if dmask is None else [dmask] * m,
                                       predictor_smoothing=smoothing, mask_threshold=thr, workspace=ws, u16=u16)
        return runners[key]

    nb = (n + B - 1) // B
    out = []
    try:
        with cf.ThreadPoolExecutor(max_workers=1) as pool:
            fut = pool.submit(stage, 0, 0)
            for k in range(nb):
                slot = k % 2
                m = fut.result()
                if k + 1 < nb:  # batch k+1 streams in while batch k is analysed
                    fut = pool.submit(stage, k + 1, (k + 1) % 2)
                events[slot].synchronize()
                res = runner_for(slot, m).run().results(copy=True)
                if k + 1 < nb:
                    fut.result()  # the next buffers are filled before this set is refilled
                    fut = _Done(fut.result())
                for j, r in enumerate(res):
                    i = k * B + j + 1
                    out.append(r)
                    if on_result is not None:
                        on_result(i, r)
                    if callable(progress):
                        progress(i, n)
    finally:
        for r in runners.values():
            r.close()
        if own:
            ws.close()
    return out


def run_piv_batch_stream(batches, passes, *, masks=None, predictor_smoothing=True, mask_threshold=0.5,
                         workspace=None, u16="normalised", on_batch=None):
    """A stream of batches of the same composition (for example every camera
    of a rig at each time step): batch k+1's frames are copied to the device
    on a copy stream while batch k is analysed, so the host-to-device copies
    overlap the analysis. Returns one list of PIVResult per batch (in order),
    equal to run_piv_batch on that batch; `on_batch(k, results)` is called as
    each batch completes (0-based k).

    Every batch holds the same number of pairs, and pair j has the same
    shape and pixel type (float32 or UInt16) in every batch. Frames in
    page-locked memory (for example numpy views of pinned torch tensors,
    column-major) are copied directly; others go through page-locked
    staging buffers first. `masks`: None or one mask (or None) per pair,
    the same for every batch (copied to the device once). Needs a CUDA
    device visible to torch. With a caller's
    workspace, the device frames and prepared runners of a composition are
    kept in it for the next call of the same composition."""
    import concurrent.futures as cf

    import torch

    it = iter(batches)
    try:
        first = list(next(it))
    except StopIteration:
        return []
    if not first:
        raise ArgumentError("batches must not be empty")
    n = len(first)
    spec = []
    for a, b in first:
        if tuple(a.shape) != tuple(b.shape) or len(a.shape) != 2:
            raise DimensionMismatch("each pair's frames must be matrices of one size")
        tdt = torch.uint16 if _is_u16(a) else torch.float32
        spec.append((int(a.shape[0]), int(a.shape[1]), tdt))
    own = workspace is None
    ws = workspace if workspace is not None else PIVWorkspace()
    scheds, index = _schedules(passes, n)
    if masks is not None:
        masks = list(masks)
        if len(masks) != n:
            raise DimensionMismatch(f"got {len(masks)} masks for {n} pairs")
    mkey = None if masks is None else tuple(
        None if m is None else zlib.crc32(np.asfortranarray(np.asarray(m) != 0).tobytes(order="F")) for m in masks)
    key = (tuple(spec), tuple(index), b"".join(bytes(q.to_desc()) for sc in scheds for q in sc),
           bool(predictor_smoothing), float(mask_threshold), u16, mkey)
    cache = None if own else ws.__dict__.setdefault("_stream_sessions", {})
    sess = None if cache is None else cache.get(key)
    if sess is None:
        sess = dict(copy_stream=torch.cuda.Stream(),
                    # two sets of device frames (column-major: tensors (nc, nr) seen through .T)
                    dev=[[(torch.empty((nc, nr), dtype=t, device="cuda"), torch.empty((nc, nr), dtype=t, device="cuda"))
                          for nr, nc, t in spec] for _ in range(2)],
                    stage_host={},  # page-locked staging for frames that are not page-locked already
                    events=[torch.cuda.Event(), torch.cuda.Event()], runners=None,
                    masks=None if masks is None else [None if m is None else _device_mask(m, sp[:2])
                                                      for m, sp in zip(masks, spec)])
    copy_stream, dev, stage_host, events = sess["copy_stream"], sess["dev"], sess["stage_host"], sess["events"]

    def host_tensor(x, j, which, slot):
        nr, nc, t = spec[j]
        if tuple(x.shape) != (nr, nc):
            raise DimensionMismatch(f"pair {j} changed size in the stream: {tuple(x.shape)} vs {(nr, nc)}")
        nd = np.uint16 if t == torch.uint16 else np.float32
        xt = np.asarray(x).T  # (nc, nr); C-contiguous when x is column-major
        if xt.dtype == nd and xt.flags["C_CONTIGUOUS"]:
            h = torch.from_numpy(xt)
            if h.is_pinned():
                return h
        key = (slot, j, which)
        if key not in stage_host:
            stage_host[key] = torch.empty((nc, nr), dtype=t, pin_memory=True)
        stage_host[key].numpy()[...] = xt.astype(nd, copy=False)
        return stage_host[key]

    def stage(batch, slot, after):
        """Queue the copies of `batch` into device set `slot` on the copy
        stream, behind `after` (the event behind the analysis that last read
        that set, or None)."""
        batch = list(batch)
        if len(batch) != n:
            raise DimensionMismatch(f"every batch must hold {n} pairs, got {len(batch)}")
        events[slot].synchronize()  # the last copies out of this set's staging buffers are done
        srcs = [(host_tensor(a, j, 0, slot), host_tensor(b, j, 1, slot)) for j, (a, b) in enumerate(batch)]
        with torch.cuda.stream(copy_stream):
            if after is not None:
                copy_stream.wait_event(after)
            for (da, db), (ha, hb_) in zip(dev[slot], srcs):
                da.copy_(ha, non_blocking=True)
                db.copy_(hb_, non_blocking=True)
            events[slot].record(copy_stream)
        return srcs  # kept alive until the copies are done

    out = []
    conv = [None, None]  # result conversion of the batch last analysed by each runner
    runners = sess["runners"]

    def collect(k, slot, done):
        done.synchronize()  # the run and read-back of batch k have finished
        res = runners[slot].results(copy=True)
        if on_batch is not None:
            on_batch(k, res)
        return res

    try:
        with cf.ThreadPoolExecutor(max_workers=1) as pool, cf.ThreadPoolExecutor(max_workers=1) as post:
            lib_stream = torch.cuda.ExternalStream(ws.stream(), device=torch.device("cuda", ws.device))
            done = [None, None]  # the event behind each runner's last queued run
            fut = pool.submit(stage, first, 0, None)
            if runners is None:  # prepared while the first batch is copied in
                runners = [BatchRunner([(a.T, b.T) for a, b in dev[s]], passes, masks=sess["masks"],
                                       predictor_smoothing=predictor_smoothing, mask_threshold=mask_threshold,
                                       workspace=ws, u16=u16) for s in range(2)]
                if cache is not None:
                    sess["runners"] = runners
                    cache[key] = sess
            k = 0
            pend = None  # the batch analysed last, not yet handed to the post thread
            while fut is not None:
                slot = k % 2
                fut.result()
                # the library stream waits for batch k's frames; the host does
                # not, so the device runs the queued batches back to back
                lib_stream.wait_event(events[slot])
                if conv[slot] is not None:  # this runner's buffers still hold batch k-2
                    out.append(conv[slot].result())
                    conv[slot] = None
                try:
                    nxt = next(it)
                except StopIteration:
                    nxt = None
                # batch k+1 streams into the other set while batch k is
                # analysed (that set's previous batch, k-1, finished before
                # this point), and the results of batch k-1 become PIVResults.
                # Both are handed over just before the library call, which
                # releases the interpreter lock: the helper threads then do
                # their Python work while the device runs, instead of holding
                # the lock while this thread prepares the call
                fut = pool.submit(stage, nxt, 1 - slot, done[1 - slot]) if nxt is not None else None
                if pend is not None:
                    conv[pend[1]] = post.submit(collect, *pend)
                runners[slot].run(wait=False)
                ev = torch.cuda.Event()
                ev.record(lib_stream)
                done[slot] = ev
                pend = (k, slot, ev)
                k += 1
            if pend is not None:
                conv[pend[1]] = post.submit(collect, *pend)
            for j in range(k - 2, k):
                if j >= 0 and conv[j % 2] is not None:
                    out.append(conv[j % 2].result())
                    conv[j % 2] = None
    finally:
        if ws.__dict__.get("_ctx") is not None:
            # no queued run still reads the frames
            torch.cuda.ExternalStream(ws.stream(), device=torch.device("cuda", ws.device)).synchronize()
        if own:
            for r in runners or ():
                r.close()
            ws.close()
    return out


class _Done:
    """A finished future (the staged size of the next batch)."""

    def __init__(self, v):
        self.v = v

    def result(self):
        return self.v
