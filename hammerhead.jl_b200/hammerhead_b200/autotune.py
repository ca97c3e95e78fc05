"""Autotuning of the correlation kernel's CTA shape and FFT split.

Every (FFT size, window) of the correlation kernel is built in
HH_CORR_VARIANTS variants: CTA shapes (windows per CTA, threads per window,
register budget) that compute the same results, and an alternative split
of each axis's DFT whose results differ by rounding. `autotune` times them on the
workspace's device (hh_autotune_correlation) for every pass class of a
schedule and makes the fastest the workspace's choice; the choices are kept
in a JSON cache keyed by device and (FFT size, window, peaks), so later runs
on the same kind of device reuse them without timing.
"""
import ctypes
import json
import os
import tempfile

import numpy as np

from . import _lib
from ._lib import ArgumentError
from .params import PIVParameters

VARIANTS = 5  # HH_CORR_VARIANTS


def _flatten(passes):
    if isinstance(passes, PIVParameters):
        return [passes]
    out = []
    for p in passes:
        out.extend(_flatten(p) if not isinstance(p, PIVParameters) else [p])
    return out


def pass_classes(passes):
    """The distinct (FFT size, window, peaks) of the equal-area passes of a
    pass, a schedule or a list of schedules that run on the fused
    correlation kernels, in first-seen order."""
    seen = []
    for p in _flatten(passes):
        if p.search_area_size != p.window_size:
            continue  # enlarged search areas have one shape
        if not _lib.lib().hh_corr_fused(ctypes.byref(p.to_desc())):
            continue  # the general-shape kernel has one shape
        w = p.window_size[0]
        c = (2 * w if p.padding else w, w, p.n_peaks)
        if c not in seen:
            seen.append(c)
    return seen


def tune_key(device, n, w, k):
    return f"{device}|N={n}|W={w}|K={k}"


def load_cache(path):
    """The cache's entries ({} when the file does not exist)."""
    if path is None or not os.path.exists(path):
        return {}
    with open(path) as f:
        data = json.load(f)
    if not isinstance(data, dict):
        raise ArgumentError(f"autotune cache {path} does not hold a JSON object")
    return data


def save_cache(path, data):
    """Write the cache atomically (a temporary file renamed over it)."""
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=d, suffix=".tmp")
    with os.fdopen(fd, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _device_name(ws):
    try:
        import torch

        return torch.cuda.get_device_name(ws.device).replace("|", "/")
    except Exception:  # noqa: BLE001 -- no CUDA torch: a device-index key
        return f"cuda:{ws.device}"


def set_variant(workspace, fft_size, window, variant):
    """Make `variant` the workspace's CTA shape for (fft_size, window)."""
    _lib.check(_lib.lib().hh_set_corr_variant(workspace.ctx, int(fft_size), int(window), int(variant)),
               workspace.ctx)


def autotune(passes, workspace, *, cache=None, reps=5, image_size=(1024, 1024), seed=11, retune=False):
    """Choose the correlation kernel's CTA shape for every pass class of
    `passes` on the workspace's device. With `cache` (a JSON file path),
    entries for this device are applied without timing unless `retune`;
    timed choices are written back. Returns {key: {"variant", "ms",
    "source"}} with `ms` the mean milliseconds per launch of each shape
    (None for cached entries)."""
    from . import synthetic

    if reps < 1:
        raise ArgumentError(f"reps must be at least 1, got {reps}")
    classes = pass_classes(passes)
    data = load_cache(cache)
    dev = _device_name(workspace)
    out = {}
    staged = False
    L = _lib.lib()
    for n, w, k in classes:
        key = tune_key(dev, n, w, k)
        entry = data.get(key)
        if entry is not None and not retune:
            set_variant(workspace, n, w, int(entry["variant"]))
            out[key] = {"variant": int(entry["variant"]), "ms": None, "source": "cache"}
            continue
        if not staged:
            A, B = synthetic.particle_pair(tuple(image_size), synthetic.uniform_flow(2.3, -1.7), seed=seed)
            A, B = _lib.as_f32_colmajor(A), _lib.as_f32_colmajor(B)
            _lib.check(L.hh_stage_pair(workspace.ctx, _lib.fptr(A), _lib.fptr(B), A.shape[0], A.shape[1]),
                       workspace.ctx)
            staged = True
        p = PIVParameters(window_size=w, overlap=w // 2, padding=n == 2 * w, apodization="gauss", n_peaks=k)
        d = p.to_desc()
        ms = (ctypes.c_float * VARIANTS)()
        best = ctypes.c_int32(0)
        _lib.check(L.hh_autotune_correlation(workspace.ctx, ctypes.byref(d), int(reps), ms, ctypes.byref(best)),
                   workspace.ctx)
        out[key] = {"variant": int(best.value), "ms": [float(x) for x in ms], "source": "timed"}
        data[key] = {"variant": int(best.value), "ms": [float(x) for x in ms]}
    if cache is not None and any(v["source"] == "timed" for v in out.values()):
        save_cache(cache, data)
    return out
