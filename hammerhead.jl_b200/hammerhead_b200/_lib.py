"""ctypes binding of libhammerhead_b200.so (the C ABI in include/hammerhead_b200.h).

The shared library sits next to this file (built by hammerhead.jl_b200/build.py).
There is no fallback: if the library is missing, importing the device entry
points raises immediately.
"""
import ctypes
import os

import numpy as np

LIBNAME = "libhammerhead_b200.so"
LIBPATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIBNAME)

HH_OK = 0
HH_ERR_ARG = 1
HH_ERR_OOM = 2
HH_ERR_CUDA = 3
HH_ERR_TIMEOUT = 4
HH_ERR_UNSUPPORTED = 5
HH_ERR_STATE = 6

MAX_VALIDATORS = 8

# int32_t (*)(void* user, int32_t pass, float* planes, int64_t nplanes, double* stats, int64_t nstats, void* stream)
ENSEMBLE_REDUCER = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64,
                                    ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p)


class hh_validator(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("neighborhood", ctypes.c_int32),
        ("threshold", ctypes.c_double),
        ("vmin", ctypes.c_double),
        ("vmax", ctypes.c_double),
        ("epsilon", ctypes.c_double),
    ]


class hh_pass_desc(ctypes.Structure):
    _fields_ = [
        ("window", ctypes.c_int32 * 2),
        ("search", ctypes.c_int32 * 2),
        ("overlap", ctypes.c_int32 * 2),
        ("method", ctypes.c_int32),
        ("padding", ctypes.c_int32),
        ("apodization", ctypes.c_int32),
        ("subpixel", ctypes.c_int32),
        ("n_peaks", ctypes.c_int32),
        ("peak_finder", ctypes.c_int32),
        ("uncertainty", ctypes.c_int32),
        ("uod_enable", ctypes.c_int32),
        ("uod_threshold", ctypes.c_double),
        ("uod_neighborhood", ctypes.c_int32),
        ("replace_outliers", ctypes.c_int32),
        ("min_peak_ratio", ctypes.c_double),
        ("max_iterations", ctypes.c_int32),
        ("keep_correlation_planes", ctypes.c_int32),
        ("convergence_tol", ctypes.c_double),
        ("n_validators", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
        ("validators", hh_validator * MAX_VALIDATORS),
    ]


_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_I32 = ctypes.POINTER(ctypes.c_int32)
_I64 = ctypes.POINTER(ctypes.c_int64)


class hh_result(ctypes.Structure):
    _fields_ = [
        ("ny", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("x", _F),
        ("y", _F),
        ("u", _F),
        ("v", _F),
        ("peak_ratio", _F),
        ("correlation_moment", _F),
        ("uncertainty_u", _F),
        ("uncertainty_v", _F),
        ("outliers", _U8),
        ("mask", _U8),
    ]


class hh_batch_pair(ctypes.Structure):
    _fields_ = [
        ("A", ctypes.c_void_p),
        ("B", ctypes.c_void_p),
        ("mask", ctypes.c_void_p),
        ("nr", ctypes.c_int64),
        ("nc", ctypes.c_int64),
        ("schedule", ctypes.c_int32),
        ("format", ctypes.c_int32),
    ]


class hh_batch_result(ctypes.Structure):
    _fields_ = [
        ("ny", _I32),
        ("nx", _I32),
        ("offsets", _I64),
        ("u", _F),
        ("v", _F),
        ("peak_ratio", _F),
        ("correlation_moment", _F),
        ("uncertainty_u", _F),
        ("uncertainty_v", _F),
        ("outliers", _U8),
        ("mask", _U8),
        ("sweeps", _I32),
    ]


HH_BATCH_DEVICE_INPUTS = 1
HH_BATCH_NO_GRAPH = 2
HH_BATCH_ASYNC = 4
HH_PIX_F32 = 0
HH_PIX_U16 = 1
HH_PIX_U16_RAW = 2


class hh_kernel_profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("ms", ctypes.c_double), ("flops", ctypes.c_double),
                ("bytes", ctypes.c_double), ("units", ctypes.c_int64)]


KERNEL_CLASSES = ("correlate", "deform", "prefilter", "uq", "vector")

# Every symbol the header declares: (name, restype, argtypes)
_PASS = ctypes.POINTER(hh_pass_desc)
_CTX = ctypes.c_void_p
SIGNATURES = [
    ("hh_version", ctypes.c_char_p, []),
    ("hh_last_error", ctypes.c_char_p, [_CTX]),
    ("hh_pass_validate", ctypes.c_int32, [_PASS]),
    ("hh_check_backend_params", ctypes.c_int32, [_PASS, ctypes.c_int32]),
    ("hh_pass_grid", ctypes.c_int32,
     [ctypes.c_int64, ctypes.c_int64, _PASS, _U8, ctypes.c_double, _I32, _I32, _F, _F, _U8, _I32, _I64]),
    ("hh_ctx_create", ctypes.c_int32, [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    ("hh_ctx_destroy", None, [_CTX]),
    ("hh_ctx_stream", ctypes.c_void_p, [_CTX]),
    ("hh_run_piv", ctypes.c_int32,
     [_CTX, _F, _F, ctypes.c_int64, ctypes.c_int64, _PASS, ctypes.c_int32, _U8, ctypes.c_double, ctypes.c_int32,
      ctypes.POINTER(hh_result)]),
    ("hh_run_piv_device", ctypes.c_int32,
     [_CTX, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, _PASS, ctypes.c_int32, ctypes.c_void_p,
      ctypes.c_double, ctypes.c_int32, ctypes.POINTER(hh_result)]),
    ("hh_last_pass_times", ctypes.c_int32, [_CTX, ctypes.c_int32, _F, _I32]),
    ("hh_batch_grid", ctypes.c_int32,
     [ctypes.POINTER(hh_batch_pair), ctypes.c_int32, _PASS, _I32, ctypes.c_int32, _I32, _I32, _I64]),
    ("hh_run_batched", ctypes.c_int32,
     [_CTX, ctypes.POINTER(hh_batch_pair), ctypes.c_int32, _PASS, _I32, ctypes.c_int32, ctypes.c_double,
      ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(hh_batch_result)]),
    ("hh_stage_pair", ctypes.c_int32, [_CTX, _F, _F, ctypes.c_int64, ctypes.c_int64]),
    ("hh_apply_predictor", ctypes.c_int32,
     [_CTX, _F, _F, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
      _F, ctypes.c_int32, _F, ctypes.c_int32, _F, _F, _F, _F]),
    ("hh_stage_mask", ctypes.c_int32, [_CTX, _U8]),
    ("hh_process_windows", ctypes.c_int32, [_CTX, _PASS, _I32, ctypes.c_int64, _F, _I32, _D]),
    ("hh_analyze_planes", ctypes.c_int32,
     [_CTX, _F, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _F,
      _I32]),
    ("hh_correlation_planes", ctypes.c_int32, [_CTX, _PASS, _I32, ctypes.c_int64, _F]),
    ("hh_validate", ctypes.c_int32,
     [_CTX, _PASS, ctypes.c_int32, ctypes.c_int32, _F, _F, _F, _F, _U8, _U8, _F, _F, ctypes.c_int32, ctypes.c_int32]),
    ("hh_uod", ctypes.c_int32,
     [_CTX, _F, _F, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_double, _U8, _U8]),
    ("hh_replace_vectors", ctypes.c_int32, [_CTX, _F, _F, ctypes.c_int32, ctypes.c_int32, _U8]),
    ("hh_smooth_field", ctypes.c_int32, [_CTX, _F, ctypes.c_int32, ctypes.c_int32, _F]),
    ("hh_field_change", ctypes.c_int32, [_CTX, _F, _F, _F, _F, _U8, ctypes.c_int64, _F]),
    ("hh_finalize_uncertainty", ctypes.c_int32, [_D, ctypes.c_int64, _F, _F]),
    ("hh_run_ensemble", ctypes.c_int32,
     [_CTX, ctypes.POINTER(hh_batch_pair), ctypes.c_int32, _PASS, ctypes.c_int32, _U8, ctypes.c_double,
      ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(hh_result)]),
    ("hh_set_ensemble_reducer", ctypes.c_int32, [_CTX, ctypes.c_void_p, ctypes.c_void_p]),
    ("hh_autotune_correlation", ctypes.c_int32,
     [_CTX, _PASS, ctypes.c_int32, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int32)]),
    ("hh_set_corr_variant", ctypes.c_int32, [_CTX, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    ("hh_corr_fused", ctypes.c_int32, [_PASS]),
    ("hh_ncc_loss_grad", ctypes.c_int32,
     [_CTX, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
      ctypes.c_float, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
      ctypes.c_void_p]),
    ("hh_set_profiling", ctypes.c_int32, [_CTX, ctypes.c_int32]),
    ("hh_profile_read", ctypes.c_int32, [_CTX, ctypes.POINTER(hh_kernel_profile), ctypes.c_int32]),
    ("hh_launch_count", ctypes.c_int64, [_CTX]),
    ("hh_debug_fail_alloc", ctypes.c_int32, [_CTX, ctypes.c_int64]),
    ("hh_field_change_noalloc", ctypes.c_int32,
     [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
      ctypes.c_void_p, ctypes.c_void_p]),
    ("hh_noalloc_last_error", ctypes.c_char_p, []),
]


def profile_read(ctx, reset=False):
    """Per-kernel-class totals {name: dict(launches, ms, flops, bytes, units)}."""
    arr = (hh_kernel_profile * len(KERNEL_CLASSES))()
    check(lib().hh_profile_read(ctx, arr, int(reset)), ctx)
    return {name: dict(launches=e.launches, ms=e.ms, flops=e.flops, bytes=e.bytes, units=e.units)
            for name, e in zip(KERNEL_CLASSES, arr)}

_lib = None


def lib():
    """The loaded library (loaded once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(
                f"{LIBNAME} not found at {LIBPATH}; build it with `python hammerhead.jl_b200/build.py` "
                "(the b200 backend has no CPU fallback)")
        L = ctypes.CDLL(LIBPATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class HammerheadError(RuntimeError):
    """A device-side failure reported by the library (status != HH_OK)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class ArgumentError(ValueError):
    """The reference's ArgumentError: an invalid option, raised before any work."""


class DimensionMismatch(ValueError):
    """The reference's DimensionMismatch."""


def last_error(ctx=None):
    msg = lib().hh_last_error(ctx)
    return msg.decode("utf-8", "replace") if msg else ""


def check(status, ctx=None):
    if status == HH_OK:
        return
    msg = last_error(ctx)
    if status in (HH_ERR_ARG, HH_ERR_UNSUPPORTED):
        raise ArgumentError(msg)
    raise HammerheadError(status, msg)


def fptr(a):
    return a.ctypes.data_as(_F) if a is not None else None


def dptr(a):
    return a.ctypes.data_as(_D) if a is not None else None


def u8ptr(a):
    return a.ctypes.data_as(_U8) if a is not None else None


def i32ptr(a):
    return a.ctypes.data_as(_I32) if a is not None else None


def as_f32_colmajor(a):
    return np.asfortranarray(np.asarray(a), dtype=np.float32)
