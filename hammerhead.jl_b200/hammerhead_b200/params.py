"""Pass configuration: PIVParameters, multipass_parameters, effort_schedule.

Mirror of the reference's PIVParameters (src/types.jl:212-291),
multipass_parameters (src/pipeline.jl:509-524) and effort_schedule
(src/pipeline.jl:172-234). Symbols are Python strings (``"cross"`` for
``:cross``); numeric checks run in the library's hh_pass_validate so the C
ABI and this layer reject exactly the same combinations with the same text.
"""
import ctypes
import math

from . import _lib
from ._lib import ArgumentError

_METHODS = {"cross": 0, "phase": 1}
_APOD = {"none": 0, "gauss": 1}
_SUBPIXEL = {"gauss3": 0, "gauss9": 1, "gauss2d": 2, "none": 3}
_FINDERS = {"regionalmax": 0, "exclusion": 1}


def _sym(x):
    return x[1:] if isinstance(x, str) and x.startswith(":") else x


def _pair(v, name):
    if isinstance(v, (int,)) and not isinstance(v, bool):
        return (int(v), int(v))
    try:
        a, b = v
        return (int(a), int(b))
    except Exception as e:  # noqa: BLE001
        raise ArgumentError(f"{name} must be an Int or a (rows, cols) tuple, got {v!r}") from e


def _fmt(t):
    return f"({t[0]}, {t[1]})"


class PeakRatioValidator:
    """Flag vectors whose peak ratio is below `threshold` (NaN flagged)."""
    kind = 0

    def __init__(self, threshold):
        self.threshold = float(threshold)

    def __repr__(self):
        return f"PeakRatioValidator({self.threshold})"


class CorrelationMomentValidator:
    """Flag vectors whose correlation moment exceeds `threshold` (NaN flagged)."""
    kind = 1

    def __init__(self, threshold):
        self.threshold = float(threshold)

    def __repr__(self):
        return f"CorrelationMomentValidator({self.threshold})"


class VelocityMagnitudeValidator:
    """Flag vectors whose |(u, v)| lies outside [min, max] (NaN flagged)."""
    kind = 2

    def __init__(self, min=0.0, max=math.inf):  # noqa: A002
        self.min = float(min)
        self.max = float(max)

    def __repr__(self):
        return f"VelocityMagnitudeValidator({self.min}, {self.max})"


class UniversalOutlierValidator:
    """Normalized median test (universal_outlier_detection)."""
    kind = 3

    def __init__(self, threshold, neighborhood_size=2, epsilon=0.1):
        self.threshold = float(threshold)
        self.neighborhood_size = int(neighborhood_size)
        self.epsilon = float(epsilon)

    def __repr__(self):
        return (f"UniversalOutlierValidator({self.threshold}, neighborhood_size={self.neighborhood_size}, "
                f"epsilon={self.epsilon})")


_VALIDATOR_TYPES = (PeakRatioValidator, CorrelationMomentValidator, VelocityMagnitudeValidator,
                    UniversalOutlierValidator)


def parse_validator(spec):
    """parse_validator (src/quality.jl:426-450): objects pass through,
    ``(name, value)`` pairs build the validator."""
    if isinstance(spec, _VALIDATOR_TYPES):
        return spec
    if isinstance(spec, tuple) and len(spec) == 2 and isinstance(spec[0], str):
        name, val = _sym(spec[0]), spec[1]
        if isinstance(val, (int, float)) and not isinstance(val, bool):
            if name == "peak_ratio":
                return PeakRatioValidator(val)
            if name == "correlation_moment":
                return CorrelationMomentValidator(val)
            raise ArgumentError(f"unknown validator :{name} (expected :peak_ratio or :correlation_moment)")
        if isinstance(val, dict):
            if name in ("uod", "universal_outlier"):
                return UniversalOutlierValidator(val["threshold"], val.get("neighborhood_size", 2),
                                                 val.get("epsilon", 0.1))
            if name == "velocity_magnitude":
                return VelocityMagnitudeValidator(val.get("min", 0.0), val["max"])
            raise ArgumentError(f"unknown validator :{name} (expected :uod or :velocity_magnitude)")
    raise ArgumentError(f"cannot interpret {spec!r} as a validator")


class PIVParameters:
    """Immutable, validated configuration for one PIV pass.

    Keyword arguments, defaults and error messages follow the reference
    PIVParameters constructor (src/types.jl:212-291).
    """

    __slots__ = ("window_size", "search_area_size", "overlap", "correlation_method", "padding", "apodization",
                 "subpixel_method", "n_peaks", "peak_finder", "uncertainty", "uod_enable", "uod_threshold",
                 "uod_neighborhood", "min_peak_ratio", "validation", "replace_outliers", "max_iterations",
                 "convergence_tol", "keep_correlation_planes")

    def __init__(self, *, window_size=(32, 32), search_area_size=None, overlap=(16, 16), correlation_method="cross",
                 padding=False, apodization="none", subpixel_method="gauss3", n_peaks=3, peak_finder="regionalmax",
                 uncertainty=False, uod_enable=True, uod_threshold=2.0, uod_neighborhood=2, min_peak_ratio=1.0,
                 validation=(), replace_outliers=True, max_iterations=1, convergence_tol=0.05,
                 keep_correlation_planes=False):
        ws = _pair(window_size, "window_size")
        ss = ws if search_area_size is None else _pair(search_area_size, "search_area_size")
        ov = _pair(overlap, "overlap")
        cm, ap, sp, pf = _sym(correlation_method), _sym(apodization), _sym(subpixel_method), _sym(peak_finder)
        if cm not in _METHODS:
            raise ArgumentError(f"correlation_method must be :cross or :phase, got :{cm}")
        if ap not in _APOD:
            raise ArgumentError(f"apodization must be :none or :gauss, got :{ap}")
        if sp not in _SUBPIXEL:
            raise ArgumentError(f"subpixel_method must be :gauss3, :gauss9, :gauss2d, or :none, got :{sp}")
        if pf not in _FINDERS:
            raise ArgumentError(f"peak_finder must be :exclusion or :regionalmax, got :{pf}")
        set_ = object.__setattr__
        set_(self, "window_size", ws)
        set_(self, "search_area_size", ss)
        set_(self, "overlap", ov)
        set_(self, "correlation_method", cm)
        set_(self, "padding", bool(padding))
        set_(self, "apodization", ap)
        set_(self, "subpixel_method", sp)
        set_(self, "n_peaks", int(n_peaks))
        set_(self, "peak_finder", pf)
        set_(self, "uncertainty", bool(uncertainty))
        set_(self, "uod_enable", bool(uod_enable))
        set_(self, "uod_threshold", float(uod_threshold))
        set_(self, "uod_neighborhood", int(uod_neighborhood))
        set_(self, "min_peak_ratio", float(min_peak_ratio))
        vals = validation if isinstance(validation, (tuple, list)) else (validation,)
        set_(self, "validation", tuple(parse_validator(v) for v in vals))
        set_(self, "replace_outliers", bool(replace_outliers))
        set_(self, "max_iterations", int(max_iterations))
        set_(self, "convergence_tol", float(convergence_tol))
        set_(self, "keep_correlation_planes", bool(keep_correlation_planes))
        _lib.check(_lib.lib().hh_pass_validate(ctypes.byref(self.to_desc())))

    def __setattr__(self, k, v):
        raise AttributeError("PIVParameters is immutable")

    def _replace(self, **kw):
        d = {k: getattr(self, k) for k in self.__slots__}
        d.update(kw)
        return PIVParameters(**d)

    def to_desc(self):
        """The hh_pass_desc of this pass."""
        d = _lib.hh_pass_desc()
        d.window[0], d.window[1] = self.window_size
        d.search[0], d.search[1] = self.search_area_size
        d.overlap[0], d.overlap[1] = self.overlap
        d.method = _METHODS[self.correlation_method]
        d.padding = int(self.padding)
        d.apodization = _APOD[self.apodization]
        d.subpixel = _SUBPIXEL[self.subpixel_method]
        d.n_peaks = self.n_peaks
        d.peak_finder = _FINDERS[self.peak_finder]
        d.uncertainty = int(self.uncertainty)
        d.uod_enable = int(self.uod_enable)
        d.uod_threshold = self.uod_threshold
        d.uod_neighborhood = self.uod_neighborhood
        d.replace_outliers = int(self.replace_outliers)
        d.min_peak_ratio = self.min_peak_ratio
        d.max_iterations = self.max_iterations
        d.keep_correlation_planes = int(self.keep_correlation_planes)
        d.convergence_tol = self.convergence_tol
        if len(self.validation) > _lib.MAX_VALIDATORS:
            raise ArgumentError(f"at most {_lib.MAX_VALIDATORS} extra validators are supported")
        d.n_validators = len(self.validation)
        for i, v in enumerate(self.validation):
            e = d.validators[i]
            e.kind = v.kind
            e.neighborhood = getattr(v, "neighborhood_size", 0)
            e.threshold = getattr(v, "threshold", 0.0)
            e.vmin = getattr(v, "min", 0.0)
            e.vmax = getattr(v, "max", 0.0)
            e.epsilon = getattr(v, "epsilon", 0.0)
        return d

    def __eq__(self, other):
        return isinstance(other, PIVParameters) and all(
            repr(getattr(self, k)) == repr(getattr(other, k)) for k in self.__slots__)

    def __hash__(self):
        return hash(tuple(repr(getattr(self, k)) for k in self.__slots__))

    def __repr__(self):
        s = f"PIVParameters(window_size={_fmt(self.window_size)}"
        if self.search_area_size != self.window_size:
            s += f", search_area_size={_fmt(self.search_area_size)}"
        s += (f", overlap={_fmt(self.overlap)}, correlation_method=:{self.correlation_method}, "
              f"padding={str(self.padding).lower()}, apodization=:{self.apodization}, "
              f"subpixel_method=:{self.subpixel_method}, n_peaks={self.n_peaks}, ")
        if self.peak_finder != "regionalmax":
            s += f"peak_finder=:{self.peak_finder}, "
        if self.uncertainty:
            s += "uncertainty=true, "
        s += "uod=" + (f"(threshold={self.uod_threshold}, neighborhood={self.uod_neighborhood})"
                       if self.uod_enable else "off")
        s += f", min_peak_ratio={self.min_peak_ratio}"
        if self.validation:
            s += f", validation={self.validation}"
        s += f", replace_outliers={str(self.replace_outliers).lower()}"
        if self.max_iterations > 1:
            s += f", max_iterations={self.max_iterations}, convergence_tol={self.convergence_tol}"
        if self.keep_correlation_planes:
            s += ", keep_correlation_planes=true"
        return s + ")"

    __str__ = __repr__


def multipass_parameters(window_sizes, *, overlap_fraction=0.5, final=None, **kwargs):
    """One PIVParameters per window size with overlap = floor(w * fraction);
    `final` overrides apply to the last pass only (src/pipeline.jl:509-524)."""
    if not (0 <= overlap_fraction < 1):
        raise ArgumentError(f"overlap_fraction must be in [0, 1), got {overlap_fraction}")
    window_sizes = list(window_sizes)
    if not window_sizes:
        raise ArgumentError("window_sizes must not be empty")
    final = dict(final or {})
    out = []
    n = len(window_sizes)
    for i, w in enumerate(window_sizes):
        ws = _pair(w, "window_size")
        extra = dict(kwargs)
        if i == n - 1:
            extra.update(final)
        out.append(PIVParameters(window_size=ws, overlap=(math.floor(ws[0] * overlap_fraction),
                                                          math.floor(ws[1] * overlap_fraction)), **extra))
    return out


EFFORT_LEVELS = ("low", "medium", "high")
_EFFORT_FINAL_ONLY = ("uncertainty", "max_iterations", "keep_correlation_planes")


def effort_schedule(level, *, ensemble=False, image_size=None, final=None, **kwargs):
    """Preset schedules of `effort = :low/:medium/:high` (src/pipeline.jl:172-234)."""
    level = _sym(level)
    if level not in EFFORT_LEVELS:
        raise ArgumentError("unknown effort :%s; expected one of :low, :medium, :high" % level)
    if level == "low":
        base, shared, pfinal = [(32, 32)], {}, {}
    elif level == "medium":
        base, shared, pfinal = [(64, 64), (32, 32)], {}, {}
    else:
        base = [(128, 128), (64, 64), (32, 32), (32, 32)] if ensemble else [(128, 128), (64, 64), (32, 32)]
        shared, pfinal = {"padding": True, "apodization": "gauss", "max_iterations": 2}, {"uncertainty": True}
    if "window_size" in kwargs:
        t = _pair(kwargs["window_size"], "window_size")
        bf = base[-1]
        windows = [(max(4, round(w[0] * t[0] / bf[0])), max(4, round(w[1] * t[1] / bf[1]))) for w in base]
    else:
        windows = list(base)
    if image_size is not None:
        windows = [(min(w[0], image_size[0]), min(w[1], image_size[1])) for w in windows]
    shared_ov = {k: v for k, v in kwargs.items() if k not in ("window_size", "search_area_size")
                 and k not in _EFFORT_FINAL_ONLY}
    final_ov = {k: v for k, v in kwargs.items() if k in _EFFORT_FINAL_ONLY}
    shared = {**shared, **shared_ov}
    final_all = {**pfinal, **final_ov, **dict(final or {})}
    if "search_area_size" in kwargs:
        t = _pair(final_all.get("search_area_size", kwargs["search_area_size"]), "search_area_size")
        final_wo = {k: v for k, v in final_all.items() if k != "search_area_size"}
        fw = windows[-1]
        if not (t[0] >= fw[0] and t[1] >= fw[1]):
            raise ArgumentError(f"search_area_size must be at least the final window_size {fw}, got {t}")
        if (t[0] - fw[0]) % 2 or (t[1] - fw[1]) % 2:
            raise ArgumentError(f"search_area_size - final window_size must be even in each dimension, got {t} and {fw}")
        out = []
        for i, w in enumerate(windows):
            s = []
            for d in range(2):
                x = max(w[d], round(t[d] * w[d] / fw[d]))
                if (x - w[d]) % 2:
                    x += 1
                if image_size is not None and x > image_size[d]:
                    x = image_size[d] - (image_size[d] - w[d]) % 2
                s.append(x)
            extra = {**shared, **final_wo} if i == len(windows) - 1 else shared
            out.append(PIVParameters(window_size=w, search_area_size=tuple(s),
                                     overlap=(math.floor(w[0] * 0.5), math.floor(w[1] * 0.5)), **extra))
        return out
    return multipass_parameters(windows, final=final_all, **shared)
