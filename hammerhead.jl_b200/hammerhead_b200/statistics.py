"""Ground-truth error statistics (error_statistics, src/statistics.jl:219-250)."""
import numpy as np


def sample_valid(result, include_invalid=False):
    ok = np.isfinite(result.u) & np.isfinite(result.v) & ~result.mask
    if not include_invalid:
        ok &= ~result.outliers
    return ok


def error_statistics(result, u_ref, v_ref, include_invalid=False):
    """Signed error fields and bias / RMS over valid vectors. u_ref, v_ref are
    grid-shaped arrays or functions (x, y) -> value (x along columns)."""
    X, Y = np.meshgrid(result.x.astype(float), result.y.astype(float))

    def field(f):
        return np.asarray(f, float) if not callable(f) else np.asarray(f(X, Y), float)

    ur, vr = field(u_ref), field(v_ref)
    ok = sample_valid(result, include_invalid)
    eu = np.where(ok, result.u.astype(float) - ur, np.nan)
    ev = np.where(ok, result.v.astype(float) - vr, np.nan)
    n = int(ok.sum())
    if n == 0:
        return dict(err_u=eu, err_v=ev, bias_u=np.nan, bias_v=np.nan, rms_u=np.nan, rms_v=np.nan, n=0)
    return dict(err_u=eu, err_v=ev, bias_u=float(np.nanmean(eu)), bias_v=float(np.nanmean(ev)),
                rms_u=float(np.sqrt(np.nanmean(eu ** 2))), rms_v=float(np.sqrt(np.nanmean(ev ** 2))), n=n)


def rms_error(result, flow, midpoint=True):
    """RMS of the vector error |d - d_true| over valid vectors, truth at the
    trajectory midpoint (bench/run_benchmarks.jl:199-215)."""
    from .synthetic import midpoint_truth

    X, Y = np.meshgrid(result.x.astype(float), result.y.astype(float))
    ut, vt = midpoint_truth(flow, X, Y) if midpoint else flow(X, Y)
    ok = sample_valid(result)
    e2 = (result.u.astype(float) - ut) ** 2 + (result.v.astype(float) - vt) ** 2
    return float(np.sqrt(np.mean(e2[ok]))) if ok.any() else float("nan")
