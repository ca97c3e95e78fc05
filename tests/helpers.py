"""Test-image helpers restating test/runtests.jl:11-34 of the reference.

add_particle!: a Gaussian particle with diameter ~ 2 sigma, cut at 5 sigma.
particle_pair: the same particles displaced by (dv, du) = (drow, dcol).
Positions are (row, col), 1-based, like the Julia tests. The reference draws
positions from Julia RNG streams that do not exist here; tests draw them
from numpy generators with the same distributions.
"""
import numpy as np


def add_particle(array, centroid, diameter):
    sigma = diameter / 2
    nr, nc = array.shape
    i = np.arange(1, nr + 1)[:, None]
    j = np.arange(1, nc + 1)[None, :]
    d2 = (i - centroid[0]) ** 2 + (j - centroid[1]) ** 2
    val = np.exp(-0.5 * d2 / sigma ** 2)
    array += np.where(d2 > (5 * sigma) ** 2, 0.0, val)
    return array


def particle_pair(image_size, positions, dv, du, diameter=3.0):
    A = np.zeros(image_size, np.float64)
    B = np.zeros(image_size, np.float64)
    for p in positions:
        add_particle(A, p, diameter)
        add_particle(B, (p[0] + dv, p[1] + du), diameter)
    return np.asfortranarray(A), np.asfortranarray(B)


def random_positions(rng, n, extent, margin=10):
    return [(rng.uniform() * (extent + 2 * margin) - margin, rng.uniform() * (extent + 2 * margin) - margin)
            for _ in range(n)]


def shear_pair(seed, n=128, a=1 / 16, count=900):
    """u(y) = a (y - 64), v = 0 (test/runtests.jl:338-352)."""
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    B = np.zeros((n, n))
    for _ in range(count):
        p = (rng.uniform() * (n + 20) - 10, rng.uniform() * (n + 20) - 10)
        add_particle(A, p, 3.0)
        add_particle(B, (p[0], p[1] + a * (p[0] - 64)), 3.0)
    return np.asfortranarray(A), np.asfortranarray(B)


class Grid:
    """Duck-typed result for error statistics over an oracle output dict."""

    def __init__(self, d):
        for k in ("x", "y", "u", "v", "mask", "outliers"):
            setattr(self, k, d[k])


def plane_decision_margin(R, locs_a, locs_b, k, finder="regionalmax", excl=2):
    """Smallest gap, in the plane R, between two values whose order decides
    the peaks a finder reports: consecutive values of the ranked candidates
    (the first k + 1), each reported location (of either result) against its
    neighbourhood (8 neighbours for regional maxima, the exclusion box for the
    exclusion finder), and each secondary value against zero. Two planes that
    differ by at most e element-wise can report different peaks only when
    this margin is at most 2 e (src/localmax.jl:3-19, src/correlators.jl:390-454)."""
    import oracle

    nr, nc = R.shape
    R64 = np.asarray(R, np.float64)
    cand = oracle.find_peaks(R64, k + 1, finder, excl)
    vals = [v for v, _ in cand]
    gaps = [abs(vals[i] - vals[i + 1]) for i in range(len(vals) - 1)]
    gaps += [abs(v) for v in vals[1:k + 1]]
    rad = 1 if finder == "regionalmax" else excl
    locs = set()
    for L in (locs_a, locs_b):
        L = np.asarray(L).ravel()
        for m in range(0, len(L) - 1, 2):
            r, c = int(L[m]), int(L[m + 1])
            if 1 <= r <= nr and 1 <= c <= nc:
                locs.add((r, c))
    for r, c in locs:
        r0, r1 = max(r - 1 - rad, 0), min(r + rad, nr)
        c0, c1 = max(c - 1 - rad, 0), min(c + rad, nc)
        box = R64[r0:r1, c0:c1].copy()
        box[r - 1 - r0, c - 1 - c0] = -np.inf
        nb = box.max() if box.size > 1 else -np.inf
        if np.isfinite(nb):
            gaps.append(abs(R64[r - 1, c - 1] - nb))
    return min(gaps) if gaps else np.inf


def compare_runs(r, o, tol=1e-3, all_sweeps=True):
    """A device run against the oracle's Float32 run of the same schedule:
    grid masks, validation flags and sweep counts identical, every unmasked
    vector within `tol` px (the maximum, no quantile), and the uncertainty
    finite on the same cells with 99 % of it within 1e-3 px (a ring of the
    covariance sums that sits at finalize_uncertainty's 0.05 S00 threshold,
    src/uncertainty.jl:162-179, is decided by round-off). all_sweeps=False
    compares the final pass's sweep count only."""
    assert np.array_equal(r.mask, o["mask"])
    flips = np.argwhere(r.outliers != o["outliers"])
    assert len(flips) == 0, f"outlier flags differ at {flips[:10].tolist()}"
    # the batched form reports the final pass's sweep count only
    assert list(r.sweeps) == list(o["sweeps"]) if all_sweeps else r.sweeps[-1] == o["sweeps"][-1]
    ok = ~o["mask"]
    du, dv = np.abs(r.u - o["u"])[ok], np.abs(r.v - o["v"])[ok]
    assert du.max() <= tol and dv.max() <= tol, (du.max(), dv.max())
    fin = np.isfinite(r.uncertainty_u)
    assert np.array_equal(fin, np.isfinite(o["uncertainty_u"]))
    if fin.any():
        assert np.quantile(np.abs(r.uncertainty_u - o["uncertainty_u"])[fin], 0.99) < 1e-3
    return du.max(), dv.max()
