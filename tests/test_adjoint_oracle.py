"""The FP64 restatement of the correlation loss and its analytic gradient
(the reference for the device adjoint), pinned against central finite
differences of the same FP64 loss. CPU only."""
import numpy as np


def _case(orc, hb, shape=(88, 104), seed=3):
    syn = hb.synthetic
    flow = syn.sine_shear_flow(2.0, 96.0)
    A, B = syn.particle_pair(shape, flow, seed=seed)
    cA = orc.prefilter(A, dtype=np.float64)
    cB = orc.prefilter(B, dtype=np.float64)
    # nodes on the 16-px window centres at 8-px spacing (50 % overlap)
    y = 8.5 + 8.0 * np.arange((shape[0] - 16) // 8 + 1)
    x = 8.5 + 8.0 * np.arange((shape[1] - 16) // 8 + 1)
    rng = np.random.default_rng(seed)
    P = np.zeros((len(y), len(x), 2))
    for i, yy in enumerate(y):
        for j, xx in enumerate(x):
            P[i, j] = flow(xx, yy)
    P += rng.normal(0, 0.3, P.shape)
    return cA, cB, shape, P, (y[0], 8.0, x[0], 8.0)


def test_oracle_gradient_matches_central_differences(orc, hb):
    cA, cB, shape, P, grid = _case(orc, hb)
    L, g = orc.ncc_loss_grad(cA, cB, shape, P, grid)
    assert np.isfinite(L) and L < 0
    rng = np.random.default_rng(11)
    h = 1e-4
    scale = np.abs(g).max()
    for _ in range(24):
        i, j, c = rng.integers(P.shape[0]), rng.integers(P.shape[1]), rng.integers(2)
        Pp, Pm = P.copy(), P.copy()
        Pp[i, j, c] += h
        Pm[i, j, c] -= h
        fd = (orc.ncc_loss_grad(cA, cB, shape, Pp, grid, grad=False)[0] -
              orc.ncc_loss_grad(cA, cB, shape, Pm, grid, grad=False)[0]) / (2 * h)
        assert abs(fd - g[i, j, c]) <= 1e-5 * max(abs(fd), scale), (i, j, c, fd, g[i, j, c])


def test_oracle_loss_window_subsets_add_up(orc, hb):
    cA, cB, shape, P, grid = _case(orc, hb, seed=5)
    wins = orc.ncc_windows(shape, 16, 8)
    L, g = orc.ncc_loss_grad(cA, cB, shape, P, grid)
    half = len(wins) // 2
    L1, g1 = orc.ncc_loss_grad(cA, cB, shape, P, grid, windows=wins[:half])
    L2, g2 = orc.ncc_loss_grad(cA, cB, shape, P, grid, windows=wins[half:])
    assert abs(L - (L1 + L2)) < 1e-9 * abs(L)
    assert np.allclose(g, g1 + g2, rtol=0, atol=1e-12 * np.abs(g).max())
    # NCC of identical frames is 1 everywhere: L = -(number of windows), gradient 0 at P = 0
    L0, g0 = orc.ncc_loss_grad(cA, cA, shape, np.zeros_like(P), grid)
    assert abs(L0 + len(wins)) < 1e-9 * len(wins)
    assert np.abs(g0).max() < 1e-9
