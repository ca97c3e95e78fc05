"""Device adjoint of deformation + zero-lag correlation (hh_ncc_loss_grad)
on the differentiation case: the 1024 x 1024 vortex pair, P = truth on the
127 x 127 window-centre grid + N(0, 0.3 px), 16 x 16 windows at 50 %.

Checks (tolerances as stated for this case): the FP32 device gradient
against FP64 central differences (h = 1e-3 px) on 64 random components,
relative error <= 1e-3; against the full FP64 analytic gradient of the
oracle, relative L2 error <= 1e-3 and every component within 1e-3 of the
largest; the loss within 1e-5 relative of the FP64 loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(hb, orc, ws):
    A, B, flow, P, grid = hb.synthetic.config2_case()
    loss = hb.NCCLoss(A, B, window=16, overlap=8, workspace=ws)
    L, g = loss.value_and_grad(P, grid)
    cA = orc.prefilter(A, dtype=np.float64)
    cB = orc.prefilter(B, dtype=np.float64)
    return dict(A=A, B=B, P=P, grid=grid, loss=loss, L=L, g=g, cA=cA, cB=cB)


def test_adjoint_vs_fp64_gradient(case, orc):
    L64, g64 = orc.ncc_loss_grad(case["cA"], case["cB"], case["A"].shape, case["P"].astype(np.float64),
                                 case["grid"], nthreads=16)
    assert abs(case["L"] - L64) <= 1e-5 * abs(L64)
    g = case["g"].astype(np.float64)
    assert np.linalg.norm(g - g64) <= 1e-3 * np.linalg.norm(g64)
    assert np.abs(g - g64).max() <= 1e-3 * np.abs(g64).max()


def _support_windows(orc, shape, grid, i, j, window=16, overlap=8):
    """Loss windows whose pixels reach node (i, j) through the bilinear stencil."""
    y0, ysp, x0, xsp = grid
    r_lo, r_hi = y0 + (i - 1) * ysp, y0 + (i + 1) * ysp
    c_lo, c_hi = x0 + (j - 1) * xsp, x0 + (j + 1) * xsp
    w = orc.ncc_windows(shape, window, overlap)
    rows_hit = (w[:, 0] + window >= r_lo) & (w[:, 0] + 1 <= r_hi)
    cols_hit = (w[:, 1] + window >= c_lo) & (w[:, 1] + 1 <= c_hi)
    return w[rows_hit & cols_hit]


def test_adjoint_vs_central_differences(case, orc):
    P = case["P"].astype(np.float64)
    shape, grid, g = case["A"].shape, case["grid"], case["g"]
    rng = np.random.default_rng(2024)
    h = 1e-3
    gmax = np.abs(g).max()
    errs = []
    for _ in range(64):
        i, j, c = rng.integers(P.shape[0]), rng.integers(P.shape[1]), rng.integers(2)
        wins = _support_windows(orc, shape, grid, i, j)
        Pp, Pm = P.copy(), P.copy()
        Pp[i, j, c] += h
        Pm[i, j, c] -= h
        Lp = orc.ncc_loss_grad(case["cA"], case["cB"], shape, Pp, grid, windows=wins, grad=False, nthreads=1)[0]
        Lm = orc.ncc_loss_grad(case["cA"], case["cB"], shape, Pm, grid, windows=wins, grad=False, nthreads=1)[0]
        fd = (Lp - Lm) / (2 * h)
        errs.append(abs(g[i, j, c] - fd) / max(abs(fd), 1e-2 * gmax))
    assert max(errs) <= 1e-3, max(errs)


def test_adjoint_loss_only_and_device_form(case, hb):
    import torch

    loss, P, grid = case["loss"], case["P"], case["grid"]
    assert loss.value(P, grid) == case["L"]
    gny, gnx = P.shape[:2]
    Pd = torch.from_numpy(hb.adjoint.to_planes(P)).cuda()
    gd = torch.empty_like(Pd)
    L = loss.device_value_and_grad(Pd, gny, gnx, grid, gd)
    assert L == case["L"]
    assert np.array_equal(hb.adjoint.from_planes(gd.cpu().numpy(), gny, gnx), case["g"])
    # autograd wrapper (the rrule): d(3 L)/dP = 3 dL/dP
    F = hb.adjoint.ncc_loss_function()
    Pt = Pd.clone().view(2, gnx, gny).requires_grad_(True)
    out = 3.0 * F.apply(Pt, loss, grid)
    out.backward()
    assert torch.allclose(Pt.grad.view(-1), 3.0 * gd)
