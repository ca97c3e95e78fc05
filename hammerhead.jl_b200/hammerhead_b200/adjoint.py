"""Differentiable correlation loss of a predictor field (hh_ncc_loss_grad).

L(P) = - sum over W x W windows j of NCC0_j, the zero-lag normalised
correlation of the pair deformed by the predictor P exactly as a WIDIM sweep
deforms it (bilinear predictor with flat extrapolation, symmetric cubic
B-spline sampling; deform_columns!, src/pipeline.jl:957-965). The gradient
dL/dP comes from a hand-written adjoint on the GPU that recomputes the
deformed windows instead of storing them.

P has shape (gny, gnx, 2): P[..., 0] = u (column displacement), P[..., 1] = v,
on nodes y0 + i*ysp (rows), x0 + j*xsp (columns), 1-based pixel coordinates
like PIVResult.x / .y.
"""
import ctypes

import numpy as np

from . import _lib
from .pipeline import PIVWorkspace, _is_device_tensor


def _grid(grid, gny, gnx):
    """(y0, ysp, x0, xsp) from a 4-tuple or from node coordinate vectors (y, x)."""
    if len(grid) == 4:
        return tuple(float(g) for g in grid)
    y, x = np.asarray(grid[0], np.float32), np.asarray(grid[1], np.float32)
    if len(y) != gny or len(x) != gnx:
        raise _lib.DimensionMismatch("node coordinates do not match the predictor grid")
    ysp = float(y[1] - y[0]) if gny > 1 else 1.0
    xsp = float(x[1] - x[0]) if gnx > 1 else 1.0
    return float(y[0]), ysp, float(x[0]), xsp


def to_planes(P):
    """(gny, gnx, 2) field -> the library layout: u then v, column-major planes."""
    P = np.asarray(P, np.float32)
    return np.concatenate([P[..., 0].ravel(order="F"), P[..., 1].ravel(order="F")])


def from_planes(flat, gny, gnx):
    G = gny * gnx
    out = np.empty((gny, gnx, 2), np.float32)
    out[..., 0] = np.reshape(flat[:G], (gny, gnx), order="F")
    out[..., 1] = np.reshape(flat[G:], (gny, gnx), order="F")
    return out


class NCCLoss:
    """The correlation loss of one image pair: the pair is staged and
    prefiltered once; every evaluation deforms, correlates and (optionally)
    back-propagates on the device."""

    def __init__(self, A, B, *, window=16, overlap=8, workspace=None):
        self.window = int(window)
        self.overlap = int(overlap)
        self._own = workspace is None
        self.ws = workspace if workspace is not None else PIVWorkspace()
        A = _lib.as_f32_colmajor(A)
        B = _lib.as_f32_colmajor(B)
        if A.shape != B.shape:
            raise _lib.DimensionMismatch(f"images must have the same size, got {A.shape} and {B.shape}")
        self.shape = A.shape
        _lib.check(_lib.lib().hh_stage_pair(self.ws.ctx, _lib.fptr(A), _lib.fptr(B), A.shape[0], A.shape[1]),
                   self.ws.ctx)

    def _call(self, Pptr, gny, gnx, grid, gptr, device):
        y0, ysp, x0, xsp = grid
        loss = ctypes.c_double()
        st = _lib.lib().hh_ncc_loss_grad(self.ws.ctx, Pptr, gny, gnx, y0, ysp, x0, xsp, self.window, self.overlap,
                                         int(device), ctypes.byref(loss), gptr)
        _lib.check(st, self.ws.ctx)
        return loss.value

    def value(self, P, grid):
        gny, gnx = P.shape[0], P.shape[1]
        flat = to_planes(P)
        return self._call(flat.ctypes.data, gny, gnx, _grid(grid, gny, gnx), None, False)

    def value_and_grad(self, P, grid):
        """(L, dL/dP) with dL/dP shaped like P."""
        gny, gnx = P.shape[0], P.shape[1]
        flat = to_planes(P)
        g = np.empty_like(flat)
        L = self._call(flat.ctypes.data, gny, gnx, _grid(grid, gny, gnx), g.ctypes.data, False)
        return L, from_planes(g, gny, gnx)

    def device_value_and_grad(self, Pdev, gny, gnx, grid, gdev=None):
        """Device form: Pdev and gdev are float32 CUDA tensors of 2*gny*gnx
        elements in the library layout (u then v, column-major planes)."""
        if not (_is_device_tensor(Pdev) and Pdev.is_contiguous() and Pdev.numel() == 2 * gny * gnx):
            raise _lib.ArgumentError("device predictor must be a contiguous CUDA tensor of 2*gny*gnx floats")
        gptr = None if gdev is None else gdev.data_ptr()
        return self._call(Pdev.data_ptr(), gny, gnx, _grid(grid, gny, gnx), gptr, True)

    def close(self):
        if self._own and self.ws is not None:
            self.ws.close()
        self.ws = None


def ncc_loss_function():
    """A torch.autograd.Function over NCCLoss: forward(P, loss_obj, grid)
    returns L as a 0-d tensor, backward scales the adjoint gradient (the
    rrule of the loss). P: CUDA tensor (2, gnx, gny) in the library layout."""
    import torch

    class _NCC(torch.autograd.Function):
        @staticmethod
        def forward(ctx, P, loss_obj, grid):
            P = P.detach().contiguous()
            gny, gnx = P.shape[2], P.shape[1]
            g = torch.empty_like(P)
            L = loss_obj.device_value_and_grad(P, gny, gnx, grid, g)
            ctx.save_for_backward(g)
            return torch.tensor(L, dtype=torch.float64, device=P.device)

        @staticmethod
        def backward(ctx, dL):
            (g,) = ctx.saved_tensors
            return (dL.to(g.dtype) * g, None, None)

    return _NCC
