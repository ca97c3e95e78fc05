"""The allocation-free entry point against the allocating one.

hh_field_change_noalloc serves callers that cannot let the library allocate
device memory (memory owned by the caller's own pool allocator, loops that
cannot absorb an allocation stall, fixed memory budgets). It works on
caller-owned device buffers with scratch compiled into the library. This
test calls it twice in a row through the C ABI and checks each result
against hh_field_change on the same data. It runs last (file name) so a
failure here leaves every other test already run, and it passes both alone
in a fresh process and after the rest of the suite.
"""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _field(rng, n):
    u = rng.standard_normal(n).astype(np.float32)
    v = rng.standard_normal(n).astype(np.float32)
    pu = (u + 0.02 * rng.standard_normal(n)).astype(np.float32)
    pv = (v + 0.02 * rng.standard_normal(n)).astype(np.float32)
    u[1] = np.nan          # NaN transition: counts as an infinite change
    u[2] = pu[2] = np.nan  # NaN in both sweeps: skipped
    mask = (rng.uniform(size=n) < 0.05).astype(np.uint8)
    return u, v, pu, pv, mask


def test_field_change_noalloc_matches_allocating_entry_point(hb, ws):
    import torch

    from hammerhead_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(2024)
    out = torch.empty(1, dtype=torch.float32, device=dev)
    for call, n in enumerate((16129, 50000)):  # two calls in a row, the second larger
        u, v, pu, pv, mask = _field(rng, n)
        ref = ctypes.c_float()
        _lib.check(L.hh_field_change(ws.ctx, _lib.fptr(u), _lib.fptr(v), _lib.fptr(pu), _lib.fptr(pv),
                                     _lib.u8ptr(mask), n, ctypes.byref(ref)), ws.ctx)
        d = [torch.from_numpy(a).to(dev) for a in (u, v, pu, pv, mask)]
        st = L.hh_field_change_noalloc(*[ctypes.c_void_p(t.data_ptr()) for t in d], n,
                                       ctypes.c_void_p(out.data_ptr()), None)
        assert st == 0, L.hh_noalloc_last_error().decode()
        torch.cuda.synchronize()
        got = float(out.item())
        assert math.isfinite(got) and math.isfinite(ref.value)
        assert abs(got - ref.value) <= 1e-6 * abs(ref.value), (call, got, ref.value)


def test_field_change_noalloc_rejects_oversize(hb):
    from hammerhead_b200 import _lib

    L = _lib.lib()
    st = L.hh_field_change_noalloc(None, None, None, None, None, (1 << 20) + 1, ctypes.c_void_p(8), None)
    assert st == _lib.HH_ERR_ARG
    assert b"exceed" in L.hh_noalloc_last_error()


def _case(rng, n, kind):
    u, v, pu, pv, mask = _field(rng, max(n, 3))
    u, v, pu, pv, mask = u[:n], v[:n], pu[:n], pv[:n], mask[:n]
    if kind == "no_mask":
        mask = None
    elif kind == "all_masked":
        mask = np.ones(n, np.uint8)
    elif kind == "many_nan":  # more than 5 % infinite changes: the percentile lands on +Inf
        sel = rng.uniform(size=n) < 0.08
        u[sel] = np.nan
    return u, v, pu, pv, mask


@pytest.mark.parametrize("n,kind", [(1 << 20, "masked"), (0, "masked"), (40000, "all_masked"),
                                    (40000, "no_mask"), (40000, "many_nan")],
                         ids=["max_size", "empty", "all_masked", "no_mask", "many_nan"])
def test_field_change_noalloc_edge_cases(hb, ws, n, kind):
    """The limit size, an empty field, every vector masked, no mask, and a
    field whose 95th percentile is an infinite change: each equals the
    allocating entry point, on two calls in a row."""
    import torch

    from hammerhead_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(n + len(kind))
    out = torch.full((1,), -1.0, dtype=torch.float32, device=dev)
    u, v, pu, pv, mask = _case(rng, n, kind)
    ref = ctypes.c_float()
    _lib.check(L.hh_field_change(ws.ctx, _lib.fptr(u), _lib.fptr(v), _lib.fptr(pu), _lib.fptr(pv),
                                 _lib.u8ptr(mask), n, ctypes.byref(ref)), ws.ctx)
    d = [torch.from_numpy(a).to(dev) if a is not None and n > 0 else None for a in (u, v, pu, pv, mask)]
    ptrs = [ctypes.c_void_p(t.data_ptr()) if t is not None else None for t in d]
    for _ in range(2):
        st = L.hh_field_change_noalloc(*ptrs, n, ctypes.c_void_p(out.data_ptr()), None)
        assert st == 0, L.hh_noalloc_last_error().decode()
        assert L.hh_noalloc_last_error() == b""
        torch.cuda.synchronize()
        got = float(out.item())
        if math.isinf(ref.value):
            assert got == ref.value
        else:
            assert abs(got - ref.value) <= 1e-6 * abs(ref.value), (got, ref.value)
