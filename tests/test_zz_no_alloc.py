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
