"""Batched schedule (hh_run_batched) against the per-pair schedule.

The batched form runs the same per-window and per-cell device code as
run_piv, only over every pair of a pass slot at once, with convergence
decided on the device; so each pair's result must equal run_piv on that pair
bit for bit (the property run_piv_sequence states for the reference,
src/io.jl:225-228), for uneven pair sizes, mixed schedules, masks, early
convergence, device-resident inputs, and graph replay.
"""
import numpy as np
import pytest

FIELDS = ("u", "v", "peak_ratio", "correlation_moment", "uncertainty_u", "uncertainty_v")

pytestmark = pytest.mark.gpu


def _same(a, b):
    for k in FIELDS:
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape, k
        assert np.array_equal(x, y, equal_nan=True), (k, np.nanmax(np.abs(x - y)))
    assert np.array_equal(a.outliers, b.outliers)
    assert np.array_equal(a.mask, b.mask)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


def _mixed(hb, n=6, seed=7):
    syn = hb.synthetic
    shapes = [(256, 256), (192, 320), (320, 256), (256, 384), (128, 192), (384, 384)]
    pairs, flows = [], []
    for i in range(n):
        flow = syn.sine_shear_flow(1.5 + i * 0.7, 160.0 + 40 * i) if i % 2 == 0 else syn.uniform_flow(2.3 - i, 1.1 + 0.4 * i)
        A, B = syn.particle_pair(shapes[i % len(shapes)], flow, seed=seed + i)
        pairs.append((A, B))
        flows.append(flow)
    return pairs, flows


def _schedules(hb):
    s1 = hb.multipass_parameters([64, 32, 16], padding=True, apodization="gauss",
                                 final=dict(max_iterations=3, uncertainty=True))
    s2 = hb.multipass_parameters([48, 24], padding=True, apodization="gauss",
                                 final=dict(max_iterations=3, uncertainty=True))
    return s1, s2


def test_batch_equals_per_pair_mixed(hb, ws):
    pairs, flows = _mixed(hb)
    s1, s2 = _schedules(hb)
    sched = [s1 if i % 2 == 0 else s2 for i in range(len(pairs))]
    res = hb.run_piv_batch(pairs, sched, workspace=ws)
    assert len(res) == len(pairs)
    for (A, B), s, r, flow in zip(pairs, sched, res, flows):
        ref = hb.run_piv(A, B, s, workspace=ws)
        _same(r, ref)
        assert r.sweeps[-1] == ref.sweeps[-1]
        assert hb.rms_error(r, flow) < 0.1


def test_batch_graph_replay_and_direct(hb, ws):
    pairs, _ = _mixed(hb, n=4, seed=31)
    s1, s2 = _schedules(hb)
    sched = [s1, s2, s2, s1]
    runner = hb.BatchRunner(pairs, sched, workspace=ws, graph=True)
    first = runner.run().results()
    again = runner.run().results()      # graph replay
    for a, b in zip(first, again):
        _same(a, b)
    direct = hb.run_piv_batch(pairs, sched, workspace=ws, graph=False)
    for a, b in zip(first, direct):
        _same(a, b)
    runner.close()


def test_batch_new_images_same_shape(hb, ws):
    # a replayed graph reads the image pointers from the descriptor tables,
    # so new contents (and new arrays) of the same shapes are analysed
    s1, s2 = _schedules(hb)
    p1, _ = _mixed(hb, n=3, seed=101)
    p2, _ = _mixed(hb, n=3, seed=202)
    hb.run_piv_batch(p1, [s1, s2, s1], workspace=ws)
    res = hb.run_piv_batch(p2, [s1, s2, s1], workspace=ws)
    for (A, B), s, r in zip(p2, [s1, s2, s1], res):
        _same(r, hb.run_piv(A, B, s, workspace=ws))


def test_batch_masks(hb, ws):
    pairs, _ = _mixed(hb, n=3, seed=55)
    s1, s2 = _schedules(hb)
    masks = []
    for i, (A, _) in enumerate(pairs):
        if i == 1:
            masks.append(None)
            continue
        m = np.zeros(A.shape, bool)
        r0, c0 = A.shape[0] // 3, A.shape[1] // 4
        m[r0:r0 + 60, c0:c0 + 70] = True
        masks.append(m)
    sched = [s1, s2, s2]
    res = hb.run_piv_batch(pairs, sched, masks=masks, workspace=ws)
    for (A, B), s, m, r in zip(pairs, sched, masks, res):
        ref = hb.run_piv(A, B, s, mask=m, workspace=ws)
        _same(r, ref)
    assert res[0].mask.any() and not res[1].mask.any()


def test_batch_convergence_on_device(hb, ws):
    # convergence_tol large enough that some pairs stop after 2 sweeps while
    # others run all 4: the device-side test must reproduce each pair's count
    pairs, _ = _mixed(hb, n=6, seed=77)
    sched = hb.multipass_parameters([32, 16], padding=True, final=dict(max_iterations=4, convergence_tol=0.02))
    res = hb.run_piv_batch(pairs, sched, workspace=ws)
    counts = []
    for (A, B), r in zip(pairs, res):
        ref = hb.run_piv(A, B, sched, workspace=ws)
        _same(r, ref)
        assert r.sweeps[-1] == ref.sweeps[-1]
        counts.append(int(ref.sweeps[-1]))
    assert min(counts) >= 2


def test_batch_options_split_classes(hb, ws):
    # schedules differing in correlation method, peak finder, n_peaks,
    # validators and uncertainty run as separate job classes of one slot
    pairs, _ = _mixed(hb, n=4, seed=303)
    a = [hb.PIVParameters(window_size=32, overlap=16, correlation_method="phase", n_peaks=1),
         hb.PIVParameters(window_size=16, overlap=8, peak_finder="exclusion", n_peaks=3, uncertainty=True,
                          validation=(hb.PeakRatioValidator(1.2), hb.VelocityMagnitudeValidator(0.0, 12.0)))]
    b = [hb.PIVParameters(window_size=32, overlap=16, subpixel_method="gauss9", replace_outliers=False,
                          max_iterations=2, uncertainty=True)]
    c = [hb.PIVParameters(window_size=24, overlap=12, padding=True, min_peak_ratio=1.1)]
    sched = [a, b, c, a]
    res = hb.run_piv_batch(pairs, sched, workspace=ws)
    for (A, B), s, r in zip(pairs, sched, res):
        _same(r, hb.run_piv(A, B, s, workspace=ws))


def test_batch_device_inputs(hb, ws):
    import torch

    pairs, _ = _mixed(hb, n=3, seed=404)
    s1, s2 = _schedules(hb)
    dev = [(torch.from_numpy(np.ascontiguousarray(A.T)).cuda().T, torch.from_numpy(np.ascontiguousarray(B.T)).cuda().T)
           for A, B in pairs]
    r_dev = hb.run_piv_batch(dev, [s1, s2, s1], workspace=ws)
    r_host = hb.run_piv_batch(pairs, [s1, s2, s1], workspace=ws)
    for a, b in zip(r_dev, r_host):
        _same(a, b)


def test_batch_launch_count(hb, ws):
    # one launch per kernel per slot and sweep for the whole batch: the count
    # does not grow with the number of pairs
    from hammerhead_b200 import _lib

    s1, s2 = _schedules(hb)
    L = _lib.lib()
    counts = []
    for n in (2, 6):
        pairs, _ = _mixed(hb, n=n, seed=500)
        r = hb.BatchRunner(pairs, [s1 if i % 2 == 0 else s2 for i in range(n)], workspace=ws)
        r.run()
        c0 = L.hh_launch_count(ws.ctx)
        r.run()
        counts.append(L.hh_launch_count(ws.ctx) - c0)
        r.close()
    assert counts[0] == counts[1] and counts[0] < 200


def test_batch_uint16_frames(hb, ws):
    # 12-bit counts in UInt16 are converted on the device: normalised (x/65535)
    # equals the float32 path on the same values, raw equals x itself
    import torch

    syn = hb.synthetic
    s1, s2 = _schedules(hb)
    pairs16 = []
    for i, shape in enumerate([(256, 256), (192, 320)]):
        A, B = syn.particle_pair(shape, syn.uniform_flow(1.7, -0.9), seed=60 + i)
        pairs16.append((syn.to_uint16_12bit(A), syn.to_uint16_12bit(B)))
    sched = [s1, s2]
    res16 = hb.run_piv_batch(pairs16, sched, workspace=ws)
    as_f = [(a.astype(np.float32) / np.float32(65535), b.astype(np.float32) / np.float32(65535)) for a, b in pairs16]
    resf = hb.run_piv_batch(as_f, sched, workspace=ws)
    for a, b in zip(res16, resf):
        _same(a, b)
    runner = hb.BatchRunner(pairs16, sched, workspace=ws, u16="raw")
    rr = runner.run().results()
    runner.close()
    resr = hb.run_piv_batch([(a.astype(np.float32), b.astype(np.float32)) for a, b in pairs16], sched, workspace=ws)
    for a, b in zip(rr, resr):
        _same(a, b)
    # device-resident UInt16 frames
    dev = [(torch.from_numpy(np.ascontiguousarray(a.T)).cuda().T, torch.from_numpy(np.ascontiguousarray(b.T)).cuda().T)
           for a, b in pairs16]
    for a, b in zip(hb.run_piv_batch(dev, sched, workspace=ws), res16):
        _same(a, b)


def test_sequence_pipelined_equals_batch(hb, ws):
    syn = hb.synthetic
    s1, _ = _schedules(hb)
    pairs = [tuple(syn.to_uint16_12bit(x) for x in syn.particle_pair((256, 256), syn.sine_shear_flow(2.0, 180.0),
                                                                     seed=80 + i)) for i in range(7)]
    seen = []
    seq = hb.run_piv_sequence(pairs, s1, batch_size=3, workspace=ws, on_result=lambda i, r: seen.append(i))
    assert seen == list(range(1, 8))
    ref = hb.run_piv_batch(pairs, s1, workspace=ws)
    for a, b in zip(seq, ref):
        _same(a, b)
    unpiped = hb.run_piv_sequence(pairs, s1, batch_size=3, workspace=ws, pipeline=False)
    for a, b in zip(unpiped, ref):
        _same(a, b)


def test_batch_stream_equals_batch(hb, ws):
    # a stream of three batches of the same composition (mixed sizes and
    # schedules); batch k+1 is copied in while batch k is analysed. Frames
    # of the second batch sit in page-locked memory (copied directly), the
    # others in pageable numpy arrays (staged)
    import torch

    s1, s2 = _schedules(hb)
    sched = [s1, s2, s2, s1]
    batches = [_mixed(hb, n=4, seed=600 + 10 * k)[0] for k in range(3)]
    pinned = []
    for A, B in batches[1]:
        pa = torch.from_numpy(np.ascontiguousarray(A.T)).pin_memory().numpy().T
        pb = torch.from_numpy(np.ascontiguousarray(B.T)).pin_memory().numpy().T
        pinned.append((pa, pb))
    seen = []
    out = hb.run_piv_batch_stream([batches[0], pinned, batches[2]], sched, workspace=ws,
                                  on_batch=lambda k, r: seen.append(k))
    assert seen == [0, 1, 2] and len(out) == 3
    for k in range(3):
        ref = hb.run_piv_batch(batches[k], sched, workspace=ws)
        for a, b in zip(out[k], ref):
            _same(a, b)


def test_batch_stream_long_async(hb, ws):
    # seven batches of new images: the stream queues each run without a host
    # wait (HH_BATCH_ASYNC), so runs, copies and the plan's two upload
    # staging sets are reused several times while earlier runs are still
    # queued; every batch must still equal its own batch call bit for bit
    s1, s2 = _schedules(hb)
    sched = [s1, s2, s2]
    batches = [_mixed(hb, n=3, seed=1100 + 10 * k)[0] for k in range(7)]
    out = hb.run_piv_batch_stream(batches, sched, workspace=ws)
    assert len(out) == 7
    for k in range(7):
        for a, b in zip(out[k], hb.run_piv_batch(batches[k], sched, workspace=ws)):
            _same(a, b)


def test_batch_runner_async_run(hb, ws):
    # run(wait=False) returns with the run queued; after a wait on the
    # workspace's stream the results equal a synchronous run's
    import torch

    s1, s2 = _schedules(hb)
    pairs = _mixed(hb, n=4, seed=1200)[0]
    sync_res = hb.run_piv_batch(pairs, [s1, s2, s1, s2], workspace=ws)
    runner = hb.BatchRunner(pairs, [s1, s2, s1, s2], workspace=ws)
    runner.run(wait=False)
    torch.cuda.ExternalStream(ws.stream(), device=torch.device("cuda", ws.device)).synchronize()
    for a, b in zip(runner.results(copy=True), sync_res):
        _same(a, b)
    assert list(runner.sweeps) == [r.sweeps[-1] for r in sync_res]


def test_batch_stream_uint16(hb, ws):
    # UInt16 frames keep their pixel type on the device and are converted
    # there, in a stream exactly as in one batch call
    syn = hb.synthetic
    s1, s2 = _schedules(hb)
    batches = []
    for k in range(2):
        b = []
        for i, shape in enumerate([(256, 256), (192, 320)]):
            A, B = syn.particle_pair(shape, syn.uniform_flow(1.3 + k, -0.7), seed=900 + 10 * k + i)
            b.append((syn.to_uint16_12bit(A), syn.to_uint16_12bit(B)))
        batches.append(b)
    out = hb.run_piv_batch_stream(batches, [s1, s2], workspace=ws)
    for k in range(2):
        for a, b in zip(out[k], hb.run_piv_batch(batches[k], [s1, s2], workspace=ws)):
            _same(a, b)


def test_batch_stream_session_reused(hb, ws):
    # a second stream of the same composition on the same workspace reuses
    # the first call's device frames and prepared runners, with the same
    # results; another composition gets its own session
    s1, s2 = _schedules(hb)
    sched = [s1, s2, s2, s1]
    batches = [_mixed(hb, n=4, seed=700 + 10 * k)[0] for k in range(2)]
    ws.__dict__.pop("_stream_sessions", None)
    a = hb.run_piv_batch_stream(batches, sched, workspace=ws)
    assert len(ws._stream_sessions) == 1
    runners = next(iter(ws._stream_sessions.values()))["runners"]
    b = hb.run_piv_batch_stream(batches[::-1], sched, workspace=ws)
    assert next(iter(ws._stream_sessions.values()))["runners"] is runners
    for k in range(2):
        for x, y in zip(a[k], b[1 - k]):
            _same(x, y)
    hb.run_piv_batch_stream([batches[0][:3]], sched[:3], workspace=ws)
    assert len(ws._stream_sessions) == 2


def test_pipelined_paths_with_static_masks(hb, ws):
    # one mask per pair, the same in every batch: copied to the device once
    # and used by both pipelined paths exactly as by a batch call
    s1, s2 = _schedules(hb)
    sched = [s1, s2, s2, s1]
    batches = [_mixed(hb, n=4, seed=800 + 10 * k)[0] for k in range(2)]
    masks = []
    for j, (A, _) in enumerate(batches[0]):
        if j == 1:
            masks.append(None)
            continue
        m = np.zeros(A.shape, bool)
        m[: A.shape[0] // 3, A.shape[1] // 2:] = True
        masks.append(m)
    out = hb.run_piv_batch_stream(batches, sched, masks=masks, workspace=ws)
    for k in range(2):
        ref = hb.run_piv_batch(batches[k], sched, masks=masks, workspace=ws)
        for a, b in zip(out[k], ref):
            _same(a, b)
        assert out[k][0].mask.any() and not out[k][1].mask.any()
    # the sequence driver pipelines a single mask for every pair
    syn = hb.synthetic
    pairs = [syn.particle_pair((256, 256), syn.sine_shear_flow(2.0, 180.0), seed=90 + i) for i in range(5)]
    m = np.zeros((256, 256), bool)
    m[100:160, 40:120] = True
    piped = hb.run_piv_sequence(pairs, s1, batch_size=2, mask=m, workspace=ws)
    plain = hb.run_piv_sequence(pairs, s1, batch_size=2, mask=m, workspace=ws, pipeline=False)
    for a, b in zip(piped, plain):
        _same(a, b)
    assert piped[0].mask.any()
    with pytest.raises(hb.DimensionMismatch):
        hb.run_piv_batch_stream(batches, sched, masks=masks[:3], workspace=ws)


def test_batch_stream_error_leaves_session_usable(hb, ws):
    # a batch whose pair changed size raises DimensionMismatch; the cached
    # session of the composition stays usable for the next stream
    s1, s2 = _schedules(hb)
    sched = [s1, s2, s2, s1]
    good = [_mixed(hb, n=4, seed=900 + 10 * k)[0] for k in range(2)]
    bad = list(good[1])
    bad[2] = (bad[2][0][:-8], bad[2][1][:-8])
    with pytest.raises(hb.DimensionMismatch):
        hb.run_piv_batch_stream([good[0], bad, good[1]], sched, workspace=ws)
    out = hb.run_piv_batch_stream(good, sched, workspace=ws)
    for k in range(2):
        for a, b in zip(out[k], hb.run_piv_batch(good[k], sched, workspace=ws)):
            _same(a, b)


def test_allocation_failure_leaves_context_usable(hb, ws):
    """An injected device-allocation failure (host side, hh_debug_fail_alloc)
    surfaces as HH_ERR_OOM; the context then runs the next call normally,
    with the same results as before."""
    L = hb._lib.lib()
    syn = hb.synthetic
    A, B = syn.particle_pair((256, 224), syn.sine_shear_flow(2.0, 160.0), seed=901)
    passes = hb.multipass_parameters([32, 16], padding=True, final=dict(max_iterations=2, uncertainty=True))
    w = hb.piv_workspace()
    try:
        ref = hb.run_piv(A, B, passes, workspace=ws)
        L.hh_debug_fail_alloc(w.ctx, 0)  # the first allocation of the fresh context fails
        with pytest.raises(hb.HammerheadError) as ei:
            hb.run_piv(A, B, passes, workspace=w)
        assert ei.value.status == hb._lib.HH_ERR_OOM
        again = hb.run_piv(A, B, passes, workspace=w)
        for k in ("u", "v", "uncertainty_u"):
            assert np.array_equal(getattr(again, k), getattr(ref, k), equal_nan=True), k
        # a failure inside a batched plan: the plan is released, the next call rebuilds it
        pairs = [(A, B), syn.particle_pair((192, 256), syn.uniform_flow(1.5, 0.5), seed=902)]
        runner = hb.BatchRunner(pairs, passes, workspace=w)
        try:
            L.hh_debug_fail_alloc(w.ctx, 3)
            with pytest.raises(hb.HammerheadError) as ei:
                runner.run()
            assert ei.value.status == hb._lib.HH_ERR_OOM
        finally:
            runner.close()
        L.hh_debug_fail_alloc(w.ctx, -1)
        res = hb.run_piv_batch(pairs, passes, workspace=w)
        assert np.array_equal(res[0].u, ref.u, equal_nan=True)
    finally:
        L.hh_debug_fail_alloc(w.ctx, -1)
        w.close()


def test_batch_splits_on_allocation_failure(hb, ws):
    """run_piv_batch falls back to half batches when the whole batch's plan
    cannot be allocated; the results equal the unsplit batch."""
    L = hb._lib.lib()
    syn = hb.synthetic
    pairs = [syn.particle_pair((192, 192), syn.uniform_flow(0.5 * i, -0.3 * i), seed=910 + i) for i in range(4)]
    passes = hb.multipass_parameters([32, 16], padding=True, final=dict(max_iterations=2))
    whole = hb.run_piv_batch(pairs, passes, workspace=ws)
    w = hb.piv_workspace()
    try:
        L.hh_debug_fail_alloc(w.ctx, 0)  # the first (whole-batch) plan fails; the halves succeed
        split = hb.run_piv_batch(pairs, passes, workspace=w)
        for a, b in zip(whole, split):
            assert np.array_equal(a.u, b.u, equal_nan=True) and np.array_equal(a.v, b.v, equal_nan=True)
            assert np.array_equal(a.outliers, b.outliers)
    finally:
        L.hh_debug_fail_alloc(w.ctx, -1)
        w.close()
