"""Batched rendering of several contexts through one captured CUDA graph,
and the launch-configuration autotuner."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _y(film):
    import ctypes
    import vlr_b200 as V
    L = V.lib()
    L.vlrbCmfStrata.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    xyz = np.zeros(48, np.float32)
    integ = ctypes.c_float()
    assert L.vlrbCmfStrata(xyz.ctypes.data_as(ctypes.c_void_p), ctypes.byref(integ)) == 0
    return np.einsum("hwk,k->hw", film, xyz[16:32].astype(np.float64))


def _ctx(W, H, glass="box", light_scale=1.0, guided=False):
    from vlr_b200 import vlr as VV, scenes
    ctx = VV.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.cornell_box(ctx, W, H, glass=glass, light_scale=light_scale)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=8, max_paths_in_flight=W * H * 2)
    if guided:
        ctx.setGuiding(enabled=True, train=True, log2TableSize=14, samplesPerStep=1 << 14, warmupLaunches=2)
    return ctx, cam, keep


def test_batch_graph_replays_match_individual_renders():
    """Three plain contexts of different sizes rendered as one graph: each
    replay restarts accumulation (firstFrame) and must equal, up to the order
    of the FP64 film atomics, the same renders issued one context at a time
    (same RNG streams: the batch's warm-up render advances them exactly like
    the first individual render)."""
    from vlr_b200 import vlr as VV
    sizes = [(48, 32, 4), (64, 64, 2), (96, 40, 6)]
    ref = []
    for W, H, spp in sizes:
        ctx, cam, keep = _ctx(W, H)
        ctx.render_samples(cam, True, spp)           # matches the batch warm-up
        for _ in range(3):
            ctx.render_samples(cam, True, spp)
        ref.append(ctx.read_film())
        ctx.close()
    ctxs = [_ctx(W, H) for W, H, _ in sizes]
    batch = VV.RenderBatch([(c, cam, spp, True) for (c, cam, _), (_, _, spp) in zip(ctxs, sizes)])
    for _ in range(3):
        batch.launch()
    times = batch.item_times()
    assert all(t > 0 for t in times)
    for (c, cam, _), r in zip(ctxs, ref):
        f = c.read_film()
        assert np.allclose(f, r, rtol=1e-9, atol=1e-12)
        img = c.read_output()
        assert np.isfinite(img).all() and img[..., :3].mean() > 0
    batch.close()
    for c, _, _ in ctxs:
        c.close()


def test_batch_with_guided_items_trains_and_stays_unbiased():
    """A guided item inside the graph keeps training (the launch stamp and
    sample counters live on the device) and renders the same mean as a plain
    item of the same scene."""
    from vlr_b200 import vlr as VV
    plain, pcam, k1 = _ctx(64, 64)
    guided, gcam, k2 = _ctx(64, 64, guided=True)
    batch = VV.RenderBatch([(plain, pcam, 8, False), (guided, gcam, 8, False)])
    steps0 = guided.guiding_stats()["trainingSteps"]
    for _ in range(64):
        batch.launch()
    batch.item_times()
    st = guided.guiding_stats()
    assert np.isfinite(st["lastLoss"])
    yp = _y(plain.read_film())
    yg = _y(guided.read_film())
    assert abs(yg.sum() / yp.sum() - 1) < 0.03, yg.sum() / yp.sum()
    assert steps0 >= 1
    batch.close()
    plain.close()
    guided.close()


def test_autotune_keeps_the_fastest_configuration():
    ctx, cam, keep = _ctx(128, 128)
    trials = ctx.autotune(cam, samples_per_trial=8)
    assert len(trials) >= 4
    best = max(trials, key=lambda t: t[2])
    o = ctx.options()
    assert (o["maxPathsInFlight"], o["blocksPerSM"]) == best[:2]
    assert all(t[2] > 0 for t in trials)
    # rendering with the tuned options still works
    ctx.render_samples(cam, True, 4)
    assert np.isfinite(ctx.read_output()).all()
    ctx.close()
