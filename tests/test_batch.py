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


def _env_ctx(W, H, seed=3):
    from vlr_b200 import vlr as VV, scenes
    d = scenes.terrain_scene_desc(W, H, cells=16, n_spheres=6, seed=seed, sky=(256, 128))
    d["camera"]["aspect"] = W / H
    ctx = VV.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.build_instanced(ctx, d)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=6, max_paths_in_flight=W * H)
    return ctx, cam, keep


def test_persistent_batch_renders_what_the_wavefront_renders():
    """The plain items of a persistent batch (one kernel launch for all of
    them) against the same contexts rendered by the wavefront path tracer at
    one sample per pixel per launch, after the same warm-up: each pixel's
    samples draw from its stream in the same order through the same shading
    steps, so the RNG state after the frame is identical on at least 99% of
    pixels (a pixel differs only where the two kernels' FMA contraction
    rounds a branch decision differently), the film of those pixels agrees
    within 1e-4 relative on 99.5% of them, and the totals within 1e-3.  Two
    Cornell boxes (GGX metal and glass) and a terrain under the sky."""
    from vlr_b200 import vlr as VV
    specs = [("cornell", 48, 32, 4), ("env", 64, 36, 3), ("cornell", 64, 64, 2)]

    def make(kind, W, H):
        if kind == "env":
            return _env_ctx(W, H)
        ctx, cam, keep = _ctx(W, H)
        ctx.setOptions(max_paths_in_flight=W * H)
        return ctx, cam, keep

    ref_films, ref_states = [], []
    for kind, W, H, spp in specs:
        ctx, cam, keep = make(kind, W, H)
        ctx.render_samples(cam, True, spp)           # the batch's warm-up render
        ctx.render_samples(cam, True, spp)
        ref_films.append(_y(ctx.read_film()))
        ref_states.append(ctx.read_pixel_rng_states())
        ctx.close()
    ctxs = [make(kind, W, H) for kind, W, H, _ in specs]
    batch = VV.RenderBatch([(c, cam, spp, True) for (c, cam, _), (_, _, _, spp) in zip(ctxs, specs)],
                           persistent=True)
    batch.launch()
    times = batch.item_times()
    assert all(t > 0 for t in times)
    for (c, cam, _), rf, rs, (_, W, H, spp) in zip(ctxs, ref_films, ref_states, specs):
        g = _y(c.read_film())
        gs = c.read_pixel_rng_states()
        same = (gs == rs).reshape(H, W)
        assert same.mean() >= 0.99, same.mean()
        rel = (np.abs(g - rf) / np.maximum(np.abs(rf), 1e-3 * rf.mean()))[same]
        assert np.mean(rel <= 1e-4) >= 0.995, np.mean(rel <= 1e-4)
        assert abs(g.sum() / rf.sum() - 1) < 1e-3, g.sum() / rf.sum()
        img = c.read_output()
        assert np.isfinite(img).all() and img[..., :3].mean() > 0
    batch.close()
    for c, _, _ in ctxs:
        c.close()


def test_persistent_batch_keeps_guided_items_and_orders_by_work():
    """A persistent batch with a guided item: the guided item keeps its own
    launches (and keeps training) beside the persistent kernel and renders the
    plain item's mean; replays accumulate when firstFrame is false; the
    persistent items finish in the order of their work (the smaller first)."""
    from vlr_b200 import vlr as VV
    small, scam, k0 = _ctx(32, 32)
    plain, pcam, k1 = _ctx(64, 64)
    guided, gcam, k2 = _ctx(64, 64, guided=True)
    batch = VV.RenderBatch([(plain, pcam, 8, False), (guided, gcam, 8, False), (small, scam, 1, False)],
                           persistent=True)
    for _ in range(32):
        batch.launch()
    t = batch.item_times()
    assert 0 < t[2] <= t[0]
    assert np.isfinite(guided.guiding_stats()["lastLoss"])
    yp = _y(plain.read_film())
    yg = _y(guided.read_film())
    assert abs(yg.sum() / yp.sum() - 1) < 0.03, yg.sum() / yp.sum()
    assert plain.stats()["frames"] >= 8 * 33
    batch.close()
    for c in (small, plain, guided):
        c.close()
