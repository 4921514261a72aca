"""Guided path tracing through the C API: unbiased against plain path
tracing, and what the trained network learns in a scene lit only
indirectly."""
import ctypes

import numpy as np
import pytest

import vlr_b200 as V

pytestmark = pytest.mark.gpu


def _y(film):
    L = V.lib()
    L.vlrbCmfStrata.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    xyz = np.zeros(48, np.float32)
    integ = ctypes.c_float()
    assert L.vlrbCmfStrata(xyz.ctypes.data_as(ctypes.c_void_p), ctypes.byref(integ)) == 0
    return np.einsum("hwk,k->hw", film, xyz[16:32].astype(np.float64))


def _render(W, H, spp, glass="box", light_scale=1.0, guided=False, pretrain=0, paths=1 << 16, seed=0,
            consistent=True):
    from vlr_b200 import vlr as VV, scenes
    ctx = VV.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.cornell_box(ctx, W, H, glass=glass, light_scale=light_scale)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=8, max_paths_in_flight=paths, rng_seed=seed,
                   consistent_dielectric_pdf=consistent)
    if guided:
        ctx.setGuiding(enabled=True, train=True, log2TableSize=16, samplesPerStep=1 << 14, warmupLaunches=4)
    if pretrain:
        ctx.render_samples(cam, True, pretrain)
    ctx.render_samples(cam, True, spp)
    y = _y(ctx.read_film()) / spp
    gst = ctx.guiding_stats() if guided else None
    ctx.close()
    return y, gst


def _block_z(g, c, b=8):
    H, W = g.shape
    gb = g.reshape(H // b, b, W // b, b).sum(axis=(1, 3))
    cb = c.reshape(H // b, b, W // b, b).sum(axis=(1, 3))
    sg = g.reshape(H // b, b, W // b, b).std(axis=(1, 3)) * b
    sc = c.reshape(H // b, b, W // b, b).std(axis=(1, 3)) * b
    lit = cb > 1e-3 * cb.max()
    return np.abs(gb - cb)[lit] / np.sqrt(sg[lit] ** 2 + sc[lit] ** 2 + (1e-3 * cb[lit]) ** 2)


def test_guided_path_tracing_is_unbiased():
    """Guided sampling with online training (one-sample MIS with the BSDF)
    converges to the plain estimator's mean on the Cornell box: whole image
    within 2%, 8x8 blocks within 6 combined standard errors."""
    W = H = 64
    plain, _ = _render(W, H, 1024)
    guided, st = _render(W, H, 1024, guided=True)
    assert st["trainingSteps"] > 0 and st["guidedLaunches"] > 0
    assert np.isfinite(st["lastLoss"])
    assert np.isfinite(guided).all()
    assert abs(guided.sum() / plain.sum() - 1) < 0.02, guided.sum() / plain.sum()
    assert np.all(_block_z(guided, plain) < 6)


def test_trained_network_concentrates_on_the_indirect_light():
    """What the network gains over BSDF sampling alone.  In the Cornell box
    lit only indirectly (the light faces the ceiling, so the floor sees no
    light but the bright ceiling patch above it), the network trained online
    by the renderer puts at least 3x the cosine density in the direction of
    that patch at floor points; guided rendering keeps the plain mean (one
    sample MIS with the BSDF)."""
    from vlr_b200 import vlr as VV, scenes
    from oracle import guide_ref as G
    W = H = 96
    ctx = VV.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.cornell_box(ctx, W, H, light_up=True)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=8, max_paths_in_flight=W * H)
    ctx.setGuiding(enabled=True, train=True, log2TableSize=16, samplesPerStep=1 << 14, warmupLaunches=4)
    ctx.render_samples(cam, True, 128)
    net = ctx.guide_net()
    pts = np.array([[x, 0.0, z] for x in (-1.0, 0.0, 1.0) for z in (-1.0, 0.0, 1.0)], np.float32)
    wo = np.array([0.0, 1.5, 6.0]) - pts
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    nrm = np.tile([0.0, 1.0, 0.0], (len(pts), 1)).astype(np.float32)
    raw = net.infer(pts, wo.astype(np.float32), nrm)
    net.close()
    patch = np.array([0.0, 3.0, 0.0]) - pts
    patch /= np.linalg.norm(patch, axis=1, keepdims=True)
    q = G.mixture_pdf(raw.astype(np.float64), patch)
    cosine = patch[:, 1] / np.pi
    assert np.median(q / cosine) >= 3.0, q / cosine
    ctx.render_samples(cam, True, 256)
    guided = _y(ctx.read_film()) / 256
    ctx.close()
    plain, _ = _render_indirect(W, H, 256)
    assert abs(guided.sum() / plain.sum() - 1) < 0.03, guided.sum() / plain.sum()


def _render_indirect(W, H, spp):
    from vlr_b200 import vlr as VV, scenes
    ctx = VV.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = scenes.cornell_box(ctx, W, H, light_up=True)
    ctx.setScene(scene)
    ctx.setOptions(max_path_length=8, rng_seed=12345)
    ctx.render_samples(cam, True, spp)
    y = _y(ctx.read_film()) / spp
    ctx.close()
    return y, None


def test_consistent_dielectric_pdf_agrees_with_bidirectional():
    """With the consistent dielectric pdf, path tracing and LVC-BPT (both
    unbiased then) agree on the glossy-caustic scene: whole image within 3%."""
    from vlr_b200 import vlr as VV, scenes
    W = H = 64
    means = []
    for renderer in (VV.RENDERER_PATH_TRACING, VV.RENDERER_BPT):
        ctx = VV.Context()
        ctx.bindOutputBuffer(W, H)
        scene, cam, keep = scenes.cornell_box(ctx, W, H, glass="sphere", light_scale=0.1)
        ctx.setScene(scene)
        ctx.setRenderer(renderer)
        ctx.setOptions(max_path_length=8, consistent_dielectric_pdf=True)
        ctx.render_samples(cam, True, 4096)
        means.append(_y(ctx.read_film()).mean())
        ctx.close()
    assert abs(means[1] / means[0] - 1) < 0.03, means
