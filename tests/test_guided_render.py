"""Guided path tracing through the C API: unbiased against plain path
tracing, and lower error than plain path tracing at equal sample count on
the glossy-caustic scene once the network has trained."""
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


def test_trained_guiding_lowers_error_on_glossy_caustic():
    """What the network gains: on the glossy-caustic scene (GGX dielectric
    sphere, light at 0.1x area) the guided tracer, after 64 training
    launches, has a lower error at equal sample count than plain path
    tracing.  Error: RMSE of 4x4-pixel block means of CIE Y against an 8192
    spp plain reference (its own RNG seed), relative to the reference mean.
    All renders use the dielectric pdf consistent with its value: with the
    reference's pdf, NEE through the sphere's exits is double counted and
    its unsuppressed fireflies dominate every error."""
    W = H = 96
    ref, _ = _render(W, H, 8192, glass="sphere", light_scale=0.1, paths=1 << 20, seed=0x9E3779B97F4A7C15)
    plain, _ = _render(W, H, 256, glass="sphere", light_scale=0.1)
    guided, st = _render(W, H, 256, glass="sphere", light_scale=0.1, guided=True, pretrain=64, paths=W * H)
    assert st["trainingSteps"] == 64 + 256

    def err(img):
        b = 4
        a = img.reshape(H // b, b, W // b, b).mean(axis=(1, 3))
        r = ref.reshape(H // b, b, W // b, b).mean(axis=(1, 3))
        return np.sqrt(np.mean((a - r) ** 2)) / r.mean()

    e_plain, e_guided = err(plain), err(guided)
    print("relative block RMSE plain", e_plain, "guided", e_guided)
    assert abs(guided.sum() / ref.sum() - 1) < 0.03
    assert e_guided < 0.85 * e_plain, (e_plain, e_guided)


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
