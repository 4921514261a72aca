"""The environment-light part of the oracle on CPU: its two importance maps
(the CUDA build's full-resolution FP64 map and the reference's own 4x
smaller FP32 one) give the same image mean, and the error the FP64 CDF
removes, measured as texels an FP32 CDF can never sample."""
import numpy as np
import pytest

from oracle import ref, triangle

needs_ref = pytest.mark.skipif(not ref.available(), reason="reference host build (oracle/_ref) not built")


def _y(film):
    _, _, cmf, _ = ref.tables()
    return np.einsum("hwk,k->hw", film, cmf[1].astype(np.float64))


@needs_ref
def test_both_importance_maps_estimate_the_same_image():
    from vlr_b200 import scenes
    W, H = 24, 14
    d = scenes.terrain_scene_desc(W, H, cells=8, n_spheres=3, seed=3, sky=(128, 64))
    flat = scenes.flatten_instanced_desc(d)
    means = []
    for mode in (0, 1):
        ref.env_set(d["env"], mode=mode)
        try:
            f, _, _ = ref.pt_render(flat, d["camera"], W, H, 96, 4, rng_states=ref.seed_states(W * H, 99 + mode))
        finally:
            ref.env_set(None)
        y = _y(f)
        assert np.isfinite(y).all()
        means.append(y.mean())
    assert abs(means[1] / means[0] - 1) < 0.03, means


@needs_ref
def test_fp32_cdf_loses_texels_the_fp64_cdf_keeps():
    """On the terrain workload's 2048x1024 sky (sun at 1e4 times the zenith)
    no positive texel falls below an FP32 CDF step, in the reference's 4x
    smaller map or at full resolution: the FP64 CDF removes no sampling
    error there.  With a brighter sun sharing rows with dim sky (a texel at
    the half-precision limit in every row of a dim sky), the FP32 CDF after
    that texel no longer resolves the dim texels: they are never sampled,
    while the FP64 CDF keeps every one."""
    from vlr_b200 import scenes
    ref.env_set({"image": scenes.sky_image(2048, 1024), "scale": 1.0}, mode=0)
    c = ref.env_unsampleable()
    assert c["positive_full"] == 2048 * 1024 and c["fp64_full"] == 0 and c["fp32_full"] == 0
    assert c["fp32_quarter"] == 0
    img = np.zeros((64, 2048, 4), np.float32)
    img[..., 0:3] = 1e-3
    img[:, 100, 0:3] = 2e4
    img[..., 3] = 1
    ref.env_set({"image": img, "scale": 1.0}, mode=0)
    c = ref.env_unsampleable()
    ref.env_set(None)
    assert c["fp64_full"] == 0
    assert c["fp32_full"] > 0.25 * c["positive_full"], c      # 51,126 of 131,072 here


@needs_ref
def test_oracle_hierarchy_finds_the_brute_force_hits():
    """Scenes above 4,096 triangles are intersected through the oracle's own
    median-split hierarchy: its closest hits for the camera rays of a terrain
    scene (8,192 + 960 triangles) are the brute-force search's with the same
    watertight triangle test (oracle/triangle.py), wherever the closest t is
    unique."""
    from vlr_b200 import scenes
    W, H = 32, 18
    d = scenes.terrain_scene_desc(W, H, cells=64, n_spheres=3, seed=5, sky=(64, 32))
    flat = scenes.flatten_instanced_desc(d)
    assert len(flat["tris"]) > 4096
    ref.env_set(d["env"])
    try:
        _, _, rays = ref.pt_camera_rays(flat, d["camera"], W, H, 1)
    finally:
        ref.env_set(None)
    prim = rays[:, 3].view(np.uint32)
    q = rays.copy()
    q[:, 3] = np.float32(3.4e38)
    tri = flat["pos"][flat["tris"][:, 0:3]].astype(np.float32)
    _, best, unique = triangle.closest_hits(tri, q)
    assert unique.mean() > 0.99
    assert np.array_equal(best[unique], prim[unique])
