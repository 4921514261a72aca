"""CPU tests: the oracle, the host-side spectral path of the library, the
C ABI surface.  No GPU is used."""
import ctypes
import os
import re

import numpy as np
import pytest

import vlr_b200 as V
from oracle import ref, lbvh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference host build (oracle/_ref) not built")


def _lib():
    L = V.lib()
    L.vlrbUpsampleSpectrum.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_void_p]
    L.vlrbEvaluateSpectrum.argtypes = [ctypes.c_void_p] * 3
    L.vlrbCmfStrata.argtypes = [ctypes.c_void_p] * 2
    return L


def header_functions():
    names = []
    for h in ("vlr/vlr.h", "vlrb.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^(?:VLRResult|const char\*)\s+(vlr\w+)\(", text, re.M)
    return names


def test_library_exports_every_declared_symbol():
    L = V.lib()
    names = header_functions()
    assert len(names) >= 95
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_reference_header_functions_all_present():
    # every entry point of the reference C API has a declaration here
    ref_names = ["vlrGetErrorMessage", "vlrCreateContext", "vlrDestroyContext", "vlrContextRender",
                 "vlrTriangleMeshSurfaceNodeAddMaterialGroup", "vlrSceneSetEnvironmentRotation",
                 "vlrQueryableSetImmediateSpectrum", "vlrCameraCreate", "vlrParentNodeGetChildAt"]
    names = set(header_functions())
    for n in ref_names:
        assert n in names
    assert len([n for n in names if n.startswith("vlr") and not n.startswith("vlrb")]) == 87


def test_error_messages_and_enums():
    L = V.lib()
    L.vlrGetErrorMessage.restype = ctypes.c_char_p
    assert L.vlrGetErrorMessage(0) == b"No Error"
    assert L.vlrGetErrorMessage(3) == b"Invalid Argument"
    n = ctypes.c_uint32()
    assert L.vlrGetNumEnumMembers(b"ColorSpace", ctypes.byref(n)) == 0 and n.value == 4
    v = ctypes.c_char_p()
    assert L.vlrGetEnumMember(b"ColorSpace", 1, ctypes.byref(v)) == 0 and v.value == b"Rec709(D65)"
    assert L.vlrGetEnumMember(b"ColorSpace", 9, ctypes.byref(v)) == V.INVALID_ARGUMENT
    assert L.vlrGetNumEnumMembers(b"NoSuchEnum", ctypes.byref(n)) == V.INVALID_ARGUMENT


def test_null_handles_are_invalid_argument():
    L = V.lib()
    L.vlrDestroyContext.argtypes = [ctypes.c_void_p]
    assert L.vlrDestroyContext(None) == V.INVALID_ARGUMENT
    L.vlrContextBindOutputBuffer.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    assert L.vlrContextBindOutputBuffer(None, 4, 4, 0) == V.INVALID_ARGUMENT


@needs_ref
def test_generated_tables_match_reference_build():
    L = _lib()
    grid, pts, cmf, integral = ref.tables()
    xyz = np.zeros(48, np.float32)
    integ = ctypes.c_float()
    assert L.vlrbCmfStrata(xyz.ctypes.data_as(ctypes.c_void_p), ctypes.byref(integ)) == 0
    assert np.array_equal(xyz.reshape(3, 16), cmf)
    assert integ.value == np.float32(integral)


@needs_ref
def test_upsampling_bit_exact_against_reference():
    L = _lib()
    rng = np.random.default_rng(5)
    cases = [(0, 1, *rng.uniform(0, 1, 3)) for _ in range(600)]
    cases += [(1, 1, *rng.uniform(0, 20, 3)) for _ in range(200)]
    cases += [(2, 1, x, x, x) for x in rng.uniform(1.0, 2.0, 100)]
    cases += [(0, 0, *rng.uniform(0, 1, 3)) for _ in range(200)]   # sRGB gamma
    cases += [(0, 1, 0.0, 0.0, 0.0), (1, 1, 15.0, 15.0, 15.0), (0, 1, 1.0, 0.0, 0.0), (0, 1, 0.0, 1.0, 0.0),
              (0, 1, 0.0, 0.0, 1.0), (0, 1, 1.0, 1.0, 1.0)]
    lam = np.array([395.25, 512.75, 630.25, 747.75], np.float32)
    out = np.zeros(3, np.uint32)
    vals = np.zeros(4, np.float32)
    for st, cs, a, b, c in cases:
        r = np.array(ref.upsample(st, cs, a, b, c), np.uint32)
        assert L.vlrbUpsampleSpectrum(st, cs, a, b, c, out.ctypes.data_as(ctypes.c_void_p)) == 0
        assert np.array_equal(out, r), (st, cs, a, b, c)
        assert L.vlrbEvaluateSpectrum(out.ctypes.data_as(ctypes.c_void_p), lam.ctypes.data_as(ctypes.c_void_p),
                                      vals.ctypes.data_as(ctypes.c_void_p)) == 0
        rv = np.zeros(4, np.float32)
        ref.lib().vlrref_eval_upsampled(r.ctypes.data_as(ctypes.c_void_p), lam.ctypes.data_as(ctypes.c_void_p),
                                        rv.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(vals, rv)


def test_tabulated_material_spectra_match_evaluate():
    """Material colours as the renderers evaluate them (tabulated once on the
    95-sample grid, then interpolated) against the reference's evaluate
    order (interpolate each table point, then weight): equal to float
    rounding, at random wavelengths including the grid ends."""
    L = _lib()
    L.vlrbEvaluateSpectrumTabulated.argtypes = [ctypes.c_void_p] * 3
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rng = np.random.default_rng(9)
    packed = np.zeros(3, np.uint32)
    a = np.zeros(4, np.float32)
    b = np.zeros(4, np.float32)
    worst = 0.0
    for k in range(400):
        st = (0, 1, 2)[k % 3]
        rgb = rng.uniform(0, 1, 3) if st == 0 else (rng.uniform(0, 20, 3) if st == 1 else np.full(3, rng.uniform(1, 2)))
        assert L.vlrbUpsampleSpectrum(st, 1, *map(float, rgb), P(packed)) == 0
        lam = rng.uniform(360.0, 830.0, 4).astype(np.float32)
        if k % 50 == 0:
            lam[:2] = (360.0, 830.0)
        assert L.vlrbEvaluateSpectrum(P(packed), P(lam), P(a)) == 0
        assert L.vlrbEvaluateSpectrumTabulated(P(packed), P(lam), P(b)) == 0
        scale = max(np.abs(a).max(), 1e-30)
        worst = max(worst, float(np.abs(a - b).max() / scale))
    assert worst < 1e-5, worst


@needs_ref
def test_oracle_bsdf_self_consistency():
    """The reference BSDFs: evaluatePDF at the sampled direction reproduces
    the sampled pdf for the non-delta materials (materials.cu sample vs
    evaluatePDF), a property the GPU parity test inherits."""
    inp = V.make_bsdf_batch_inputs(20000, seed=11)
    out = ref.bsdf_batch(inp)
    m = inp["material"]
    ok = out["pdf"] > 0
    # Matte, GGX conductor, Lambertian, UE4.  The GGX dielectric is left out:
    # its evaluatePDF rebuilds the transmission half vector from the hero
    # wavelength and returns 0 whenever that vector faces away from the view
    # direction (materials.cu:1434-1442), so it does not invert its sampler.
    nondelta = ok & np.isin(m, [0, 2, 4, 5])
    rel = np.abs(out["evalPdf"][nondelta] - out["pdf"][nondelta]) / out["pdf"][nondelta]
    assert np.quantile(rel, 0.99) < 1e-3
    # delta reflection evaluates to zero off the sampled direction
    assert np.all(out["evalValue"][ok & (m == 1)] == 0)


def test_lbvh_oracle_structure():
    rng = np.random.default_rng(3)
    n = 5000
    v = (rng.uniform(-1, 1, (n, 1, 3)) + rng.normal(0, 0.02, (n, 3, 3))).astype(np.float32).reshape(n, 9)
    codes, prims, ch, boxes = lbvh.build_lbvh(v)
    assert np.all(np.diff(codes.astype(np.int64)) >= 0)
    assert sorted(prims.tolist()) == list(range(n))
    leaves = sorted((~c) for c in ch if c < 0)
    assert leaves == list(range(n))
    internal = sorted(c for c in ch if c >= 0)
    assert internal == list(range(1, n - 1))
    # root box contains every triangle
    tri = v.reshape(n, 3, 3)
    assert np.all(boxes[0:3] <= tri.min(axis=(0, 1))) and np.all(boxes[3:6] >= tri.max(axis=(0, 1)))


def _sah(ch, boxes, v, prims):
    """SAH cost (1.2 per node area, 1.0 per triangle box area) over the root area."""
    n = len(prims)
    tri = v.reshape(n, 3, 3)[prims]
    tlo, thi = tri.min(axis=1), tri.max(axis=1)
    area = lambda lo, hi: 2 * ((hi - lo)[..., 0] * (hi - lo)[..., 1] + (hi - lo)[..., 1] * (hi - lo)[..., 2]
                               + (hi - lo)[..., 2] * (hi - lo)[..., 0])
    b = boxes.reshape(-1, 6).astype(np.float64)
    return (1.2 * area(b[:, :3], b[:, 3:]).sum() + area(tlo, thi).sum()) / area(b[0, :3], b[0, 3:])


def _closest_hits(v, prims, ch, boxes, rays):
    """Closest hit per ray by walking every box the ray meets (no ordering)."""
    n = len(prims)
    tri = v.reshape(n, 3, 3).astype(np.float64)
    b = boxes.reshape(-1, 6).astype(np.float64)
    out = []
    for o, d in rays:
        inv = 1.0 / d
        best, hit = np.inf, -1
        stack = [0]
        while stack:
            x = stack.pop()
            for c in (ch[2 * x], ch[2 * x + 1]):
                if c >= 0:
                    t0, t1 = (b[c, :3] - o) * inv, (b[c, 3:] - o) * inv
                    if max(np.minimum(t0, t1).max(), 0.0) <= min(np.maximum(t0, t1).min(), best):
                        stack.append(c)
                else:
                    a, p1, p2 = tri[prims[~c]]
                    e1, e2 = p1 - a, p2 - a
                    p = np.cross(d, e2)
                    det = e1 @ p
                    if det == 0:
                        continue
                    s = o - a
                    u = (s @ p) / det
                    q = np.cross(s, e1)
                    w = (d @ q) / det
                    t = (e2 @ q) / det
                    if u >= 0 and w >= 0 and u + w <= 1 and 0 < t < best:
                        best, hit = t, int(prims[~c])
        out.append(hit)
    return out


def test_treelet_oracle_keeps_the_tree_valid_and_lowers_its_sah_cost():
    """Treelet restructuring (host restatement): still a binary tree over the
    same leaves, every node box the union of its children's, a lower SAH cost,
    and the same closest hits as the LBVH it started from."""
    rng = np.random.default_rng(5)
    n = 3000
    scale = np.exp(rng.uniform(-4, 0, (n, 1, 1)))
    v = (rng.uniform(-1, 1, (n, 1, 3)) + 0.1 * scale * rng.normal(0, 1, (n, 3, 3))).astype(np.float32).reshape(n, 9)
    codes, prims, ch, boxes = lbvh.build_lbvh(v)
    och, obx, nr = lbvh.optimize_lbvh(v, prims, ch, boxes, 3)
    assert nr > 0
    assert sorted((~c) for c in och if c < 0) == list(range(n))
    assert sorted(c for c in och if c >= 0) == list(range(1, n - 1))
    tri = v.reshape(n, 3, 3)[prims]
    cb = lambda c: (obx[6 * c:6 * c + 3], obx[6 * c + 3:6 * c + 6]) if c >= 0 else \
        (tri[~c].min(axis=0), tri[~c].max(axis=0))
    for x in range(n - 1):
        (l0, h0), (l1, h1) = cb(och[2 * x]), cb(och[2 * x + 1])
        assert np.array_equal(obx[6 * x:6 * x + 3], np.minimum(l0, l1))
        assert np.array_equal(obx[6 * x + 3:6 * x + 6], np.maximum(h0, h1))
    assert np.array_equal(obx[:6], boxes[:6])
    before, after = _sah(ch, boxes, v, prims), _sah(och, obx, v, prims)
    assert after < 0.95 * before, (before, after)
    rays = []
    for _ in range(150):
        o = rng.uniform(-1.5, 1.5, 3)
        d = rng.normal(size=3)
        rays.append((o, d / np.linalg.norm(d)))
    assert _closest_hits(v, prims, ch, boxes, rays) == _closest_hits(v, prims, och, obx, rays)
    # a second call on the same input gives the same tree
    och2, obx2, nr2 = lbvh.optimize_lbvh(v, prims, ch, boxes, 3)
    assert np.array_equal(och, och2) and np.array_equal(obx, obx2) and nr == nr2


@needs_ref
def test_seed_states_match_mt19937_64_recurrence():
    """The oracle's per-pixel RNG seeds (std::mt19937_64 of the host build,
    context.cpp:1176-1190) equal the published 64-bit Mersenne Twister
    recurrence, including across the 312-word state refills."""
    for seed in (591842031321323413, 1, 0x9E3779B97F4A7C15):
        assert np.array_equal(ref.seed_states(1000, seed), ref.seed_states_py(1000, seed))


def _max_leaf_depth(ch):
    """Internal nodes on the deepest root-to-leaf path."""
    n1 = len(ch) // 2
    if n1 == 0:
        return 0
    depth = np.zeros(n1, np.int64)
    best = 0
    order = [0]
    for x in order:                       # breadth first: parents before children
        for c in (ch[2 * x], ch[2 * x + 1]):
            if c >= 0:
                depth[c] = depth[x] + 1
                order.append(c)
            else:
                best = max(best, depth[x] + 1)
    return best


def test_lbvh_depth_stays_within_the_traversal_stack():
    """The traversal keeps one stack entry per tree level (64 entries).  In
    the Karras hierarchy every level splits at a longer common prefix of the
    30-bit Morton code extended by the index, so a path has at most
    30 + ceil(log2 n) internal nodes.  Inputs that reach for that bound:
    centroids spaced by powers of two (one new Morton bit per level), each
    repeated 64 times (index tie-break levels below), near-equal centroids,
    and a uniform cloud.  The restructured trees of the same inputs stay
    within the stack too (the build falls back to the plain LBVH when one
    would not)."""
    rng = np.random.default_rng(11)
    pts = np.array([[2.0 ** -i, 2.0 ** -j, 2.0 ** -k] for i in range(11) for j in range(0, 11, 5)
                    for k in range(0, 11, 5)])
    cases = [pts, np.repeat(pts, 64, axis=0), np.zeros((4096, 3)), rng.uniform(-1, 1, (20000, 3))]
    for c in cases:
        n = len(c)
        v = (c[:, None, :] + 1e-4 * rng.normal(size=(n, 3, 3))).astype(np.float32).reshape(n, 9)
        codes, prims, ch, boxes = lbvh.build_lbvh(v)
        d = _max_leaf_depth(ch)
        assert d <= 30 + int(np.ceil(np.log2(n))) and d <= 64, (n, d)
        och, obx, _ = lbvh.optimize_lbvh(v, prims, ch, boxes, 3)
        assert _max_leaf_depth(och) <= 64


@needs_ref
def test_fp64_film_against_the_reference_fp32_kahan_film():
    """The same contributions summed three ways by the CPU path tracer:
    FP64 (the CUDA renderers' film), the reference's own FP32 SpectrumStorage
    (Kahan pairs per stratum) and a plain FP32 sum.  On the Cornell box at
    1024 spp the Kahan film stays within 2e-7 of FP64 per stratum and the
    plain FP32 sum drifts further; at 512x512 and 4096 spp the figures are
    1.1e-7 and 4.1e-6 (python -m oracle.film_precision)."""
    from vlr_b200 import scenes
    W = H = 32
    desc = scenes.cornell_box_desc(W, H)
    f64, kahan, plain, _ = ref.pt_render_fp32_films(scenes.flatten_desc(desc), desc["camera"], W, H, 1024, 8)
    lit = f64 > 0
    k_err = np.abs(kahan.astype(np.float64) - f64)[lit] / f64[lit]
    p_err = np.abs(plain.astype(np.float64) - f64)[lit] / f64[lit]
    assert k_err.max() < 2e-7, k_err.max()
    assert p_err.max() > k_err.max()


@pytest.mark.skipif(not ref.available64(), reason="FP64 oracle (oracle/_ref/libvlrref64.so) not built")
def test_fp64_oracle_is_the_reference_algorithm_in_double():
    """The FP64 oracle runs the reference's own BSDF code in double: on every
    BSDF its results differ from the FP32 build's (it is not the FP32 code)
    by FP32 rounding only, a median norm-wise difference below 1e-4 per
    output, and it samples the same lobes (the same zero/non-zero pattern)."""
    import vlr_b200 as V
    inp = V.make_bsdf_batch_inputs(1 << 15, seed=77, materials=7)
    r32, r64 = ref.bsdf_batch(inp), ref.bsdf_batch64(inp)
    mat = inp["material"]
    assert np.any(r32["value"].astype(np.float64) != r64["value"])
    for k in ("value", "pdf", "wi", "evalValue", "evalPdf"):
        a, b = r32[k].astype(np.float64), r64[k]
        a2, b2 = a.reshape(len(mat), -1), b.reshape(len(mat), -1)
        assert np.mean(np.any(a2 != 0, axis=1) == np.any(b2 != 0, axis=1)) > 0.999, k
        for m in range(7):
            sel = mat == m
            d = np.abs(a2[sel] - b2[sel]).max(axis=1) / np.maximum(np.abs(b2[sel]).max(axis=1), 1e-30)
            assert np.median(d) < 1e-4, (k, m, np.median(d))


def _point_lit_desc(W, H):
    """The Cornell box description with every material diffuse and the
    ceiling light turned into a plain Matte quad (the scene the point-light
    tests light with one point at (0, 2.4, 0))."""
    from vlr_b200 import scenes
    desc = scenes.cornell_box_desc(W, H)
    for m in ("metal", "glass"):
        desc["materials"][m] = ("Matte", {"albedo": ("Rec709(D65)", 0.5, 0.5, 0.5)})
    desc["materials"]["light"] = ("Matte", {"albedo": ("Rec709(D65)", 0.8, 0.8, 0.8)})
    return desc


BULB = np.array([[0.0, 2.4, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 0.0]], np.float32)


@needs_ref
def test_oracle_point_emitter_is_linear_in_its_intensity():
    """The oracle's point emitter (samplePoint, point.cu:38-80, with the
    reference's PointEDF, materials.cu:2194-2250): with the same seeds,
    doubling the PointEmitter's scale doubles every film value exactly, in
    the path tracer and in the LVC-BPT restatement (the light enters each
    path's contribution as one factor, and neither Russian roulette nor the
    MIS weights see it); without the point the box has no light at all."""
    from vlr_b200 import scenes
    W = H = 16
    desc = _point_lit_desc(W, H)
    flat = scenes.flatten_desc(desc)
    films, bfilms = [], []
    try:
        for scale in (1.0, 2.0):
            ref.points_set(BULB, 1, (4.0, 4.0, 4.0), scale)
            f, _, _ = ref.pt_render(flat, desc["camera"], W, H, 8, 6, rng_states=ref.seed_states(W * H))
            films.append(f)
            b, _, _, _ = ref.bpt_render(flat, desc["camera"], W, H, 8, 6, W * H)
            bfilms.append(b)
    finally:
        ref.points_set(None)
    assert np.isfinite(films[0]).all() and films[0].sum() > 0
    assert np.array_equal(films[1], 2 * films[0])
    assert bfilms[0].sum() > 0
    assert np.array_equal(bfilms[1], 2 * bfilms[0])
    dark, _, _ = ref.pt_render(flat, desc["camera"], W, H, 8, 6, rng_states=ref.seed_states(W * H))
    assert dark.sum() == 0.0


def _poster_desc(W, H, albedo=("Rec709(D65)", 0.5, 0.5, 0.5)):
    """The diffuse Cornell box with its back wall split off as a "poster"
    material (u left to right, v bottom to top across the wall)."""
    from vlr_b200 import scenes
    desc = scenes.cornell_box_desc(W, H)
    for m in ("metal", "glass"):
        desc["materials"][m] = ("Matte", {"albedo": ("Rec709(D65)", 0.5, 0.5, 0.5)})
    desc["materials"]["poster"] = ("Matte", {"albedo": albedo})
    mesh = desc["meshes"][0]
    verts = mesh["verts"].copy()
    verts[4:8, 9:11] = [[0, 0], [1, 0], [1, 1], [0, 1]]
    mesh["verts"] = verts
    groups = [(np.array([0, 1, 2, 0, 2, 3, 8, 9, 10, 8, 10, 11], np.uint32), "white"),
              (np.array([4, 5, 6, 4, 6, 7], np.uint32), "poster")]
    mesh["groups"] = groups + mesh["groups"][1:]
    return desc


@needs_ref
def test_oracle_texture_of_a_constant_is_the_immediate_colour():
    """The oracle's Image2DTexture albedo (shader_nodes.cu:410-445, the
    texture unit restated): a point-sampled texture holding the immediate
    linear colour everywhere gives the same film, bit for bit, with the same
    seeds; a black texture darkens the image (the poster reflects nothing);
    the LVC-BPT restatement refuses textures."""
    from vlr_b200 import scenes
    W = H = 16
    desc = _poster_desc(W, H)
    flat = scenes.flatten_desc(desc)
    poster = list(desc["materials"]).index("poster")
    films = []
    for value in (None, 0.5, 0.0):
        if value is not None:
            ref.texture_set(poster, np.full((3, 5, 4), value, np.float32), flat["uv"], nearest=True)
        try:
            f, _, _ = ref.pt_render(flat, desc["camera"], W, H, 8, 6, rng_states=ref.seed_states(W * H))
            if value == 0.0:
                with pytest.raises(AssertionError):
                    ref.bpt_render(flat, desc["camera"], W, H, 1, 6, W * H)
        finally:
            ref.texture_set()
        films.append(f)
    assert np.array_equal(films[0], films[1])
    assert films[2].sum() < films[0].sum()


@needs_ref
def test_oracle_normal_map_of_the_vertex_normal_changes_nothing():
    """The oracle's normal map (shader_nodes.cu:349-391 with
    applyBumpMapping, renderer_common.h:554-576): a map that stores the
    untilted normal (0, 0, 1) leaves the film unchanged bit for bit (the
    bump is skipped when the mapped normal has no tangential part), while a
    tilted one changes it; the LVC-BPT restatement refuses normal maps."""
    from vlr_b200 import scenes
    W = H = 16
    desc = scenes.floor_desc(W, H)
    flat = scenes.flatten_desc(desc)
    films = []
    for n in (None, (0.0, 0.0, 1.0), (0.3, 0.4, np.sqrt(0.75))):
        if n is not None:
            rgba = np.ones((2, 2, 4), np.float32)
            rgba[..., :3] = (np.array(n) + 1) / 2
            ref.normal_map_set(0, rgba, flat["uv"], nearest=True, coeff=17 / 16)
        try:
            f, _, _ = ref.pt_render(flat, desc["camera"], W, H, 8, 4, rng_states=ref.seed_states(W * H))
            if n is not None and n[0] != 0.0:
                with pytest.raises(AssertionError):
                    ref.bpt_render(flat, desc["camera"], W, H, 1, 4, W * H)
        finally:
            ref.normal_map_set()
        films.append(f)
    assert films[0].sum() > 0
    assert np.array_equal(films[0], films[1])
    assert not np.array_equal(films[0], films[2])


@needs_ref
def test_oracle_alpha_map_limits():
    """The oracle's alpha map: with a clear sheet (alpha 0) the film is bit
    for bit that of the scene without the sheet; an opaque one (alpha 1)
    takes all the light (the floor is lit only through the black sheet);
    the LVC-BPT restatement refuses alpha maps."""
    from vlr_b200 import scenes
    W = H = 16
    desc = scenes.floor_desc(W, H, light_at=(0.0, 0.0), sheet=True)
    flat = scenes.flatten_desc(desc)
    bare_desc = scenes.floor_desc(W, H, light_at=(0.0, 0.0))
    bare, _, _ = ref.pt_render(scenes.flatten_desc(bare_desc), bare_desc["camera"], W, H, 8, 4,
                               rng_states=ref.seed_states(W * H))
    films = []
    for a in (0.0, 1.0):
        rgba = np.zeros((2, 2, 4), np.float32)
        rgba[..., 3] = a
        ref.alpha_map_set(2, rgba, flat["uv"], channel=3)
        try:
            f, _, _ = ref.pt_render(flat, desc["camera"], W, H, 8, 4, rng_states=ref.seed_states(W * H))
            with pytest.raises(AssertionError):
                ref.bpt_render(flat, desc["camera"], W, H, 1, 4, W * H)
        finally:
            ref.alpha_map_set()
        films.append(f)
    assert bare.sum() > 0
    assert np.array_equal(films[0], bare)
    assert films[1].sum() == 0.0


@needs_ref
def test_oracle_multi_material_of_two_mattes_is_their_sum():
    """The oracle's Multi material (the reference's MultiBSDF,
    materials.cu:2255-2532, restated over its BSDF classes): a Multi of grey
    Mattes 0.3 and 0.4 samples the same cosine direction from the same
    numbers as one Matte 0.7, with the summed value (Meng spectra of one
    chromaticity scale with brightness) and the blended density of two equal
    pdfs, so the film matches Matte 0.7's with the same seeds to float
    round-off; the LVC-BPT restatement refuses Multi materials."""
    from vlr_b200 import scenes
    W = H = 16
    desc = scenes.floor_desc(W, H, light_at=(0.6, 0.0))
    desc["materials"]["floor"] = ("Matte", {"albedo": ("Rec709(D65)", 0.7, 0.7, 0.7)})
    desc["materials"]["sub0"] = ("Matte", {"albedo": ("Rec709(D65)", 0.3, 0.3, 0.3)})
    desc["materials"]["sub1"] = ("Matte", {"albedo": ("Rec709(D65)", 0.4, 0.4, 0.4)})
    flat = scenes.flatten_desc(desc)
    names = list(desc["materials"])
    single, _, _ = ref.pt_render(flat, desc["camera"], W, H, 16, 4, rng_states=ref.seed_states(W * H))
    ref.multi_set(names.index("floor"), [names.index("sub0"), names.index("sub1")])
    try:
        multi, _, _ = ref.pt_render(flat, desc["camera"], W, H, 16, 4, rng_states=ref.seed_states(W * H))
        with pytest.raises(AssertionError):
            ref.bpt_render(flat, desc["camera"], W, H, 1, 4, W * H)
    finally:
        ref.multi_set()
    assert single.sum() > 0
    assert np.allclose(multi, single, rtol=1e-5, atol=1e-6 * single.max())


@needs_ref
def test_oracle_directional_emitter_reaches_only_light_subpaths():
    """The oracle's directional emitter (the reference's DirectionalEDF,
    materials.cu:2100-2160: a delta direction, zero evaluation): the path
    tracer restatement gets no light from it, the LVC-BPT restatement's
    light subpaths leave it along its normal and light the box."""
    from vlr_b200 import scenes
    W = H = 16
    desc = _point_lit_desc(W, H)
    desc["materials"]["light"] = ("DirectionalEmitter", {"emittance": ("Rec709(D65)", 5.0, 5.0, 5.0)})
    flat = scenes.flatten_desc(desc)
    pt, _, _ = ref.pt_render(flat, desc["camera"], W, H, 8, 6, rng_states=ref.seed_states(W * H))
    bpt, _, _, _ = ref.bpt_render(flat, desc["camera"], W, H, 8, 6, W * H)
    assert pt.sum() == 0.0
    assert np.isfinite(bpt).all() and bpt.sum() > 0


@needs_ref
def test_oracle_light_tracer_matches_oracle_path_tracer():
    """The CPU restatement of light_tracing.cu and that of path_tracing.cu
    estimate the same image: on the diffuse Cornell box the totals agree
    within 1.5% (1024 frames of 32 x 32 light subpaths against 1024 spp)."""
    from vlr_b200 import scenes
    W = H = 32
    desc = _point_lit_desc(W, H)
    desc["materials"]["light"] = scenes.cornell_box_desc(W, H)["materials"]["light"]
    flat = scenes.flatten_desc(desc)
    pt, _, _ = ref.pt_render(flat, desc["camera"], W, H, 1024, 8)
    lt, _, _ = ref.lt_render(flat, desc["camera"], W, H, 1024, 8, W * H)
    assert pt.sum() > 0
    assert abs(lt.sum() / pt.sum() - 1) < 0.015, lt.sum() / pt.sum()


@needs_ref
def test_oracle_bilinear_weights_reproduce_the_measured_texture_unit():
    """The oracle's model of the texture unit's bilinear weights, against
    fetches measured on a B200 (a linear fetch of a 2 x 2 texture whose
    texels are the four unit vectors returns the weights): the fractions in
    8 fractional bits rounded to nearest, ties up, the far corner's weight
    rounded from their product, the other three completing 256ths.
    Measured cases, fractions in 256ths and weights in 256ths of (near,
    x-neighbour, y-neighbour, far): (127.5, 128.5) -> (64, 63, 64, 65);
    (63.5, 129.5) -> (95, 31, 97, 33); (10.5, 10.5) -> (234, 11, 11, 0);
    (200.5, 77.5) -> (38, 140, 17, 61); (0.5, 255.5) -> (0, 0, 255, 1).
    Every model weight is a multiple of 1/256 and the four sum to 1."""
    L = ref.lib()
    L.vlrref_bilinear_weights.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_void_p]
    out = np.zeros(4, np.float32)

    def w(fa, fb):
        L.vlrref_bilinear_weights(fa / 256, fb / 256, out.ctypes.data_as(ctypes.c_void_p))
        return tuple(int(x) for x in np.round(out * 256))

    assert w(127.5, 128.5) == (64, 63, 64, 65)
    assert w(63.5, 129.5) == (95, 31, 97, 33)
    assert w(10.5, 10.5) == (234, 11, 11, 0)
    assert w(200.5, 77.5) == (38, 140, 17, 61)
    assert w(0.5, 255.5) == (0, 0, 255, 1)
    rng = np.random.default_rng(5)
    for fa, fb in rng.uniform(0, 1, (500, 2)).astype(np.float32):
        L.vlrref_bilinear_weights(float(fa), float(fb), out.ctypes.data_as(ctypes.c_void_p))
        q = out * 256
        assert np.all(q == np.round(q)) and q.sum() == 256 and np.all(q >= 0)
