"""ctypes access to the reference's own host-compiled BSDF/spectral code
(oracle/_ref/libvlrref.so, built by oracle/build_ref.sh).
TEST INFRASTRUCTURE ONLY."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libvlrref.so")
_lib = None

BATCH_INPUTS = ("wo", "material", "roughness", "ior", "albedo", "metallic", "u", "wavelengthU")
BATCH_OUTPUTS = {"value": 4, "pdf": 1, "wi": 3, "evalValue": 4, "evalPdf": 1}


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(REF_LIB)
        _lib.vlrref_init()
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _camera_array(camera):
    """The restatements' camera record: position, orientation (x, y, z, w),
    aspect, sensitivity, fovy, lens radius, op distance, kind (0
    perspective, 1 equirectangular), h angle, v angle."""
    equi = camera.get("type", "Perspective") == "Equirectangular"
    return np.array(list(camera["position"]) + list(camera["orientation"]) +
                    [camera.get("aspect", 1.0), camera["sensitivity"], camera.get("fovy", 1.0),
                     0.0 if equi else camera["lens radius"], camera.get("op distance", 1.0),
                     1.0 if equi else 0.0, camera.get("h angle", 0.0), camera.get("v angle", 0.0)], np.float32)


def bsdf_batch(inputs, threads=0):
    """Run the reference BSDF classes over a batch (see vlrref_bsdf_batch)."""
    n = len(inputs["material"])
    ins = [np.ascontiguousarray(inputs[k]) for k in BATCH_INPUTS]
    outs = {k: np.zeros((n, c) if c > 1 else n, np.float32) for k, c in BATCH_OUTPUTS.items()}
    lib().vlrref_bsdf_batch(ctypes.c_int64(n), ctypes.c_int(threads), *[_p(a) for a in ins],
                            *[_p(outs[k]) for k in BATCH_OUTPUTS])
    return outs


REF64_LIB = os.path.join(HERE, "_ref", "libvlrref64.so")
_lib64 = None


def available64():
    return os.path.exists(REF64_LIB)


def bsdf_batch64(inputs, threads=0):
    """The same batch through the FP64 build of the reference's BSDF and
    spectral classes (oracle/ref_shim64.cpp: every float of the reference
    sources compiled as double; FP32 inputs widened exactly).  Returns
    float64 outputs."""
    global _lib64
    if _lib64 is None:
        _lib64 = ctypes.CDLL(REF64_LIB)
        _lib64.vlrref64_init()
    n = len(inputs["material"])
    ins = [np.ascontiguousarray(inputs[k]) for k in BATCH_INPUTS]
    outs = {k: np.zeros((n, c) if c > 1 else n, np.float64) for k, c in BATCH_OUTPUTS.items()}
    _lib64.vlrref64_bsdf_batch(ctypes.c_int64(n), ctypes.c_int(threads), *[_p(a) for a in ins],
                               *[_p(outs[k]) for k in BATCH_OUTPUTS])
    return outs


def upsample(sp_type, color_space, e0, e1, e2):
    out = (ctypes.c_uint32 * 3)()
    lib().vlrref_upsample(sp_type, color_space, ctypes.c_float(e0), ctypes.c_float(e1),
                          ctypes.c_float(e2), out)
    return tuple(out)


def tables():
    """(grid bytes [168*8], points float32 [186*99], cmf16 [3,16], integralCMF)."""
    g = ctypes.c_void_p()
    p = ctypes.c_void_p()
    c = ctypes.POINTER(ctypes.c_float)()
    integ = ctypes.c_float()
    lib().vlrref_tables(ctypes.byref(g), ctypes.byref(p), ctypes.byref(c), ctypes.byref(integ))
    grid = np.ctypeslib.as_array(ctypes.cast(g, ctypes.POINTER(ctypes.c_uint8)), (168 * 8,)).copy()
    pts = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_float)), (186 * 99,)).copy()
    cmf = np.ctypeslib.as_array(c, (48,)).copy().reshape(3, 16)
    return grid, pts, cmf, integ.value


def pt_render(flat, camera, width, height, spp, max_path_length, rng_states=None, film=None, threads=0):
    """Render with the CPU restatement of the reference path tracer
    (oracle/ref_pt.inc).  Returns (film [H,W,16] float64 sum, rng_states, segments)."""
    if rng_states is None:
        rng_states = seed_states(width * height)
    if film is None:
        film = np.zeros((height, width, 16), np.float64)
    cam = _camera_array(camera)
    seg = ctypes.c_uint64()
    rc = lib().vlrref_pt_render(
        _p(flat["pos"]), _p(flat["nrm"]), _p(flat["tan"]), ctypes.c_uint32(len(flat["pos"])),
        _p(flat["tris"]), ctypes.c_uint32(len(flat["tris"])), _p(flat["groupMaterial"]),
        _p(flat["groupLightInst"]), ctypes.c_uint32(len(flat["groupMaterial"])), _p(flat["mats"]),
        ctypes.c_uint32(len(flat["mats"])), _p(cam), ctypes.c_uint32(width), ctypes.c_uint32(height),
        ctypes.c_uint32(spp), ctypes.c_uint32(max_path_length), ctypes.c_int(threads), _p(rng_states), _p(film),
        ctypes.byref(seg))
    assert rc == 0
    return film, rng_states, seg.value


LIGHT_SEED = 459182033132123413


def bpt_render(flat, camera, width, height, frames, max_path_length, num_light_paths, state=None, film=None,
               threads=0):
    """Render `frames` LVC-BPT frames with the CPU restatement of the
    reference's lvc_bpt.cu (oracle/ref_bpt.inc); the environment of env_set
    applies.  state carries the eye RNG states (per pixel), the light RNG
    states (per light subpath, seeded from std::mt19937_64(459182033132123413)
    as the reference seeds them) and the per-frame wavelength generator's
    draws across calls.  Returns (film [H,W,16] float64 sum, state, segments,
    light vertices stored)."""
    if state is None:
        state = {"eye": seed_states(width * height), "light": seed_states(num_light_paths, LIGHT_SEED),
                 "wl": np.zeros(1, np.uint64)}
    if film is None:
        film = np.zeros((height, width, 16), np.float64)
    cam = _camera_array(camera)
    seg, nlv = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().vlrref_bpt_render(
        _p(flat["pos"]), _p(flat["nrm"]), _p(flat["tan"]), ctypes.c_uint32(len(flat["pos"])),
        _p(flat["tris"]), ctypes.c_uint32(len(flat["tris"])), _p(flat["groupMaterial"]),
        _p(flat["groupLightInst"]), ctypes.c_uint32(len(flat["groupMaterial"])), _p(flat["mats"]),
        ctypes.c_uint32(len(flat["mats"])), _p(cam), ctypes.c_uint32(width), ctypes.c_uint32(height),
        ctypes.c_uint32(frames), ctypes.c_uint32(max_path_length), ctypes.c_uint32(num_light_paths),
        ctypes.c_int(threads), _p(state["eye"]), _p(state["light"]), _p(state["wl"]), _p(film),
        ctypes.byref(seg), ctypes.byref(nlv))
    assert rc == 0
    return film, state, seg.value, nlv.value


def lt_render(flat, camera, width, height, frames, max_path_length, num_light_paths, light_states=None, film=None,
              threads=0):
    """Render `frames` light-tracing frames with the CPU restatement of the
    reference's light_tracing.cu (oracle/ref_bpt.inc): per frame
    num_light_paths light subpaths, each with its own hero wavelengths,
    splatting a lens connection from every vertex.  light_states: one PCG32
    state per light subpath (advanced in place).  Returns (film [H,W,16]
    float64 sum, light_states, segments)."""
    if light_states is None:
        light_states = seed_states(num_light_paths, LIGHT_SEED)
    if film is None:
        film = np.zeros((height, width, 16), np.float64)
    cam = _camera_array(camera)
    seg = ctypes.c_uint64()
    rc = lib().vlrref_lt_render(
        _p(flat["pos"]), _p(flat["nrm"]), _p(flat["tan"]), ctypes.c_uint32(len(flat["pos"])),
        _p(flat["tris"]), ctypes.c_uint32(len(flat["tris"])), _p(flat["groupMaterial"]),
        _p(flat["groupLightInst"]), ctypes.c_uint32(len(flat["groupMaterial"])), _p(flat["mats"]),
        ctypes.c_uint32(len(flat["mats"])), _p(cam), ctypes.c_uint32(width), ctypes.c_uint32(height),
        ctypes.c_uint32(frames), ctypes.c_uint32(max_path_length), ctypes.c_uint32(num_light_paths),
        ctypes.c_int(threads), _p(light_states), _p(film), ctypes.byref(seg))
    assert rc == 0
    return film, light_states, seg.value


def pt_camera_rays(flat, camera, width, height, max_path_length, rng_states=None):
    """One frame of one sample per pixel (as pt_render) that also returns each
    pixel's camera ray and its brute-force closest hit: (film, rng_states,
    rays [H*W, 8] = org xyz, prim bits, dir xyz, t)."""
    if rng_states is None:
        rng_states = seed_states(width * height)
    film = np.zeros((height, width, 16), np.float64)
    cam = _camera_array(camera)
    rays = np.zeros((width * height, 8), np.float32)
    rc = lib().vlrref_pt_camera_rays(
        _p(flat["pos"]), _p(flat["nrm"]), _p(flat["tan"]), ctypes.c_uint32(len(flat["pos"])),
        _p(flat["tris"]), ctypes.c_uint32(len(flat["tris"])), _p(flat["groupMaterial"]),
        _p(flat["groupLightInst"]), ctypes.c_uint32(len(flat["groupMaterial"])), _p(flat["mats"]),
        ctypes.c_uint32(len(flat["mats"])), _p(cam), ctypes.c_uint32(width), ctypes.c_uint32(height),
        ctypes.c_uint32(max_path_length), _p(rng_states), _p(film), _p(rays))
    assert rc == 0
    return film, rng_states, rays


def env_set(env=None, mode=0, tex_weight_rounding=0):
    """Environment light of the following pt_render calls: env = the
    description's {"image": HxWx4 float32, "scale", "rotation"} (None removes
    it); mode 0 samples the full-resolution FP64 importance map the CUDA
    build uses, mode 1 the reference's own 4x smaller FP32 map."""
    if env is None:
        lib().vlrref_env_set(0, None, 0, 0, None, ctypes.c_float(1.0), ctypes.c_float(0.0), 0, 0)
        return
    img = env.get("image")
    const = np.array(env.get("constant", (0.0, 0.0, 0.0)), np.float32)
    if img is not None:
        img = np.ascontiguousarray(img, np.float32)
        h, w = img.shape[:2]
        ptr = _p(img)
    else:
        h = w = 0
        ptr = None
    lib().vlrref_env_set(1, ptr, ctypes.c_uint32(w), ctypes.c_uint32(h), _p(const),
                         ctypes.c_float(env.get("scale", 1.0)), ctypes.c_float(env.get("rotation", 0.0)),
                         ctypes.c_int(mode), ctypes.c_int(tex_weight_rounding))


def points_set(points=None, color_space=1, intensity=(1.0, 1.0, 1.0), scale=1.0):
    """Point emitters of the following pt_render calls: one PointSurfaceNode
    with a PointEmitter material, its points an (n, 9) array of world-space
    position, normal and tangent; intensity in color space `color_space`
    (0 Rec709 sRGB gamma, 1 Rec709 linear, 2 XYZ, 3 xyY).  The node is the
    light instance after the meshes' instances.  None removes it."""
    if points is None:
        lib().vlrref_pt_set_points(None, ctypes.c_uint32(0), ctypes.c_int32(1), None, ctypes.c_float(1.0))
        return
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 9)
    inten = np.array(intensity, np.float32)
    lib().vlrref_pt_set_points(_p(pts), ctypes.c_uint32(len(pts)), ctypes.c_int32(color_space), _p(inten),
                               ctypes.c_float(scale))


def texture_set(material=-1, rgba=None, uv=None, nearest=False, color_space=1, weight_rounding=0, scalars=False):
    """Image2DTexture on the albedo of Matte material `material` (index in
    the flattened material records) for the following pt_render calls: an
    (h, w, 4) float image (row 0 at v = 0) in color space `color_space`,
    nearest or linear filtering, repeat wrapping, and the scene's per-vertex
    texture coordinates (flatten_desc's "uv").  weight_rounding: the
    linear filter's weights as the texture unit forms them (0, measured) or
    as FP32 products (2); shared with the environment texture.  scalars:
    the texture feeds the float3 plug of a UE4 material (occlusion,
    roughness, metallic) or a microfacet material (roughness, anisotropy,
    rotation) instead of a Matte's albedo.  material = -1 removes it."""
    if material < 0 or rgba is None:
        lib().vlrref_pt_set_texture(ctypes.c_int32(-1), None, ctypes.c_uint32(0), ctypes.c_uint32(0), 0,
                                    ctypes.c_int32(1), None, ctypes.c_uint32(0), ctypes.c_int(0), ctypes.c_int(0))
        return
    img = np.ascontiguousarray(rgba, np.float32)
    h, w = img.shape[:2]
    tc = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    lib().vlrref_pt_set_texture(ctypes.c_int32(material), _p(img), ctypes.c_uint32(w), ctypes.c_uint32(h),
                                ctypes.c_int(1 if nearest else 0), ctypes.c_int32(color_space), _p(tc),
                                ctypes.c_uint32(len(tc)), ctypes.c_int(weight_rounding),
                                ctypes.c_int(1 if scalars else 0))


def normal_map_set(group=-1, rgba=None, uv=None, nearest=False, directx=False, coeff=1.0, height=False, channel=0):
    """Normal map on geometry group `group` of the following pt_render
    calls: an Image2DTexture read through its xyz plug ((n + 1) / 2 per
    texel, DirectX or OpenGL convention) or, with height=True, a height map
    read through channel `channel` from the texture-gather footprint (repeat
    addressing); the bump coefficient as the kernels receive it and the
    scene's per-vertex texture coordinates.  group = -1 removes it."""
    if group < 0 or rgba is None:
        lib().vlrref_pt_set_normal_map(ctypes.c_int32(-1), None, ctypes.c_uint32(0), ctypes.c_uint32(0), 0, 0, 0,
                                       ctypes.c_float(1.0), None, ctypes.c_uint32(0))
        return
    img = np.ascontiguousarray(rgba, np.float32)
    h, w = img.shape[:2]
    tc = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    kind = 2 if height else (1 if directx else 0)
    lib().vlrref_pt_set_normal_map(ctypes.c_int32(group), _p(img), ctypes.c_uint32(w), ctypes.c_uint32(h),
                                   ctypes.c_int(1 if nearest else 0), ctypes.c_int(kind), ctypes.c_int(channel),
                                   ctypes.c_float(coeff), _p(tc), ctypes.c_uint32(len(tc)))


def alpha_map_set(group=-1, rgba=None, uv=None, nearest=False, channel=3):
    """Alpha map (channel `channel` of an Image2DTexture) on geometry group
    `group` of the following pt_render calls, with the scene's per-vertex
    texture coordinates: closest-hit rays keep an intersection with the
    CUDA build's per-(path state, primitive) decision, shadow rays carry the
    product of (1 - alpha).  Brute-force scenes only (under 4,096
    triangles).  group = -1 removes it."""
    if group < 0 or rgba is None:
        lib().vlrref_pt_set_alpha_map(ctypes.c_int32(-1), None, ctypes.c_uint32(0), ctypes.c_uint32(0), 0, 3,
                                      None, ctypes.c_uint32(0))
        return
    img = np.ascontiguousarray(rgba, np.float32)
    h, w = img.shape[:2]
    tc = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    lib().vlrref_pt_set_alpha_map(ctypes.c_int32(group), _p(img), ctypes.c_uint32(w), ctypes.c_uint32(h),
                                  ctypes.c_int(1 if nearest else 0), ctypes.c_int(channel), _p(tc),
                                  ctypes.c_uint32(len(tc)))


def multi_set(material=-1, subs=()):
    """Multi material of the following pt_render calls: material index
    `material` (in the flattened records) stands for the sum of the BSDFs of
    the 1-4 sub-material indices `subs`, as the reference's MultiBSDF
    samples, evaluates and blends them.  material = -1 removes it."""
    if material < 0 or not len(subs):
        lib().vlrref_pt_set_multi(ctypes.c_int32(-1), None, ctypes.c_uint32(0))
        return
    arr = np.array(subs, np.int32)
    lib().vlrref_pt_set_multi(ctypes.c_int32(material), _p(arr), ctypes.c_uint32(len(arr)))


def env_unsampleable():
    """Texels with positive luminance that the importance map can never
    sample (zero CDF step): FP64 full-resolution map, the same map built by
    the reference's FP32 Kahan builder, and the reference's own 4x smaller
    FP32 map; with the positive-texel counts."""
    v = [ctypes.c_uint64() for _ in range(5)]
    lib().vlrref_env_unsampleable(*[ctypes.byref(x) for x in v])
    return {"fp64_full": v[0].value, "fp32_full": v[1].value, "positive_full": v[2].value,
            "fp32_quarter": v[3].value, "positive_quarter": v[4].value}


def pt_render_fp32_films(flat, camera, width, height, spp, max_path_length, rng_states=None, threads=0):
    """pt_render that also feeds every contribution to two FP32 films: the
    reference's own SpectrumStorage (FP32 Kahan pairs per stratum, summed per
    sample) and a plain FP32 sum.  Returns (film64 [H,W,16], kahan_sum
    [H,W,16], plain [H,W,16], rng_states)."""
    kahan = np.zeros((height, width, 32), np.float32)
    plain = np.zeros((height, width, 16), np.float32)
    lib().vlrref_pt_set_fp32_films(_p(kahan), _p(plain))
    try:
        film, states, _ = pt_render(flat, camera, width, height, spp, max_path_length, rng_states=rng_states,
                                    threads=threads)
    finally:
        lib().vlrref_pt_set_fp32_films(None, None)
    return film, kahan[..., :16].copy(), plain, states


def pt_render_census(flat, camera, width, height, spp, max_path_length, rng_states=None, threads=0):
    """pt_render that also counts, per bounce, the rays traced and where they
    ended: [64, 16] uint64 in the layout of the CUDA path tracer's queue
    counters ([0] rays, [2 + k] hits on BSDF kind k, [10] misses).  Returns
    (film, rng_states, census)."""
    census = np.zeros((64, 16), np.uint64)
    lib().vlrref_pt_set_census(_p(census))
    try:
        film, states, _ = pt_render(flat, camera, width, height, spp, max_path_length, rng_states=rng_states,
                                    threads=threads)
    finally:
        lib().vlrref_pt_set_census(None)
    return film, states, census


def last_render_seconds():
    """Wall time of the last pt_render / bpt_render loop, scene set-up
    (BVH build) excluded."""
    f = lib().vlrref_last_render_seconds
    f.restype = ctypes.c_double
    return f()


def seed_states(n, seed=591842031321323413):
    """std::mt19937_64 outputs (the reference's per-pixel PCG32 seeding,
    libVLR/context.cpp:1176-1190) from the C++ standard library generator in
    the host build, as a uint64 array."""
    out = np.zeros(n, np.uint64)
    lib().vlrref_seed_states(ctypes.c_uint64(seed), ctypes.c_uint64(n), _p(out))
    return out


def seed_states_py(n, seed=591842031321323413):
    """The same outputs from the published 64-bit Mersenne Twister recurrence
    in pure Python (slow; pins the C++ generator on small n)."""
    return np.array(_mt19937_64(seed, n), np.uint64)


def _mt19937_64(seed, n):
    NN, MM = 312, 156
    MATRIX_A = 0xB5026F5AA96619E9
    UM, LM = 0xFFFFFFFF80000000, 0x7FFFFFFF
    mask = (1 << 64) - 1
    mt = [0] * NN
    mt[0] = seed & mask
    for i in range(1, NN):
        mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & mask
    idx = NN
    out = []
    for _ in range(n):
        if idx >= NN:
            for i in range(NN):
                x = (mt[i] & UM) | (mt[(i + 1) % NN] & LM)
                xa = x >> 1
                if x & 1:
                    xa ^= MATRIX_A
                mt[i] = mt[(i + MM) % NN] ^ xa
            idx = 0
        x = mt[idx]
        idx += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        out.append(x & mask)
    return out
