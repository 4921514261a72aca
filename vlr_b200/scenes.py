"""Seeded procedural scenes built through the C API (vlr_b200.vlr).

cornell_box    the Cornell box of the path-tracing workload: the reference's
               3x3x3 box frame, ceiling light and camera
               (HostProgram/scene.cpp:537-562, :787-802), white/red/green
               Matte walls, a 0.6-unit anisotropic GGX metal box, a 0.3-unit
               GGX glass box (IOR 1.5, roughness 0.01) and a 1x1 ceiling
               light with Rec.709(D65) emittance 15.  With glass="sphere" the
               glass box becomes a 20k-triangle GGX dielectric sphere
               (roughness 0.02) and the light shrinks to 0.1x area: the
               glossy-caustic scene of the guiding workload.
terrain_scene  1024x1024-cell fBm heightfield (2,097,152 triangles) plus 4096
               instanced 320-triangle icospheres under a procedural sky with
               a sun lobe (LVC-BPT + environment workload).
"""
import math

import numpy as np

from . import vlr as V


def _quad(p0, p1, p2, p3, n, t):
    return [list(p) + list(n) + list(t) + [0.0, 0.0] for p in (p0, p1, p2, p3)]


def _box(center, size, rot_y):
    """Axis-aligned box rotated about +y; 24 vertices, 12 triangles, flat normals."""
    c, s = math.cos(rot_y), math.sin(rot_y)

    def R(v):
        return (c * v[0] + s * v[2], v[1], -s * v[0] + c * v[2])

    hx = hz = size / 2
    h = size
    verts, idx = [], []
    faces = [
        ((0, 1, 0), [(-hx, h, -hz), (-hx, h, hz), (hx, h, hz), (hx, h, -hz)], (1, 0, 0)),
        ((0, -1, 0), [(-hx, 0, hz), (-hx, 0, -hz), (hx, 0, -hz), (hx, 0, hz)], (1, 0, 0)),
        ((0, 0, 1), [(-hx, 0, hz), (hx, 0, hz), (hx, h, hz), (-hx, h, hz)], (1, 0, 0)),
        ((0, 0, -1), [(hx, 0, -hz), (-hx, 0, -hz), (-hx, h, -hz), (hx, h, -hz)], (-1, 0, 0)),
        ((1, 0, 0), [(hx, 0, hz), (hx, 0, -hz), (hx, h, -hz), (hx, h, hz)], (0, 0, -1)),
        ((-1, 0, 0), [(-hx, 0, -hz), (-hx, 0, hz), (-hx, h, hz), (-hx, h, -hz)], (0, 0, 1)),
    ]
    for n, ps, t in faces:
        b = len(verts)
        for p in ps:
            q = R(p)
            verts.append([q[0] + center[0], q[1] + center[1], q[2] + center[2]] + list(R(n)) + list(R(t)) + [0, 0])
        idx += [b, b + 1, b + 2, b, b + 2, b + 3]
    return np.array(verts, np.float32), np.array(idx, np.uint32)


def uv_sphere(center, radius, n_lat, n_lon):
    """UV sphere with smooth normals: 2 * n_lon * (n_lat - 1) triangles."""
    verts, idx = [], []
    for i in range(n_lat + 1):
        th = math.pi * i / n_lat
        for j in range(n_lon + 1):
            ph = 2 * math.pi * j / n_lon
            n = (math.sin(th) * math.cos(ph), math.cos(th), math.sin(th) * math.sin(ph))
            t = (-math.sin(ph), 0.0, math.cos(ph))
            verts.append([center[0] + radius * n[0], center[1] + radius * n[1], center[2] + radius * n[2]]
                         + list(n) + list(t) + [j / n_lon, i / n_lat])
    row = n_lon + 1
    for i in range(n_lat):
        for j in range(n_lon):
            a, b, c, d = i * row + j, i * row + j + 1, (i + 1) * row + j + 1, (i + 1) * row + j
            if i != 0:
                idx += [a, c, b]
            if i != n_lat - 1:
                idx += [a, d, c]
    return np.array(verts, np.float32), np.array(idx, np.uint32)


MAT_TYPES = {"Matte": 0, "SpecularReflection": 1, "MicrofacetReflection": 2, "MicrofacetScattering": 3,
             "LambertianScattering": 4, "UE4": 5, "SpecularScattering": 6, "DiffuseEmitter": 7,
             "DirectionalEmitter": 8}
COLOR_SPACES = {"Rec709(D65) sRGB Gamma": 0, "Rec709(D65)": 1, "XYZ": 2, "xyY": 3}
# spectrum parameter of each slot, per material type
SPEC_SLOTS = {"Matte": ("albedo",), "SpecularReflection": ("coeff", "eta", "k"),
              "MicrofacetReflection": (None, "eta", "k"), "MicrofacetScattering": ("coeff", "eta ext", "eta int"),
              "LambertianScattering": ("coeff",), "UE4": ("base color",),
              "SpecularScattering": ("coeff", "eta ext", "eta int"), "DiffuseEmitter": ("emittance",),
              "DirectionalEmitter": ("emittance",)}
FLOAT_SLOTS = {"MicrofacetReflection": ("roughness", "anisotropy", "rotation"),
               "MicrofacetScattering": ("roughness", "anisotropy", "rotation"),
               "LambertianScattering": ("f0",), "UE4": ("roughness", "metallic")}
FLOAT_DEFAULTS = {"roughness": 0.1, "anisotropy": 0.0, "rotation": 0.0, "f0": 0.04, "metallic": 0.0}


def cornell_box_desc(width=512, height=512, glass="box", light_scale=1.0, emittance=15.0, light_up=False):
    """Plain description of the Cornell box workload (see module doc).
    light_up: the light hangs at 2.4 facing the ceiling, so the room is lit
    only by the bright ceiling patch above it (indirect light that next-event
    estimation cannot reach)."""
    srgb = "Rec709(D65) sRGB Gamma"
    lin = "Rec709(D65)"
    mats = {
        "white": ("Matte", {"albedo": (srgb, 0.75, 0.75, 0.75)}),
        "red": ("Matte", {"albedo": (srgb, 0.75, 0.25, 0.25)}),
        "green": ("Matte", {"albedo": (srgb, 0.25, 0.75, 0.25)}),
        "light": ("DiffuseEmitter", {"emittance": (lin, emittance, emittance, emittance)}),
        "metal": ("MicrofacetReflection", {"eta": (lin, 0.2, 0.4, 1.4), "k": (lin, 3.9, 2.4, 1.8),
                                           "roughness": 0.3, "anisotropy": 0.8}),
        "glass": ("MicrofacetScattering", {"coeff": (lin, 1.0, 1.0, 1.0), "eta ext": (lin, 1.0, 1.0, 1.0),
                                          "eta int": (lin, 1.5, 1.5, 1.5),
                                          "roughness": 0.02 if glass == "sphere" else 0.01}),
    }
    v = []
    v += _quad((-1.5, 0, -1.5), (-1.5, 0, 1.5), (1.5, 0, 1.5), (1.5, 0, -1.5), (0, 1, 0), (1, 0, 0))      # floor
    v += _quad((-1.5, 0, -1.5), (1.5, 0, -1.5), (1.5, 3, -1.5), (-1.5, 3, -1.5), (0, 0, 1), (1, 0, 0))    # back
    v += _quad((-1.5, 3, -1.5), (1.5, 3, -1.5), (1.5, 3, 1.5), (-1.5, 3, 1.5), (0, -1, 0), (1, 0, 0))     # ceiling
    v += _quad((-1.5, 0, 1.5), (-1.5, 0, -1.5), (-1.5, 3, -1.5), (-1.5, 3, 1.5), (1, 0, 0), (0, 0, -1))   # left
    v += _quad((1.5, 0, -1.5), (1.5, 0, 1.5), (1.5, 3, 1.5), (1.5, 3, -1.5), (-1, 0, 0), (0, 0, 1))       # right
    hl = 0.5 * math.sqrt(light_scale)
    if light_up:
        v += _quad((-hl, 2.4, -hl), (-hl, 2.4, hl), (hl, 2.4, hl), (hl, 2.4, -hl), (0, 1, 0), (1, 0, 0))  # light, up
    else:
        v += _quad((-hl, 2.9, -hl), (hl, 2.9, -hl), (hl, 2.9, hl), (-hl, 2.9, hl), (0, -1, 0), (1, 0, 0))  # light
    meshes = [{"name": "CornellBox", "verts": np.array(v, np.float32), "groups": [
        (np.array([0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7, 8, 9, 10, 8, 10, 11], np.uint32), "white"),
        (np.array([12, 13, 14, 12, 14, 15], np.uint32), "red"),
        (np.array([16, 17, 18, 16, 18, 19], np.uint32), "green"),
        (np.array([20, 21, 22, 20, 22, 23], np.uint32), "light")]}]
    bv, bi = _box((-0.6, 0.0, -0.5), 0.6, math.radians(20))
    meshes.append({"name": "MetalBox", "verts": bv, "groups": [(bi, "metal")]})
    if glass == "sphere":
        gv, gi = uv_sphere((0.5, 0.55, 0.4), 0.55, 71, 142)   # 20,022 triangles
    else:
        gv, gi = _box((0.6, 0.0, 0.5), 0.3, math.radians(-15))
    meshes.append({"name": "Glass", "verts": gv, "groups": [(gi, "glass")]})
    camera = {"position": (0.0, 1.5, 6.0), "orientation": V.quat_rotate_y(math.pi), "aspect": width / height,
              "sensitivity": 1.0, "fovy": 40 * math.pi / 180, "lens radius": 0.0, "op distance": 1.0}
    return {"materials": mats, "meshes": meshes, "camera": camera, "width": width, "height": height}


def build(ctx, desc):
    """Create the described scene through the C API. Returns (scene, camera, keepalive)."""
    scene = ctx.createScene()
    keep = []
    mats = {}
    for name, (typ, params) in desc["materials"].items():
        m = ctx.createSurfaceMaterial(typ)
        for k, val in params.items():
            m.set(k, V.Spectrum(*val) if isinstance(val, tuple) else float(val))
        mats[name] = m
        keep.append(m)
    for mesh in desc["meshes"]:
        node = ctx.createTriangleMeshSurfaceNode(mesh["name"])
        node.set_vertices(mesh["verts"])
        for idx, mname in mesh["groups"]:
            node.add_material_group(idx, mats[mname])
        scene.add_child(node)
        keep.append(node)
    c = desc["camera"]
    if c.get("type", "Perspective") == "Equirectangular":
        cam = ctx.createCamera("Equirectangular")
        keys = ("sensitivity", "h angle", "v angle")
    else:
        cam = ctx.createCamera("Perspective")
        keys = ("aspect", "sensitivity", "fovy", "lens radius", "op distance")
    cam.set_point("position", c["position"])
    cam.set_quaternion("orientation", c["orientation"])
    for k in keys:
        cam.set(k, c[k])
    return scene, cam, keep


def cornell_box(ctx, width=512, height=512, glass="box", light_scale=1.0, emittance=15.0, light_up=False):
    return build(ctx, cornell_box_desc(width, height, glass, light_scale, emittance, light_up))


MAT_DTYPE = np.dtype([("type", "<i4"), ("colorSpace", "<i4", 3), ("spectra", "<f4", (3, 3)),
                      ("params", "<f4", 4), ("emitScale", "<f4")])


def flatten_desc(desc):
    """World-space arrays of a description with identity transforms, in the
    layout of the oracle's path tracer: positions, normals, tangents,
    texture coordinates, triangles (i0, i1, i2, group), group material, group
    light instance (each emitting mesh is one light instance), material
    records."""
    names = list(desc["materials"].keys())
    recs = np.zeros(len(names), MAT_DTYPE)
    for i, name in enumerate(names):
        typ, params = desc["materials"][name]
        recs[i]["type"] = MAT_TYPES[typ]
        recs[i]["emitScale"] = float(params.get("scale", 1.0))
        for k, slot in enumerate(SPEC_SLOTS[typ]):
            if slot is None:
                recs[i]["colorSpace"][k] = 1
                continue
            cs, e0, e1, e2 = params[slot]
            recs[i]["colorSpace"][k] = COLOR_SPACES[cs]
            recs[i]["spectra"][k] = (e0, e1, e2)
        for k, slot in enumerate(FLOAT_SLOTS.get(typ, ())):
            recs[i]["params"][k] = float(params.get(slot, FLOAT_DEFAULTS[slot]))
    pos, nrm, tan, uv, tris, gmat, glight = [], [], [], [], [], [], []
    base = 0
    n_light_inst = 0
    for mesh in desc["meshes"]:
        vv = mesh["verts"]
        pos.append(vv[:, 0:3]); nrm.append(vv[:, 3:6]); tan.append(vv[:, 6:9])
        uv.append(vv[:, 9:11] if vv.shape[1] >= 11 else np.zeros((len(vv), 2), np.float32))
        emitting = False
        for idx, mname in mesh["groups"]:
            g = len(gmat)
            gmat.append(names.index(mname))
            is_emit = desc["materials"][mname][0] in ("DiffuseEmitter", "DirectionalEmitter")
            glight.append(n_light_inst if is_emit else -1)
            emitting = emitting or is_emit
            t = idx.reshape(-1, 3).astype(np.uint32) + base
            tris.append(np.concatenate([t, np.full((len(t), 1), g, np.uint32)], axis=1))
        if emitting:
            n_light_inst += 1
        base += len(vv)
    return {"pos": np.ascontiguousarray(np.concatenate(pos), np.float32),
            "nrm": np.ascontiguousarray(np.concatenate(nrm), np.float32),
            "tan": np.ascontiguousarray(np.concatenate(tan), np.float32),
            "tris": np.ascontiguousarray(np.concatenate(tris), np.uint32),
            "uv": np.ascontiguousarray(np.concatenate(uv), np.float32),
            "groupMaterial": np.array(gmat, np.int32), "groupLightInst": np.array(glight, np.int32),
            "mats": recs}


def flatten_instanced_desc(desc):
    """flatten_desc() of a description with instanced meshes (terrain
    workload layout): every instance's mesh is appended in world space,
    positions transformed as the library flattens them (s * x + t in float32,
    in the same order), normals by the inverse scale, tangents by the scale."""
    flat = flatten_desc(desc)
    names = list(desc["materials"].keys())
    pos, nrm, tan, tris, gmat, glight = ([flat["pos"]], [flat["nrm"]], [flat["tan"]], [flat["tris"]],
                                         list(flat["groupMaterial"]), list(flat["groupLightInst"]))
    base = len(flat["pos"])
    for inst in desc.get("instances", []):
        mesh = desc["instanced"][inst["mesh"]]
        vv = mesh["verts"]
        s = np.float32(inst["scale"])
        t = np.array(inst["translate"], np.float32)
        zero = np.float32(0.0)
        p = vv[:, 0:3].astype(np.float32)
        x = ((s * p[:, 0] + zero * p[:, 1]) + zero * p[:, 2]) + t[0]
        y = ((zero * p[:, 0] + s * p[:, 1]) + zero * p[:, 2]) + t[1]
        z = ((zero * p[:, 0] + zero * p[:, 1]) + s * p[:, 2]) + t[2]
        pos.append(np.stack([x, y, z], 1).astype(np.float32))
        nrm.append((vv[:, 3:6] * (np.float32(1.0) / s)).astype(np.float32))
        tan.append((vv[:, 6:9] * s).astype(np.float32))
        for idx, mname in mesh["groups"]:
            g = len(gmat)
            gmat.append(names.index(mname))
            glight.append(-1)
            tri = idx.reshape(-1, 3).astype(np.uint32) + base
            tris.append(np.concatenate([tri, np.full((len(tri), 1), g, np.uint32)], axis=1))
        base += len(vv)
    out = dict(flat)
    out.update({"pos": np.ascontiguousarray(np.concatenate(pos), np.float32),
                "nrm": np.ascontiguousarray(np.concatenate(nrm), np.float32),
                "tan": np.ascontiguousarray(np.concatenate(tan), np.float32),
                "tris": np.ascontiguousarray(np.concatenate(tris), np.uint32),
                "groupMaterial": np.array(gmat, np.int32), "groupLightInst": np.array(glight, np.int32)})
    return out


def _fbm(n, seed, octaves=7):
    """(n+1)x(n+1) fractional Brownian motion heights in [-1, 1] from bilinearly
    interpolated value noise, seeded."""
    rng = np.random.default_rng(seed)
    h = np.zeros((n + 1, n + 1), np.float64)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 * (2 ** o)
        g = rng.uniform(-1, 1, (cells + 1, cells + 1))
        x = np.linspace(0, cells, n + 1)
        i = np.minimum(x.astype(int), cells - 1)
        t = x - i
        t = t * t * (3 - 2 * t)
        a = g[i][:, i] * (1 - t)[None, :] + g[i][:, i + 1] * t[None, :]
        b = g[i + 1][:, i] * (1 - t)[None, :] + g[i + 1][:, i + 1] * t[None, :]
        h += amp * (a * (1 - t)[:, None] + b * t[:, None])
        total += amp
        amp *= 0.5
    return h / total


def icosphere(level=2):
    """Unit icosphere: 20 * 4**level triangles (320 at level 2)."""
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    v = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = v[a] + v[b]
                v.append(m / np.linalg.norm(m))
                cache[k] = len(v) - 1
            return cache[k]
        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    P = np.array(v, np.float32)
    tan = np.cross(np.array([0, 1, 0], np.float32), P)
    bad = np.linalg.norm(tan, axis=1) < 1e-6
    tan[bad] = (1, 0, 0)
    tan /= np.linalg.norm(tan, axis=1, keepdims=True)
    verts = np.concatenate([P, P, tan, np.zeros((len(P), 2), np.float32)], axis=1).astype(np.float32)
    return verts, np.array(f, np.uint32).reshape(-1)


def sky_image(width=2048, height=1024, sun_dir=(0.35, 0.6, -0.72), sun_radius_deg=0.5, sun_rel=1e4):
    """Procedural RGB sky on an equirectangular grid (row 0 = zenith): a
    horizon-to-zenith gradient, dark ground below the horizon, and a sun disc
    of the given angular diameter whose radiance is sun_rel times the zenith
    sky's."""
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    theta = np.pi * v[:, None]
    phi = 2 * np.pi * u[None, :]
    # direction for (phi, theta) with y up, matching the renderer's mapping
    d = np.stack([-np.sin(phi) * np.sin(theta), np.cos(theta) * np.ones_like(phi), np.cos(phi) * np.sin(theta)], -1)
    up = d[..., 1]
    zen = np.array([0.25, 0.45, 0.95])
    hor = np.array([0.85, 0.9, 1.0])
    t = np.clip(up, 0, 1)[..., None]
    sky = hor * (1 - t) ** 3 + zen * (1 - (1 - t) ** 3)
    ground = np.array([0.18, 0.16, 0.14])
    img = np.where(up[..., None] > 0, sky, ground * np.clip(1 + up, 0, 1)[..., None])
    s = np.array(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    cosang = np.clip(d @ s, -1, 1)
    half = np.radians(sun_radius_deg / 2)
    sun = cosang >= np.cos(half)
    img[sun] = zen.max() * sun_rel * np.array([1.0, 0.95, 0.85])
    rgba = np.concatenate([img, np.ones(img.shape[:2] + (1,))], -1).astype(np.float32)
    return rgba


def terrain_scene_desc(width=1920, height=1080, cells=1024, n_spheres=4096, seed=7, sky=(2048, 1024)):
    """Description of the LVC-BPT + environment workload (see module doc).
    Terrain: cells x cells quads = 2 * cells**2 triangles; spheres: instanced
    320-triangle icospheres with random scale in [0.5, 3] and random material."""
    rng = np.random.default_rng(seed)
    size = 1024.0
    h = _fbm(cells, seed) * 60.0
    xs = np.linspace(-size / 2, size / 2, cells + 1)
    X, Z = np.meshgrid(xs, xs)
    P = np.stack([X, h, Z], -1).astype(np.float32)
    dx = np.gradient(h, xs, axis=1)
    dz = np.gradient(h, xs, axis=0)
    N = np.stack([-dx, np.ones_like(h), -dz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    T = np.stack([np.ones_like(h), dx, np.zeros_like(h)], -1)
    T /= np.linalg.norm(T, axis=-1, keepdims=True)
    verts = np.concatenate([P.reshape(-1, 3), N.reshape(-1, 3), T.reshape(-1, 3),
                            np.zeros(((cells + 1) ** 2, 2))], 1).astype(np.float32)
    i = np.arange(cells)
    r, c = np.meshgrid(i, i, indexing="ij")
    v00 = (r * (cells + 1) + c).reshape(-1)
    v01, v10, v11 = v00 + 1, v00 + cells + 1, v00 + cells + 2
    quads = np.stack([v00, v10, v11, v00, v11, v01], 1).astype(np.uint32)
    # materials: 8 terrain materials assigned per 64x64-cell patch
    mats = {}
    for k in range(8):
        rough = float(rng.uniform(0.2, 0.9))
        col = tuple(float(x) for x in rng.uniform(0.15, 0.6, 3))
        if k % 2 == 0:
            mats[f"terrain{k}"] = ("Matte", {"albedo": ("Rec709(D65)",) + col})
        else:
            mats[f"terrain{k}"] = ("UE4", {"base color": ("Rec709(D65)",) + col, "roughness": rough,
                                           "metallic": float(rng.uniform(0, 0.3))})
    patch = ((r // 64) * 7 + (c // 64) * 3).reshape(-1) % 8
    groups = [(quads[patch == k].reshape(-1), f"terrain{k}") for k in range(8)]
    meshes = [{"name": "Terrain", "verts": verts, "groups": groups}]
    # sphere materials and instances
    sv, si = icosphere(2)
    sphere_mats = []
    for k in range(8):
        name = f"sphere{k}"
        col = tuple(float(x) for x in rng.uniform(0.1, 0.9, 3))
        kind = k % 4
        if kind == 0:
            mats[name] = ("Matte", {"albedo": ("Rec709(D65)",) + col})
        elif kind == 1:
            mats[name] = ("UE4", {"base color": ("Rec709(D65)",) + col, "roughness": float(rng.uniform(0.2, 0.9)),
                                  "metallic": 1.0})
        elif kind == 2:
            mats[name] = ("MicrofacetReflection", {"eta": ("Rec709(D65)", 0.2, 0.4, 1.4),
                                                   "k": ("Rec709(D65)", 3.9, 2.4, 1.8),
                                                   "roughness": float(rng.uniform(0.2, 0.6))})
        else:
            mats[name] = ("LambertianScattering", {"coeff": ("Rec709(D65)",) + col})
        sphere_mats.append(name)
    instances = []
    for s in range(n_spheres):
        px, pz = rng.uniform(-size / 2 * 0.9, size / 2 * 0.9, 2)
        ci = int(np.clip((px + size / 2) / size * cells, 0, cells))
        ri = int(np.clip((pz + size / 2) / size * cells, 0, cells))
        scale = float(rng.uniform(0.5, 3.0))
        y = float(h[ri, ci]) + scale * 0.8
        instances.append({"mesh": sphere_mats[int(rng.integers(0, 8))], "scale": scale, "translate": (px, y, pz)})
    sphere_meshes = {name: {"name": "Ico_" + name, "verts": sv, "groups": [(si, name)]} for name in sphere_mats}
    camera = {"position": (0.0, 160.0, 420.0), "orientation": _look_quat((0.0, -0.35, -1.0)),
              "aspect": width / height, "sensitivity": 1.0, "fovy": 50 * math.pi / 180, "lens radius": 0.0,
              "op distance": 1.0}
    return {"materials": mats, "meshes": meshes, "instanced": sphere_meshes, "instances": instances,
            "camera": camera, "width": width, "height": height,
            "env": {"image": sky_image(*sky), "scale": 1.0}}


def _look_quat(forward):
    """Quaternion (x, y, z, w) rotating +z onto `forward` with +y kept up."""
    f = np.array(forward, np.float64)
    f /= np.linalg.norm(f)
    r = np.cross(np.array([0.0, 1.0, 0.0]), f)
    r /= np.linalg.norm(r)
    u = np.cross(f, r)
    m = np.stack([r, u, f], 1)   # columns: right, up, forward
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0:
        s = math.sqrt(tr + 1.0) * 2
        return ((m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s, 0.25 * s)
    i = int(np.argmax([m[0, 0], m[1, 1], m[2, 2]]))
    j, k = (i + 1) % 3, (i + 2) % 3
    s = math.sqrt(1.0 + m[i, i] - m[j, j] - m[k, k]) * 2
    q = [0.0, 0.0, 0.0, 0.0]
    q[i] = 0.25 * s
    q[j] = (m[j, i] + m[i, j]) / s
    q[k] = (m[k, i] + m[i, k]) / s
    q[3] = (m[k, j] - m[j, k]) / s
    return tuple(q)


def build_instanced(ctx, desc):
    """build() plus instanced meshes under internal nodes and the environment."""
    scene, cam, keep = build(ctx, desc)
    mats = {}
    for name, (typ, params) in desc["materials"].items():
        if name in desc.get("instanced", {}):
            pass
    # material handles created by build(), in order
    names = list(desc["materials"].keys())
    mats = dict(zip(names, keep[:len(names)]))
    meshes = {}
    for name, mesh in desc.get("instanced", {}).items():
        node = ctx.createTriangleMeshSurfaceNode(mesh["name"])
        node.set_vertices(mesh["verts"])
        for idx, mname in mesh["groups"]:
            node.add_material_group(idx, mats[mname])
        meshes[name] = node
        keep.append(node)
    for inst in desc.get("instances", []):
        s = inst["scale"]
        tx, ty, tz = inst["translate"]
        m = [s, 0, 0, 0, 0, s, 0, 0, 0, 0, s, 0, tx, ty, tz, 1]
        node = ctx.createInternalNode("inst", ctx.transform(m))
        node.add_child(meshes[inst["mesh"]])
        scene.add_child(node)
        keep.append(node)
    env = desc.get("env")
    if env is not None:
        img = ctx.createLinearImage2D(env["image"], "Light Source", "Rec709(D65)")
        tex = ctx.createShaderNode("EnvironmentTexture")
        tex.set("image", img)
        em = ctx.createSurfaceMaterial("EnvironmentEmitter")
        em.set("emittance", tex.plug())
        em.set("scale", env.get("scale", 1.0))
        scene.set_environment(em, env.get("rotation", 0.0))
        keep += [img, tex, em]
    return scene, cam, keep


def floor_desc(W, H, light_at=(1.2, -1.2), sheet=False):
    """Description of the lit-floor scene: a 4 x 4 white floor at y = 0 (u
    along +x, v along +z; tangent +x) and a 1 x 1 downward-facing light at
    height 2 over `light_at` (x, z), seen by a camera at height 0.9 looking
    straight down (40-degree field of view).  sheet: a black 6 x 6 sheet at
    height 1 between them (its third group, for an alpha map)."""
    uvs = [(0, 0), (0, 1), (1, 1), (1, 0)]

    def quad(corners, n, t):
        return np.array([list(p) + list(n) + list(t) + list(uv) for p, uv in zip(corners, uvs)], np.float32)

    lx, lz = light_at
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    return {
        "materials": {"floor": ("Matte", {"albedo": ("Rec709(D65)", 0.8, 0.8, 0.8)}),
                      "light": ("DiffuseEmitter", {"emittance": ("Rec709(D65)", 10.0, 10.0, 10.0)}),
                      "sheet": ("Matte", {"albedo": ("Rec709(D65)", 0.0, 0.0, 0.0)})},
        "meshes": [{"verts": quad([(-2, 0, -2), (-2, 0, 2), (2, 0, 2), (2, 0, -2)], (0, 1, 0), (1, 0, 0)),
                    "groups": [(idx, "floor")]},
                   {"verts": quad([(lx - .5, 2, lz - .5), (lx + .5, 2, lz - .5), (lx + .5, 2, lz + .5),
                                   (lx - .5, 2, lz + .5)], (0, -1, 0), (1, 0, 0)),
                    "groups": [(idx, "light")]}] +
                  ([{"verts": quad([(-3, 1, -3), (3, 1, -3), (3, 1, 3), (-3, 1, 3)], (0, -1, 0), (1, 0, 0)),
                     "groups": [(idx, "sheet")]}] if sheet else []),
        "camera": {"position": (0.0, 0.9, 0.0), "orientation": (np.sqrt(0.5), 0.0, 0.0, np.sqrt(0.5)),
                   "aspect": W / H, "sensitivity": 1.0, "fovy": 40 * np.pi / 180, "lens radius": 0.0,
                   "op distance": 1.0},
    }
