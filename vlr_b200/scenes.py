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
             "LambertianScattering": 4, "UE4": 5, "SpecularScattering": 6, "DiffuseEmitter": 7}
COLOR_SPACES = {"Rec709(D65) sRGB Gamma": 0, "Rec709(D65)": 1, "XYZ": 2, "xyY": 3}
# spectrum parameter of each slot, per material type
SPEC_SLOTS = {"Matte": ("albedo",), "SpecularReflection": ("coeff", "eta", "k"),
              "MicrofacetReflection": (None, "eta", "k"), "MicrofacetScattering": ("coeff", "eta ext", "eta int"),
              "LambertianScattering": ("coeff",), "UE4": ("base color",),
              "SpecularScattering": ("coeff", "eta ext", "eta int"), "DiffuseEmitter": ("emittance",)}
FLOAT_SLOTS = {"MicrofacetReflection": ("roughness", "anisotropy", "rotation"),
               "MicrofacetScattering": ("roughness", "anisotropy", "rotation"),
               "LambertianScattering": ("f0",), "UE4": ("roughness", "metallic")}
FLOAT_DEFAULTS = {"roughness": 0.1, "anisotropy": 0.0, "rotation": 0.0, "f0": 0.04, "metallic": 0.0}


def cornell_box_desc(width=512, height=512, glass="box", light_scale=1.0, emittance=15.0):
    """Plain description of the Cornell box workload (see module doc)."""
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
    v += _quad((-hl, 2.9, -hl), (hl, 2.9, -hl), (hl, 2.9, hl), (-hl, 2.9, hl), (0, -1, 0), (1, 0, 0))     # light
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
    cam = ctx.createCamera("Perspective")
    cam.set_point("position", c["position"])
    cam.set_quaternion("orientation", c["orientation"])
    for k in ("aspect", "sensitivity", "fovy", "lens radius", "op distance"):
        cam.set(k, c[k])
    return scene, cam, keep


def cornell_box(ctx, width=512, height=512, glass="box", light_scale=1.0, emittance=15.0):
    return build(ctx, cornell_box_desc(width, height, glass, light_scale, emittance))


MAT_DTYPE = np.dtype([("type", "<i4"), ("colorSpace", "<i4", 3), ("spectra", "<f4", (3, 3)),
                      ("params", "<f4", 4), ("emitScale", "<f4")])


def flatten_desc(desc):
    """World-space arrays of a description with identity transforms, in the
    layout of the oracle's path tracer: positions, normals, tangents,
    triangles (i0, i1, i2, group), group material, group light instance
    (each emitting mesh is one light instance), material records."""
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
    pos, nrm, tan, tris, gmat, glight = [], [], [], [], [], []
    base = 0
    n_light_inst = 0
    for mesh in desc["meshes"]:
        vv = mesh["verts"]
        pos.append(vv[:, 0:3]); nrm.append(vv[:, 3:6]); tan.append(vv[:, 6:9])
        emitting = False
        for idx, mname in mesh["groups"]:
            g = len(gmat)
            gmat.append(names.index(mname))
            is_emit = desc["materials"][mname][0] == "DiffuseEmitter"
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
            "groupMaterial": np.array(gmat, np.int32), "groupLightInst": np.array(glight, np.int32),
            "mats": recs}
