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


def cornell_box(ctx, width=512, height=512, glass="box", light_scale=1.0, emittance=15.0):
    scene = ctx.createScene()
    walls = ctx.createTriangleMeshSurfaceNode("CornellBox")
    v = []
    v += _quad((-1.5, 0, -1.5), (-1.5, 0, 1.5), (1.5, 0, 1.5), (1.5, 0, -1.5), (0, 1, 0), (1, 0, 0))      # floor
    v += _quad((-1.5, 0, -1.5), (1.5, 0, -1.5), (1.5, 3, -1.5), (-1.5, 3, -1.5), (0, 0, 1), (1, 0, 0))    # back
    v += _quad((-1.5, 3, -1.5), (1.5, 3, -1.5), (1.5, 3, 1.5), (-1.5, 3, 1.5), (0, -1, 0), (1, 0, 0))     # ceiling
    v += _quad((-1.5, 0, 1.5), (-1.5, 0, -1.5), (-1.5, 3, -1.5), (-1.5, 3, 1.5), (1, 0, 0), (0, 0, -1))   # left
    v += _quad((1.5, 0, -1.5), (1.5, 0, 1.5), (1.5, 3, 1.5), (1.5, 3, -1.5), (-1, 0, 0), (0, 0, 1))       # right
    hl = 0.5 * math.sqrt(light_scale)
    v += _quad((-hl, 2.9, -hl), (hl, 2.9, -hl), (hl, 2.9, hl), (-hl, 2.9, hl), (0, -1, 0), (1, 0, 0))     # light
    walls.set_vertices(np.array(v, np.float32))
    white = ctx.createSurfaceMaterial("Matte")
    white.set("albedo", V.Spectrum("Rec709(D65) sRGB Gamma", 0.75, 0.75, 0.75))
    red = ctx.createSurfaceMaterial("Matte")
    red.set("albedo", V.Spectrum("Rec709(D65) sRGB Gamma", 0.75, 0.25, 0.25))
    green = ctx.createSurfaceMaterial("Matte")
    green.set("albedo", V.Spectrum("Rec709(D65) sRGB Gamma", 0.25, 0.75, 0.25))
    light = ctx.createSurfaceMaterial("DiffuseEmitter")
    light.set("emittance", V.Spectrum("Rec709(D65)", emittance, emittance, emittance))
    walls.add_material_group([0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7, 8, 9, 10, 8, 10, 11], white)
    walls.add_material_group([12, 13, 14, 12, 14, 15], red)
    walls.add_material_group([16, 17, 18, 16, 18, 19], green)
    walls.add_material_group([20, 21, 22, 20, 22, 23], light)
    scene.add_child(walls)

    metal = ctx.createSurfaceMaterial("MicrofacetReflection")
    metal.set("eta", V.Spectrum("Rec709(D65)", 0.2, 0.4, 1.4))
    metal.set("k", V.Spectrum("Rec709(D65)", 3.9, 2.4, 1.8))
    metal.set("roughness", 0.3)
    metal.set("anisotropy", 0.8)
    box_v, box_i = _box((-0.6, 0.0, -0.5), 0.6, math.radians(20))
    mbox = ctx.createTriangleMeshSurfaceNode("MetalBox")
    mbox.set_vertices(box_v)
    mbox.add_material_group(box_i, metal)
    scene.add_child(mbox)

    glass_mat = ctx.createSurfaceMaterial("MicrofacetScattering")
    glass_mat.set("coeff", V.Spectrum("Rec709(D65)", 1.0, 1.0, 1.0))
    glass_mat.set("eta ext", V.Spectrum("Rec709(D65)", 1.0, 1.0, 1.0))
    glass_mat.set("eta int", V.Spectrum("Rec709(D65)", 1.5, 1.5, 1.5))
    gnode = ctx.createTriangleMeshSurfaceNode("Glass")
    if glass == "sphere":
        glass_mat.set("roughness", 0.02)
        gv, gi = uv_sphere((0.5, 0.55, 0.4), 0.55, 71, 142)   # 20,022 triangles
    else:
        glass_mat.set("roughness", 0.01)
        gv, gi = _box((0.6, 0.0, 0.5), 0.3, math.radians(-15))
    gnode.set_vertices(gv)
    gnode.add_material_group(gi, glass_mat)
    scene.add_child(gnode)

    cam = ctx.createCamera("Perspective")
    cam.set_point("position", (0.0, 1.5, 6.0))
    cam.set_quaternion("orientation", V.quat_rotate_y(math.pi))
    cam.set("aspect", width / height)
    cam.set("sensitivity", 1.0)
    cam.set("fovy", 40 * math.pi / 180)
    cam.set("lens radius", 0.0)
    cam.set("op distance", 1.0)
    keep = [walls, mbox, gnode, white, red, green, light, metal, glass_mat]
    return scene, cam, keep
