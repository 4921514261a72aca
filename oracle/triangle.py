"""Watertight ray/triangle intersection in numpy float32 (TEST INFRASTRUCTURE).

The triangle test that stands in for the hardware intersection under
optixTrace (path_tracing.cu:89-93): Woop, Benthin and Wald, "Watertight
Ray/Triangle Intersection", JCGT 2(1), 2013.  numpy applies each float32
operation with one rounding and never contracts, so this evaluates the same
operations in the same order as the CUDA traversal (vlr_b200/csrc/lbvh.cuh
triTest) and the oracle's C++ restatement (ref_pt.inc triHit): t and the
barycentrics agree bit for bit.
"""
import numpy as np

f32 = np.float32


def ray_shear(d):
    """(kx, ky, kz, sx, sy, sz) of a float32 direction: kz the axis of the
    largest |component| (ties to the lower axis), kx, ky the next two in
    cyclic order, swapped when d[kz] < 0."""
    ax, ay, az = (abs(f32(c)) for c in d)
    kz = (0 if ax >= az else 2) if ax >= ay else (1 if ay >= az else 2)
    kx = 0 if kz == 2 else kz + 1
    ky = 0 if kx == 2 else kx + 1
    if f32(d[kz]) < 0:
        kx, ky = ky, kx
    dz = f32(d[kz])
    return kx, ky, kz, f32(d[kx]) / dz, f32(d[ky]) / dz, f32(1.0) / dz


def intersect_all(tri, o, d, tmax):
    """Watertight test of one ray against every triangle.
    tri: [n, 3, 3] float32 vertices; o, d: float32 origin and direction.
    Returns (hit mask, t, b1, b2), b1/b2 the weights of vertices 1 and 2."""
    tri = np.asarray(tri, f32)
    o = np.asarray(o, f32)
    kx, ky, kz, sx, sy, sz = ray_shear(d)
    A, B, C = tri[:, 0] - o, tri[:, 1] - o, tri[:, 2] - o
    az, bz, cz = A[:, kz], B[:, kz], C[:, kz]
    Ax, Ay = A[:, kx] - sx * az, A[:, ky] - sy * az
    Bx, By = B[:, kx] - sx * bz, B[:, ky] - sy * bz
    Cx, Cy = C[:, kx] - sx * cz, C[:, ky] - sy * cz
    U = Cx * By - Cy * Bx
    V = Ax * Cy - Ay * Cx
    W = Bx * Ay - By * Ax
    zero = (U == 0) | (V == 0) | (W == 0)
    if zero.any():
        d64 = lambda a: a[zero].astype(np.float64)
        U[zero] = (d64(Cx) * d64(By) - d64(Cy) * d64(Bx)).astype(f32)
        V[zero] = (d64(Ax) * d64(Cy) - d64(Ay) * d64(Cx)).astype(f32)
        W[zero] = (d64(Bx) * d64(Ay) - d64(By) * d64(Ax)).astype(f32)
    ok = ~(((U < 0) | (V < 0) | (W < 0)) & ((U > 0) | (V > 0) | (W > 0)))
    det = (U + V) + W
    ok &= det != 0
    T = (U * (sz * az) + V * (sz * bz)) + W * (sz * cz)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = T / det
        b1, b2 = V / det, W / det
    ok &= (t > 0) & (t < f32(tmax))
    return ok, t, b1, b2


def closest_hits(tri, rays):
    """Closest hit per ray over every triangle.  rays: [m, 8] float32
    (origin xyz, tmax, direction xyz, -).  Returns (t, prim, unique):
    t = inf and prim = 0xFFFFFFFF for a miss; unique is False where another
    triangle has the same t (a hit on a shared edge or vertex)."""
    m = len(rays)
    best_t = np.full(m, np.inf, f32)
    best = np.full(m, 0xFFFFFFFF, np.uint32)
    unique = np.ones(m, bool)
    for i, r in enumerate(np.asarray(rays, f32)):
        ok, t, _, _ = intersect_all(tri, r[0:3], r[4:7], r[3])
        if ok.any():
            tt = np.where(ok, t, np.inf)
            j = int(np.argmin(tt))
            best_t[i], best[i] = tt[j], j
            unique[i] = np.count_nonzero(tt == tt[j]) == 1
    return best_t, best, unique
