// Linear BVH over world-space triangles: build (Morton codes, radix sort,
// Karras hierarchy, bottom-up refit) and ray traversal.
//
// This replaces the OptiX acceleration structures the reference builds
// (libVLR/scene.cpp:1318-1328) and optixTrace (path_tracing.cu:89-93,
// light_transport_common.h:169-172).
//
// Layout in device memory:
//   nodes:  N-1 internal nodes of 64 B, each holding both children's boxes so a
//           traversal step is one 64-byte load (four 16-byte vector loads);
//   tris:   N triangles in BVH (sorted) order, 48 B each: the three
//           vertices as given (the watertight test needs the vertices a
//           neighbouring triangle shares bit for bit, not edges rounded per
//           triangle) plus the original primitive index in v0.w's bits.
// Child references >= 0 are internal nodes; ~index (negative) are leaves.
//
// No hit is lost by construction:
//   * the ray/triangle test is watertight (Woop, Benthin and Wald,
//     "Watertight Ray/Triangle Intersection", JCGT 2(1), 2013): a ray through
//     an edge or vertex shared by triangles of a closed mesh hits at least one
//     of them.  The edge functions are evaluated without contraction, so the
//     two triangles of an edge compute exact negatives of each other, and in
//     double precision when one rounds to zero;
//   * the box test is conservative: the far slab distance is scaled up by
//     1 + 2*gamma(3), gamma(n) = n*eps/(1 - n*eps), which covers the three
//     roundings of (bound - origin) * (1 / direction) (Ize, "Robust BVH Ray
//     Traversal", JCGT 2(2), 2013), so a box the exact ray enters is entered;
//   * the traversal stack holds one entry per tree level, and the build keeps
//     every leaf within kTraversalStack levels (lbvh_build.h).
#pragma once

#include "core.cuh"

namespace vlrb {

struct BvhNode {
    float4 lo0;  // child 0 min xyz, child index 0 (bits) in w
    float4 hi0;  // child 0 max xyz, unused w
    float4 lo1;  // child 1 min xyz, child index 1 (bits) in w
    float4 hi1;
};

struct BvhTri {
    float4 v0;   // xyz, w = original primitive index (bits)
    float4 v1;   // xyz, w unused
    float4 v2;   // xyz, w unused
};

struct Bvh {
    const BvhNode* nodes;
    const BvhTri* tris;
    uint32_t numTris;
    uint32_t* errorFlag;   // bit 0: out-of-range node reference met; bit 1: traversal stack overflow
};

struct Hit {
    float t;
    float b1, b2;
    uint32_t prim;   // original primitive index, 0xFFFFFFFF for a miss
};

// 1 + 2*gamma(3) rounded up: gamma(3) = 3 * 2^-24 / (1 - 3 * 2^-24).
constexpr float kSlabFarScale = 1.00000036f;
// Direction components smaller than 2^-80 in magnitude enter the box test as
// +-2^-80 (sign kept), so the reciprocal stays finite: a ray lying in a box's
// face plane then gets (bound - origin) * (1/d) = 0 instead of 0 * inf = NaN,
// which the min/max of the slab test would turn into a culled box.
constexpr float kTinyDirection = 8.27180613e-25f;

VLRB_HD float slabReciprocal(float d) {
    return 1.0f / (fabsf(d) > kTinyDirection ? d : copysignf(kTinyDirection, d));
}

// Ray set-up of the watertight triangle test: kz is the axis of the largest
// |direction| component (ties to the lower axis), kx and ky the next two in
// cyclic order, swapped when direction[kz] < 0 so the winding is kept; the
// shear (sx, sy, sz) maps the ray to the +z axis of that frame.
struct RayShear {
    int kx, ky, kz;
    float sx, sy, sz;
};

VLRB_HD float axisOf(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

#if defined(__CUDACC__)

__device__ __forceinline__ RayShear rayShear(const V3 &dir) {
    RayShear r;
    const float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
    r.kz = ax >= ay ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1;
    r.ky = r.kx == 2 ? 0 : r.kx + 1;
    const float dz = axisOf(dir.x, dir.y, dir.z, r.kz);
    if (dz < 0.0f) { const int t = r.kx; r.kx = r.ky; r.ky = t; }
    r.sx = __fdiv_rn(axisOf(dir.x, dir.y, dir.z, r.kx), dz);
    r.sy = __fdiv_rn(axisOf(dir.x, dir.y, dir.z, r.ky), dz);
    r.sz = __fdiv_rn(1.0f, dz);
    return r;
}

__device__ __forceinline__ bool slabTest(const float4 &lo, const float4 &hi, const V3 &org, const V3 &invDir,
                                         float tmax, float* tEnter) {
    float tx0 = (lo.x - org.x) * invDir.x, tx1 = (hi.x - org.x) * invDir.x;
    float ty0 = (lo.y - org.y) * invDir.y, ty1 = (hi.y - org.y) * invDir.y;
    float tz0 = (lo.z - org.z) * invDir.z, tz1 = (hi.z - org.z) * invDir.z;
    float tmin = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * kSlabFarScale;
    *tEnter = tmin;
    return tmin <= fminf(tfar, tmax);
}

// Watertight ray/triangle test (Woop, Benthin and Wald 2013) on the ray's
// shear.  Every operation is rounded explicitly (no contraction), so the
// host restatement in the oracle and the tests reproduces t and the
// barycentrics bit for bit.  On a hit with t in (0, tmax): *t, and the
// scaled barycentrics V, W with their denominator det (b1 = V/det weights
// v1, b2 = W/det weights v2; the caller divides only for the hits it keeps).
__device__ __forceinline__ bool triTest(const BvhTri &tr, const V3 &org, const RayShear &r, float tmax, float* t,
                                        float* vOut, float* wOut, float* detOut) {
    // vertices relative to the origin, then on the ray's axes and sheared
    const float a0 = __fsub_rn(tr.v0.x, org.x), a1 = __fsub_rn(tr.v0.y, org.y), a2 = __fsub_rn(tr.v0.z, org.z);
    const float b0 = __fsub_rn(tr.v1.x, org.x), b1 = __fsub_rn(tr.v1.y, org.y), b2 = __fsub_rn(tr.v1.z, org.z);
    const float c0 = __fsub_rn(tr.v2.x, org.x), c1 = __fsub_rn(tr.v2.y, org.y), c2 = __fsub_rn(tr.v2.z, org.z);
    const float az = axisOf(a0, a1, a2, r.kz), bz = axisOf(b0, b1, b2, r.kz), cz = axisOf(c0, c1, c2, r.kz);
    const float Ax = __fsub_rn(axisOf(a0, a1, a2, r.kx), __fmul_rn(r.sx, az));
    const float Ay = __fsub_rn(axisOf(a0, a1, a2, r.ky), __fmul_rn(r.sy, az));
    const float Bx = __fsub_rn(axisOf(b0, b1, b2, r.kx), __fmul_rn(r.sx, bz));
    const float By = __fsub_rn(axisOf(b0, b1, b2, r.ky), __fmul_rn(r.sy, bz));
    const float Cx = __fsub_rn(axisOf(c0, c1, c2, r.kx), __fmul_rn(r.sx, cz));
    const float Cy = __fsub_rn(axisOf(c0, c1, c2, r.ky), __fmul_rn(r.sy, cz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // products of two floats are exact in double: one rounding each
        U = __double2float_rn(__dsub_rn(__dmul_rn(Cx, By), __dmul_rn(Cy, Bx)));
        V = __double2float_rn(__dsub_rn(__dmul_rn(Ax, Cy), __dmul_rn(Ay, Cx)));
        W = __double2float_rn(__dsub_rn(__dmul_rn(Bx, Ay), __dmul_rn(By, Ax)));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(r.sz, az)), __fmul_rn(V, __fmul_rn(r.sz, bz))),
                              __fmul_rn(W, __fmul_rn(r.sz, cz)));
    // Without dividing: t <= 0 when T and det differ in sign (or T is 0);
    // t >= tmax when |T| >= |det| tmax (1 + 2^-21), which the two roundings
    // of the product cannot fake.  Only the remaining hits take the division.
    if (T == 0.0f || (T < 0.0f) != (det < 0.0f)) return false;
    if (fabsf(T) >= __fmul_rn(__fmul_rn(fabsf(det), tmax), 1.00000048f)) return false;
    const float tt = __fdiv_rn(T, det);
    if (!(tt > 0.0f && tt < tmax)) return false;
    *t = tt;
    *vOut = V;
    *wOut = W;
    *detOut = det;
    return true;
}

constexpr int kTraversalStack = 64;

// Accepts every intersection (opaque geometry).  An accept functor that
// reads the barycentrics declares kNeedsBarycentrics = true; otherwise the
// traversal divides for them once, for the hit it returns.
struct AcceptAll {
    static constexpr bool kNeedsBarycentrics = false;
    __device__ __forceinline__ bool operator()(uint32_t, float, float) const { return true; }
};

// Closest hit (anyHit == false) or first hit (anyHit == true) along
// org + t*dir, t in (0, tmax), among the intersections `accept(prim, b1, b2)`
// keeps (the any-hit program's role: an ignored intersection neither ends
// the ray nor shortens it).  Ordered front-to-back descent with a short
// per-thread stack.
template <bool anyHit, class Accept>
__device__ __forceinline__ Hit traceBvhWith(const Bvh &bvh, const V3 &org, const V3 &dir, float tmax,
                                            Accept &accept) {
    Hit h;
    h.t = tmax;
    h.prim = 0xFFFFFFFFu;
    h.b1 = h.b2 = 0.0f;
    if (bvh.numTris == 0) return h;
    V3 invDir(slabReciprocal(dir.x), slabReciprocal(dir.y), slabReciprocal(dir.z));
    const RayShear shear = rayShear(dir);
    int stack[kTraversalStack];
    int sp = 0;
    bool overflow = false;   // reported once after the loop: an atomic inside it halves the speed
    float hitDet = 1.0f;     // denominator of the kept hit's barycentrics (held scaled in h.b1, h.b2)
    int node = bvh.numTris == 1 ? ~0 : 0;
    while (true) {
        // A malformed hierarchy must not send the traversal outside its
        // arrays: record the fault and stop.
        if ((node >= 0 && node >= static_cast<int>(bvh.numTris) - 1) ||
            (node < 0 && (~node) >= static_cast<int>(bvh.numTris))) {
            if (bvh.errorFlag) atomicOr(bvh.errorFlag, 1u);
            break;
        }
        if (node >= 0) {
            const float4* np = reinterpret_cast<const float4*>(bvh.nodes + node);
            float4 lo0 = __ldg(np + 0), hi0 = __ldg(np + 1), lo1 = __ldg(np + 2), hi1 = __ldg(np + 3);
            float t0, t1;
            bool hit0 = slabTest(lo0, hi0, org, invDir, h.t, &t0);
            bool hit1 = slabTest(lo1, hi1, org, invDir, h.t, &t1);
            int c0 = __float_as_int(lo0.w), c1 = __float_as_int(lo1.w);
            if (hit0 && hit1) {
                if (t1 < t0) { int tmp = c0; c0 = c1; c1 = tmp; }
                if (sp < kTraversalStack) stack[sp++] = c1;
                else overflow = true;
                node = c0;
                continue;
            }
            if (hit0) { node = c0; continue; }
            if (hit1) { node = c1; continue; }
        }
        else {
            const float4* tp = reinterpret_cast<const float4*>(bvh.tris + (~node));
            BvhTri tr;
            tr.v0 = __ldg(tp + 0); tr.v1 = __ldg(tp + 1); tr.v2 = __ldg(tp + 2);
            float t, V, W, det;
            if (triTest(tr, org, shear, h.t, &t, &V, &W, &det)) {
                const uint32_t prim = __float_as_uint(tr.v0.w);
                bool keep;
                if constexpr (Accept::kNeedsBarycentrics) keep = accept(prim, __fdiv_rn(V, det), __fdiv_rn(W, det));
                else keep = accept(prim, 0.0f, 0.0f);
                if (keep) {
                    h.t = t;
                    h.prim = prim;
                    h.b1 = V; h.b2 = W; hitDet = det;
                    if (anyHit) break;
                }
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    if (overflow && bvh.errorFlag) atomicOr(bvh.errorFlag, 2u);
    if (h.prim != 0xFFFFFFFFu) {
        h.b1 = __fdiv_rn(h.b1, hitDet);
        h.b2 = __fdiv_rn(h.b2, hitDet);
    }
    return h;
}

template <bool anyHit>
__device__ __forceinline__ Hit traceBvh(const Bvh &bvh, const V3 &org, const V3 &dir, float tmax) {
    AcceptAll all;
    return traceBvhWith<anyHit>(bvh, org, dir, tmax, all);
}

#endif

} // namespace vlrb
