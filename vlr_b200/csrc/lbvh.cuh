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
//   tris:   N triangles in BVH (sorted) order, 48 B each: v0, e1 = v1-v0,
//           e2 = v2-v0 plus the original primitive index in v0.w's bits.
// Child references >= 0 are internal nodes; ~index (negative) are leaves.
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
    float4 e1;
    float4 e2;
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

#if defined(__CUDACC__)

__device__ __forceinline__ bool slabTest(const float4 &lo, const float4 &hi, const V3 &org, const V3 &invDir,
                                         float tmax, float* tEnter) {
    float tx0 = (lo.x - org.x) * invDir.x, tx1 = (hi.x - org.x) * invDir.x;
    float ty0 = (lo.y - org.y) * invDir.y, ty1 = (hi.y - org.y) * invDir.y;
    float tz0 = (lo.z - org.z) * invDir.z, tz1 = (hi.z - org.z) * invDir.z;
    float tmin = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tm = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    *tEnter = tmin;
    return tmin <= tm;
}

// Moller-Trumbore ray/triangle test with the edges precomputed.
__device__ __forceinline__ bool triTest(const BvhTri &tr, const V3 &org, const V3 &dir, float tmax,
                                        float* t, float* b1, float* b2) {
    V3 e1(tr.e1.x, tr.e1.y, tr.e1.z), e2(tr.e2.x, tr.e2.y, tr.e2.z);
    V3 p = cross(dir, e2);
    float det = dot(e1, p);
    if (det == 0.0f) return false;
    float inv = 1.0f / det;
    V3 s = org - V3(tr.v0.x, tr.v0.y, tr.v0.z);
    float u = dot(s, p) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    V3 q = cross(s, e1);
    float v = dot(dir, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    float tt = dot(e2, q) * inv;
    if (!(tt > 0.0f && tt < tmax)) return false;
    *t = tt; *b1 = u; *b2 = v;
    return true;
}

constexpr int kTraversalStack = 64;

// Accepts every intersection (opaque geometry).
struct AcceptAll {
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
    V3 invDir(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    int stack[kTraversalStack];
    int sp = 0;
    bool overflow = false;   // reported once after the loop: an atomic inside it halves the speed
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
            tr.v0 = __ldg(tp + 0); tr.e1 = __ldg(tp + 1); tr.e2 = __ldg(tp + 2);
            float t, b1, b2;
            if (triTest(tr, org, dir, h.t, &t, &b1, &b2) && accept(__float_as_uint(tr.v0.w), b1, b2)) {
                h.t = t; h.b1 = b1; h.b2 = b2;
                h.prim = __float_as_uint(tr.v0.w);
                if (anyHit) return h;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    if (overflow && bvh.errorFlag) atomicOr(bvh.errorFlag, 2u);
    return h;
}

template <bool anyHit>
__device__ __forceinline__ Hit traceBvh(const Bvh &bvh, const V3 &org, const V3 &dir, float tmax) {
    AcceptAll all;
    return traceBvhWith<anyHit>(bvh, org, dir, tmax, all);
}

#endif

} // namespace vlrb
