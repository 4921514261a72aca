// LBVH construction entry points (implemented in lbvh.cu).
#pragma once

#include "lbvh.cuh"
#include <cuda_runtime.h>

namespace vlrb {

// Caller-owned device outputs for a build over n triangles.
struct LbvhOutput {
    uint32_t* sortedCodes;   // n   Morton codes in BVH order
    uint32_t* sortedPrims;   // n   original primitive index per sorted slot
    int32_t* children;       // 2(n-1) child refs (>= 0 internal, ~i leaf)
    float* nodeBoxes;        // 6(n-1) box of each internal node (lo, hi)
    BvhNode* nodes;          // n-1 traversal nodes
    BvhTri* tris;            // n   triangles in sorted order
};

// Device scratch the build needs for n triangles.
size_t lbvhScratchBytes(uint32_t n);

// verts: n triangles x 3 vertices x xyz, device memory.  Enqueued on stream.
void lbvhBuild(const float* verts, uint32_t n, void* scratch, LbvhOutput* out, cudaStream_t stream);

// Treelet restructuring of a built hierarchy in place (children, nodeBoxes and
// nodes change; codes, prims and tris do not): `rounds` bottom-up passes with
// treelets of 7 leaves rooted at nodes over >= 7, 14, 28, ... triangles.
// restructuredDev (device, optional) receives the number of treelets changed.
size_t lbvhOptimizeScratchBytes(uint32_t n);
void lbvhOptimize(uint32_t n, uint32_t rounds, void* scratch, LbvhOutput* out, uint32_t* restructuredDev,
                  cudaStream_t stream);

} // namespace vlrb
