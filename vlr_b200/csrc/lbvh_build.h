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

// Largest number of internal nodes on a root-to-leaf path of the hierarchy
// in `children` (synchronises `stream`).  scratch: lbvhOptimizeScratchBytes(n).
uint32_t lbvhMaxLeafDepth(uint32_t n, const int32_t* children, void* scratch, cudaStream_t stream);

// The hierarchy the traversal walks: lbvhBuild, then `rounds` of
// lbvhOptimize; if restructuring left a leaf deeper than kTraversalStack
// levels, the plain LBVH is built again instead.  Its depth is bounded by the
// key: each level of the Karras hierarchy splits at a longer common prefix of
// the 30-bit Morton code extended by the 32-bit index, so no path holds more
// than 62 internal nodes and the traversal stack (one entry per level) cannot
// overflow.  Returns the maximum leaf depth (synchronises `stream`).
size_t lbvhTraversableScratchBytes(uint32_t n);
uint32_t lbvhBuildTraversable(const float* verts, uint32_t n, uint32_t rounds, void* scratch, LbvhOutput* out,
                              uint32_t* restructuredDev, cudaStream_t stream);

} // namespace vlrb
