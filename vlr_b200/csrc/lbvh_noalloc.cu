// LBVH build that allocates no device memory: the build's scratch is a
// file-scope static device array, so the call needs neither cudaMalloc nor
// any allocating library routine.
//
// Who needs it: a caller that must not allocate while it runs, such as a
// renderer rebuilding a small dynamic mesh's BVH every frame from inside a
// fixed per-frame memory budget, or an embedding application whose device
// memory is owned by its own pool (a cudaMalloc there would bypass the pool's
// accounting, and may stall every stream of the device while it runs).  The
// regular entry (vlrbBvhBuildHost) allocates its scratch and outputs per call.
//
// Limits and rules:
//   * at most kNoAllocMaxTriangles triangles per call (the static scratch is
//     sized for exactly that many; larger builds are rejected);
//   * the scratch is one buffer per device: two calls on the same device must
//     not overlap in time (same stream, or synchronise between them);
//     overlapping calls race on the scratch and corrupt each other's result;
//   * no scratch byte needs an initial value: the build itself clears, on the
//     caller's stream, everything it accumulates into (centroid bounds,
//     parent links, arrival counters) before using it;
//   * the first call on a device performs a one-time set-up for that device
//     (the symbol lookup below, which makes the runtime load this file's
//     device code);
//   * the looked-up address is kept for the life of the process, so a
//     device reset (cudaDeviceReset) between calls is not supported: the
//     reset unloads the module and the kept address no longer points at it.
#include "vlrb_internal.h"
#include "lbvh_build.h"

#include <cstdio>
#include <exception>
#include <mutex>

namespace {

constexpr uint32_t kNoAllocMaxTriangles = VLRB_BVH_NO_ALLOC_MAX_TRIANGLES;

// Same accounting as lbvhScratchBytes(), evaluated at the maximum size.
constexpr size_t a256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kSortTileItems = 256 * 16;
constexpr size_t kMaxTiles = (kNoAllocMaxTriangles + kSortTileItems - 1) / kSortTileItems;
constexpr size_t kScratchBytes = a256(6 * 4) + 4 * a256(size_t(kNoAllocMaxTriangles) * 4) +
                                 a256(16 * kMaxTiles * 4) + 3 * a256(size_t(kNoAllocMaxTriangles) * 4) +
                                 a256(size_t(kNoAllocMaxTriangles) * 24);

static __device__ __align__(256) unsigned char g_bvhScratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
void* g_scratchOfDevice[kMaxDevices] = {};

// Device address of g_bvhScratch on the current device, looked up once.
cudaError_t scratchForCurrentDevice(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchOfDevice[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_bvhScratch);
        if (e != cudaSuccess) return e;
        g_scratchOfDevice[dev] = p;
    }
    *out = g_scratchOfDevice[dev];
    return cudaSuccess;
}

} // namespace

extern "C" VLRResult vlrbBvhBuildNoAlloc(const float* triVerts, uint32_t n, uint32_t* sortedCodes,
                                         uint32_t* sortedPrims, int32_t* children, float* nodeBoxes,
                                         void* nodes, void* tris, CUstream stream) {
    if (n > kNoAllocMaxTriangles) {
        std::fprintf(stderr, "vlrbBvhBuildNoAlloc: %u triangles exceed the static scratch limit of %u\n", n,
                     kNoAllocMaxTriangles);
        return VLRResult_InvalidArgument;
    }
    if (n == 0) return VLRResult_NoError;
    if (!triVerts || !sortedCodes || !sortedPrims || !tris || (n > 1 && (!children || !nodeBoxes || !nodes)))
        return VLRResult_InvalidArgument;
    if (vlrb::lbvhScratchBytes(n) > kScratchBytes) return VLRResult_InternalError;
    try {
        void* scratch = nullptr;
        cudaError_t e = scratchForCurrentDevice(&scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "vlrbBvhBuildNoAlloc: scratch set-up failed: %s\n", cudaGetErrorString(e));
            return VLRResult_InternalError;
        }
        vlrb::LbvhOutput out{ sortedCodes, sortedPrims, children, nodeBoxes,
                              static_cast<vlrb::BvhNode*>(nodes), static_cast<vlrb::BvhTri*>(tris) };
        vlrb::lbvhBuild(triVerts, n, scratch, &out, reinterpret_cast<cudaStream_t>(stream));
        return VLRResult_NoError;
    }
    catch (const std::exception &ex) {
        std::fprintf(stderr, "vlrbBvhBuildNoAlloc: %s\n", ex.what());
        return VLRResult_InternalError;
    }
}
