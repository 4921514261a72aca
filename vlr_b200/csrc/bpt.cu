// LVC-BPT renderer (light-vertex cache bidirectional path tracing).
#include "bpt.cuh"

#include <stdexcept>

namespace vlrb {

namespace {
inline size_t a256(size_t x) { return (x + 255) & ~size_t(255); }
}

size_t bptBufferBytes(uint32_t numPaths, uint32_t cacheCapacity) {
    return pathBufferBytes(numPaths) + a256(size_t(cacheCapacity) * sizeof(LightVertex)) + a256(16);
}

void carveBptBuffers(void* base, uint32_t numPaths, uint32_t cacheCapacity, PathBuffers* lightPaths, BptBuffers* bb) {
    char* s = static_cast<char*>(base);
    carvePathBuffers(s, numPaths, lightPaths);
    s += pathBufferBytes(numPaths);
    bb->cache = reinterpret_cast<LightVertex*>(s);
    s += a256(size_t(cacheCapacity) * sizeof(LightVertex));
    bb->counters = reinterpret_cast<uint32_t*>(s);
    bb->capacity = cacheCapacity;
}

void bptRenderLaunch(const SceneGPU &, const PathBuffers &, const PathBuffers &, const BptBuffers &, const Film &,
                     const FrameParams &, uint32_t, const WLS &, float, int, cudaStream_t) {
    throw std::runtime_error("LVC-BPT renderer not available in this build");
}

} // namespace vlrb
