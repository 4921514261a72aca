// Light-vertex-cache bidirectional path tracer (LVC-BPT): device buffers and
// host launch interface.
#pragma once

#include "pt.cuh"

namespace vlrb {

// One cached light-subpath vertex (shared/kernel_common.h:522-538), stored
// with its full shading frame so a connection needs no vertex gathers:
// 7 x 16 = 112 bytes.
struct LightVertex {
    float4 posMat;        // world position, material index (bits)
    float4 nrmFlags;      // shading normal, flags (bits): 1 wlSelected, 2 deltaSampled,
                          // 4 prevDeltaSampled, 8 atInfinity, bits 8-23 pathLength
    float4 tanGeom;       // shading tangent, geometry instance (bits)
    float4 gnConv;        // geometric normal, backwardConversionFactor
    float4 flux;          // light-subpath throughput, 4 wavelengths
    float4 dirInPdf;      // incoming direction in the shading frame, probDensity
    float4 misPdfs;       // prevProbDensity, secondPrevPartialDenomMisWeight, secondPrevProbRatioToFirst, -
    float4 texCoord;      // texture coordinates (u, v), -, -
};

// Per-path bidirectional MIS bookkeeping (the light and eye path payloads of
// shared/light_transport_common.h:61-129), structure of arrays.
struct BptExtra {
    float* probDensity;
    float* prevProbDensity;
    float* secondPrevPartial;   // secondPrevPartialDenomMisWeight
    float* secondPrevRatio;     // secondPrevProbRatioToFirst (light paths)
    float* cosTerm;
    float* prevRevAreaPDF;
};

struct BptBuffers {
    LightVertex* cache;
    uint32_t capacity;
    uint32_t* counters;    // [0] vertices stored, [1] appends dropped (cache full)
    BptExtra light, eye;
};

size_t bptBufferBytes(uint32_t numLightPaths, uint32_t numEyePaths, uint32_t cacheCapacity);
void carveBptBuffers(void* base, uint32_t numLightPaths, uint32_t numEyePaths, uint32_t cacheCapacity,
                     PathBuffers* lightPaths, BptBuffers* bb);

// One LVC-BPT frame: light subpaths fill the cache, then one eye subpath per
// pixel connects to it.  All paths share the frame's wavelength samples.
// Light tracing (light_tracing.cu:49-263): `frames` frames of numLightPaths
// light subpaths each, in one launch, with wavelength samples of their own;
// each vertex connects to a lens sample and splats to the film.  The path
// buffers and `connections` (ltConnectionBytes) hold numLightPaths x frames.
size_t ltConnectionBytes(uint32_t numPaths);
void ltRenderLaunch(const SceneGPU &scene, const PathBuffers &lightPaths, void* connections, const Film &film,
                    const FrameParams &fp, uint32_t numLightPaths, uint32_t frames, int numSMs, cudaStream_t stream,
                    StageTimer* timer);

void bptRenderLaunch(const SceneGPU &scene, const PathBuffers &eyePaths, const PathBuffers &lightPaths,
                     const BptBuffers &bb, const Film &film, const FrameParams &fp, uint32_t numLightPaths,
                     const WLS &commonWls, float wlPdf, int numSMs, cudaStream_t stream, StageTimer* timer);

} // namespace vlrb
