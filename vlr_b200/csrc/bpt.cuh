// Light-vertex-cache bidirectional path tracer (LVC-BPT): device buffers and
// host launch interface.
#pragma once

#include "pt.cuh"

namespace vlrb {

// One cached light-subpath vertex (shared/kernel_common.h:522-538), 80 bytes.
struct LightVertex {
    float4 posPrim;        // world position, primitive index (bits)
    float4 flux;           // 4-wavelength throughput of the light subpath
    float4 dirInLocalB1;   // incoming direction in the shading frame, barycentric b1 in w
    float4 pdfs;           // probDensity, prevProbDensity, secondPrevPartialDenomMisWeight, secondPrevProbRatioToFirst
    float backwardConversionFactor;
    float b2;
    uint32_t flags;        // bit0 wlSelected, bit1 deltaSampled, bit2 prevDeltaSampled, bits 8-23 pathLength
    uint32_t geomInst;
};

struct BptBuffers {
    LightVertex* cache;
    uint32_t capacity;
    uint32_t* counters;    // [0] vertices stored, [1] overflow count
};

} // namespace vlrb
