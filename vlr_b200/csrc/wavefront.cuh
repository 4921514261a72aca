// Device helpers shared by the wavefront integrators (path tracer, LVC-BPT).
#pragma once

#include "pt.cuh"

namespace vlrb {

__device__ __forceinline__ uint32_t* bounceCounters(const PathBuffers &pb, uint32_t b) {
    return pb.counters + b * kCountersPerBounce;
}

// Warp-aggregated queue append: lanes appending to the same queue share one
// atomic; returns this lane's slot.
__device__ __forceinline__ uint32_t appendSlot(uint32_t* counter, uint32_t key) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (static_cast<int>(lane) == leader)
        base = atomicAdd(counter, static_cast<uint32_t>(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

__device__ __forceinline__ S4 toS4(const float4 &v) { S4 s; s[0] = v.x; s[1] = v.y; s[2] = v.z; s[3] = v.w; return s; }
__device__ __forceinline__ float4 toF4(const S4 &s) { return make_float4(s[0], s[1], s[2], s[3]); }

// Bin a 4-wavelength value into the 16 FP64 film strata of one pixel
// (spectrum_types.h:674-684); atomic when several paths share a pixel.
__device__ __forceinline__ void filmAdd(double* strata, const float lam[4], const S4 &c) {
    const float recBinWidth = kNumStrata / (kWavelengthHigh - kWavelengthLow);
    for (int i = 0; i < 4; ++i) {
        uint32_t bin = vmin<uint32_t>(static_cast<uint32_t>((lam[i] - kWavelengthLow) /
                                      (kWavelengthHigh - kWavelengthLow) * kNumStrata), kNumStrata - 1);
        float v = c[i] * recBinWidth;
        if (v != 0.0f) atomicAdd(strata + bin, static_cast<double>(v));
    }
}

} // namespace vlrb
