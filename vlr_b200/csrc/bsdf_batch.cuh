// BSDF shading batch kernel, included by two translation units:
// bsdf_batch.cu compiles it with -fmad=false (every product and sum rounded
// like the reference's host build, for query-by-query parity) and
// bsdf_batch_contracted.cu with FMA contraction on, which is how the
// renderers' kernels compile the same BSDF code.  VLRB_BATCH_NS names the
// namespace of each copy.
//
// Each query = Meng upsampling of the query's RGB albedo and grey IOR,
// construction of one of seven BSDFs, then sample + evaluate + evaluatePDF at
// the sampled direction.
#pragma once

#include "tables.cuh"
#include "vlrb_internal.h"

#include <cuda_runtime.h>

#ifndef VLRB_BATCH_NS
#error "define VLRB_BATCH_NS before including bsdf_batch.cuh"
#endif

namespace vlrb {
namespace VLRB_BATCH_NS {


struct BsdfBatchArgs {
    int64_t n;
    const float* wo;
    const uint32_t* mat;
    const float* rough;
    const float* ior;
    const float* rgb;
    const float* metallic;
    const float* u;
    const float* wl;
    float* value;
    float* pdf;
    float* wi;
    float* evalValue;
    float* evalPdf;
    MengTables tables;
    const ColorMatrices* mats;
    UpSpec oneIOR;   // grey IOR 1 (exterior medium of the dielectric)
    UpSpec zeroIOR;  // zero extinction of the conductors
};

// Builds the BSDF of material `kind` from the query's immediate parameters in
// the way the reference's setupBSDF callables do (materials.cu:653-661,
// 776-787, 1220-1240, 1516-1536, 1674-1684, 1959-1978).
// K is the BSDF kind (batchKind maps material ids to kinds).
template <uint32_t K>
__device__ __forceinline__ Bsdf buildBatchBsdf(const BsdfBatchArgs &a, int64_t i, const WLS &wls) {
    Bsdf B;
    const ColorMatrices &M = *a.mats;
    const float r = __ldg(a.rgb + 3 * i + 0), g = __ldg(a.rgb + 3 * i + 1), b = __ldg(a.rgb + 3 * i + 2);
    const float eta = __ldg(a.ior + i);
    const float rx = __ldg(a.rough + 2 * i + 0), ry = __ldg(a.rough + 2 * i + 1);
    constexpr uint32_t kind = K;
    B.kind = kind;
    B.flags = 0;
    B.f0 = B.f1 = B.f2 = 0.0f;
    const float alphaX = fmaxf(0.001f, rx * rx);
    const float alphaY = fmaxf(0.001f, ry * ry);
    switch (kind) {
    case kMatte: {
        UpSpec alb = mengUpsample(a.tables, M, SpType::Reflectance, ColorSp::Rec709, r, g, b);
        B.a = mengEvaluate(a.tables, alb, wls);
        break;
    }
    case kSpecularBRDF: {
        UpSpec alb = mengUpsample(a.tables, M, SpType::Reflectance, ColorSp::Rec709, r, g, b);
        UpSpec e = mengUpsample(a.tables, M, SpType::IOR, ColorSp::Rec709, eta, eta, eta);
        B.a = mengEvaluate(a.tables, alb, wls);
        B.b = mengEvaluate(a.tables, e, wls);
        B.c = mengEvaluate(a.tables, a.zeroIOR, wls);
        break;
    }
    case kMicrofacetBRDF: {
        UpSpec e = mengUpsample(a.tables, M, SpType::IOR, ColorSp::Rec709, eta, eta, eta);
        B.b = mengEvaluate(a.tables, e, wls);
        B.c = mengEvaluate(a.tables, a.zeroIOR, wls);
        B.f0 = alphaX; B.f1 = alphaY; B.f2 = 0.0f;
        break;
    }
    case kMicrofacetBSDF: {
        UpSpec alb = mengUpsample(a.tables, M, SpType::Reflectance, ColorSp::Rec709, r, g, b);
        UpSpec e = mengUpsample(a.tables, M, SpType::IOR, ColorSp::Rec709, eta, eta, eta);
        B.a = mengEvaluate(a.tables, alb, wls);
        B.b = mengEvaluate(a.tables, a.oneIOR, wls);
        B.c = mengEvaluate(a.tables, e, wls);
        B.f0 = alphaX; B.f1 = alphaY; B.f2 = 0.0f;
        break;
    }
    case kLambertianBSDF: {
        UpSpec alb = mengUpsample(a.tables, M, SpType::Reflectance, ColorSp::Rec709, r, g, b);
        B.a = mengEvaluate(a.tables, alb, wls);
        B.f0 = 0.04f;
        break;
    }
    case kSpecularBSDF: {
        // SpecularScatteringSurfaceMaterial_setupBSDF (materials.cu:1046-1058):
        // coefficient, exterior IOR 1, interior IOR, dispersive unless a
        // single wavelength is selected
        UpSpec alb = mengUpsample(a.tables, M, SpType::Reflectance, ColorSp::Rec709, r, g, b);
        UpSpec e = mengUpsample(a.tables, M, SpType::IOR, ColorSp::Rec709, eta, eta, eta);
        B.a = mengEvaluate(a.tables, alb, wls);
        B.b = mengEvaluate(a.tables, a.oneIOR, wls);
        B.c = mengEvaluate(a.tables, e, wls);
        B.flags = wls.single ? 0u : 1u;
        break;
    }
    default: {
        UpSpec alb = mengUpsample(a.tables, M, SpType::Reflectance, ColorSp::Rec709, r, g, b);
        S4 base = mengEvaluate(a.tables, alb, wls);
        const float metal = __ldg(a.metallic + i);
        const float specular = 0.5f;
        B.kind = kUE4;
        B.a = base * (1 - metal);
        B.b = lerpS(0.08f * specular * S4::one(), base, metal);
        B.f0 = fmaxf(0.01f, rx);
        break;
    }
    }
    return B;
}

// One query: sample, then evaluate value and pdf at the sampled direction.
template <uint32_t K>
__device__ __forceinline__ void shadeQuery(const BsdfBatchArgs &a, int64_t i) {
    float wlPdf;
    WLS wls = WLS::equalOffsets(__ldg(a.wl + 2 * i + 0), __ldg(a.wl + 2 * i + 1), &wlPdf);
    Bsdf B = buildBatchBsdf<K>(a, i, wls);
    BsdfQuery q;
    q.dirLocal = V3(__ldg(a.wo + 3 * i + 0), __ldg(a.wo + 3 * i + 1), __ldg(a.wo + 3 * i + 2));
    q.wlHint = wls.selected;
    q.filter = dir::All;
    q.importanceMode = 0;
    const float uc = __ldg(a.u + 3 * i + 0), u0 = __ldg(a.u + 3 * i + 1), u1 = __ldg(a.u + 3 * i + 2);
    BsdfSample s;
    s.dirPDF = 0.0f;
    s.dirLocal = V3(0.0f, 0.0f, 0.0f);
    S4 fs = bsdfSampleInternal(B, q, uc, u0, u1, &s, nullptr);
    float4 v4 = make_float4(0.f, 0.f, 0.f, 0.f), e4 = v4;
    float pdf = 0.0f, epdf = 0.0f;
    V3 wi(0.0f, 0.0f, 0.0f);
    if (s.dirPDF > 0.0f) {
        v4 = make_float4(fs[0], fs[1], fs[2], fs[3]);
        pdf = s.dirPDF;
        wi = s.dirLocal;
        S4 ev = bsdfEvalInternal(B, q, wi, nullptr);
        e4 = make_float4(ev[0], ev[1], ev[2], ev[3]);
        epdf = bsdfPDFInternal(B, q, wi, nullptr);
    }
    reinterpret_cast<float4*>(a.value)[i] = v4;
    a.pdf[i] = pdf;
    a.wi[3 * i + 0] = wi.x;
    a.wi[3 * i + 1] = wi.y;
    a.wi[3 * i + 2] = wi.z;
    reinterpret_cast<float4*>(a.evalValue)[i] = e4;
    a.evalPdf[i] = epdf;
}


// Material id -> BSDF kind: ids 0-4 and 6 are their own kinds (6 is
// SpecularScattering); 5 and every id above 6 build the UE4 BSDF, as the
// reference's default branch does.
__device__ __forceinline__ uint32_t batchKind(uint32_t m) {
    return m < 5u ? m : (m == 6u ? static_cast<uint32_t>(kSpecularBSDF) : static_cast<uint32_t>(kUE4));
}

__device__ __forceinline__ void shadeQueryOfKind(uint32_t kind, const BsdfBatchArgs &a, int64_t i) {
    switch (kind) {
    case kMatte: shadeQuery<kMatte>(a, i); break;
    case kSpecularBRDF: shadeQuery<kSpecularBRDF>(a, i); break;
    case kMicrofacetBRDF: shadeQuery<kMicrofacetBRDF>(a, i); break;
    case kMicrofacetBSDF: shadeQuery<kMicrofacetBSDF>(a, i); break;
    case kLambertianBSDF: shadeQuery<kLambertianBSDF>(a, i); break;
    case kSpecularBSDF: shadeQuery<kSpecularBSDF>(a, i); break;
    default: shadeQuery<kUE4>(a, i); break;
    }
}

// Queries arrive in random material order.  One launch of persistent warps;
// each warp owns an equal contiguous share of the queries (every resident
// warp busy, balanced by count: the kernel is latency-bound, so the number
// of warps in flight matters more than the sort's fill) and works through
// it in tiles of at most kWarpTile queries: for each tile it reads
// the tile's material ids (coalesced), counting-sorts the tile's indices by
// BSDF kind into its own shared-memory list (ballot + popcount, no block
// barrier), each kind's run padded to a multiple of 32, then shades 32 sorted
// queries at a time, so every pass runs one BSDF with full lanes except the
// last of each kind.  Inputs are gathered from the tile's own slots (a few
// KB per input array, so each DRAM sector is fetched once and the other
// queries in it hit L1/L2) and outputs go back to the same slots.  Warps
// never wait for each other, so a warp with slow BSDFs holds up no one.
constexpr int kBatchThreads = 256;
constexpr int kBatchWarps = kBatchThreads / 32;
constexpr int kWarpTile = 512;
constexpr int kWarpTilePerLane = kWarpTile / 32;
constexpr uint32_t kBatchKinds = 7;
constexpr int kWarpSlots = ((kWarpTile + kBatchKinds * 31) + 31) / 32 * 32;
constexpr uint16_t kBatchPad = 0xFFFFu;
constexpr int64_t kMinWarpQueries = 64;   // fewer warps than resident for small batches

__global__ void __launch_bounds__(kBatchThreads, 3) bsdfBatchKernel(BsdfBatchArgs a) {
    __shared__ uint16_t sIdx[kBatchWarps][kWarpSlots];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lanesBelow = (1u << lane) - 1u;
    uint16_t* idx = sIdx[warp];
    const int64_t warpId = static_cast<int64_t>(blockIdx.x) * kBatchWarps + warp;
    const int64_t numWarps = static_cast<int64_t>(gridDim.x) * kBatchWarps;
    // shares in multiples of 8 queries: every share starts on a 32-byte
    // sector of every input and output array (4, 8, 12 and 16 B per query)
    const int64_t per = ((a.n + numWarps - 1) / numWarps + 7) & ~int64_t(7);
    const int64_t start = warpId * per < a.n ? warpId * per : a.n;
    const int64_t end = start + per < a.n ? start + per : a.n;
    for (int64_t base = start; base < end; base += kWarpTile) {
        const int count = static_cast<int>(end - base < kWarpTile ? end - base : kWarpTile);
        // material kinds of this lane's 16 queries, 3 bits each (7 = none)
        uint64_t packed = ~0ull;     // kind 7 (none) in every unread slot
        uint32_t counts[kBatchKinds];
#pragma unroll
        for (uint32_t k = 0; k < kBatchKinds; ++k) counts[k] = 0;
#pragma unroll
        for (int j = 0; j < kWarpTilePerLane; ++j) {
            if (j * 32 >= count) break;
            const int li = j * 32 + static_cast<int>(lane);
            const uint32_t kind = li < count ? batchKind(__ldg(a.mat + base + li)) : kBatchKinds;
            packed &= ~(static_cast<uint64_t>(7u ^ kind) << (3 * j));
#pragma unroll
            for (uint32_t k = 0; k < kBatchKinds; ++k) counts[k] += __popc(__ballot_sync(0xFFFFFFFFu, kind == k));
        }
        uint32_t off[kBatchKinds + 1];
        off[0] = 0;
#pragma unroll
        for (uint32_t k = 0; k < kBatchKinds; ++k) off[k + 1] = off[k] + ((counts[k] + 31u) & ~31u);
        for (int s = static_cast<int>(lane); s < static_cast<int>(off[kBatchKinds]); s += 32) idx[s] = kBatchPad;
        __syncwarp();
        uint32_t fill[kBatchKinds];
#pragma unroll
        for (uint32_t k = 0; k < kBatchKinds; ++k) fill[k] = off[k];
#pragma unroll
        for (int j = 0; j < kWarpTilePerLane; ++j) {
            if (j * 32 >= count) break;
            const uint32_t kind = static_cast<uint32_t>(packed >> (3 * j)) & 7u;
#pragma unroll
            for (uint32_t k = 0; k < kBatchKinds; ++k) {
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, kind == k);
                if (kind == k) idx[fill[k] + __popc(bal & lanesBelow)] = static_cast<uint16_t>(j * 32 + lane);
                fill[k] += __popc(bal);
            }
        }
        __syncwarp();
        const uint32_t tasks = off[kBatchKinds] / 32u;
        uint32_t kind = 0;
        for (uint32_t t = 0; t < tasks; ++t) {
            while (t * 32u >= off[kind + 1]) ++kind;
            const uint16_t li = idx[t * 32u + lane];
            if (li != kBatchPad) shadeQueryOfKind(kind, a, base + li);
        }
        __syncwarp();
    }
}

inline cudaError_t launch(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs) {
    if (b.count <= 0)
        return cudaSuccess;
    static int numSMs = 0, perSM = 0;
    if (numSMs == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, bsdfBatchKernel, kBatchThreads, 0);
        if (perSM < 1) perSM = 1;
    }
    BsdfBatchArgs a;
    a.n = b.count;
    a.wo = b.wo; a.mat = b.material; a.rough = b.roughness; a.ior = b.ior; a.rgb = b.albedo;
    a.metallic = b.metallic; a.u = b.u; a.wl = b.wavelengthU;
    a.value = b.value; a.pdf = b.pdf; a.wi = b.wi; a.evalValue = b.evalValue; a.evalPdf = b.evalPdf;
    a.tables = deviceMengTables();
    a.mats = deviceColorMatrices();
    const ColorMatrices &hm = hostColorMatrices();
    MengTables ht = hostMengTables();
    a.oneIOR = mengUpsample(ht, hm, SpType::IOR, ColorSp::Rec709, 1.0f, 1.0f, 1.0f);
    a.zeroIOR = mengUpsample(ht, hm, SpType::IOR, ColorSp::Rec709, 0.0f, 0.0f, 0.0f);
    // Persistent grid: every resident CTA slot of every SM (fewer for small
    // batches, at least kMinWarpQueries queries per warp).
    const int64_t resident = static_cast<int64_t>(numSMs) * perSM;
    const int64_t warpsWanted = (b.count + kMinWarpQueries - 1) / kMinWarpQueries;
    const int64_t needed = (warpsWanted + kBatchWarps - 1) / kBatchWarps;
    const int blocks = static_cast<int>(needed < resident ? needed : resident);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernelMs) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    bsdfBatchKernel<<<blocks, kBatchThreads, 0, stream>>>(a);
    cudaError_t err = cudaGetLastError();
    if (kernelMs) {
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(kernelMs, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return err;
}

} // namespace VLRB_BATCH_NS
} // namespace vlrb
