// BSDF shading batch: one thread per query, each query = Meng upsampling of
// the query's RGB albedo and grey IOR, construction of one of the six BSDFs,
// then sample + evaluate + evaluatePDF at the sampled direction.
//
// This translation unit is compiled with -fmad=false so every product and sum
// is rounded exactly like the reference's host build (materials.cu classes
// compiled by g++ for x86-64, which has no fused multiply-add).
#include "tables.cuh"
#include "vlrb_internal.h"

#include <cuda_runtime.h>

namespace vlrb {

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
__device__ __forceinline__ Bsdf buildBatchBsdf(const BsdfBatchArgs &a, int64_t i, const WLS &wls) {
    Bsdf B;
    const ColorMatrices &M = *a.mats;
    const float r = __ldg(a.rgb + 3 * i + 0), g = __ldg(a.rgb + 3 * i + 1), b = __ldg(a.rgb + 3 * i + 2);
    const float eta = __ldg(a.ior + i);
    const float rx = __ldg(a.rough + 2 * i + 0), ry = __ldg(a.rough + 2 * i + 1);
    const uint32_t kind = __ldg(a.mat + i);
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

// Queries arrive in random material order; shading them in that order makes
// every warp execute all six BSDFs.  Each CTA therefore takes a tile of 256
// queries, counting-sorts the tile's indices by material in shared memory,
// and lets thread t shade the t-th query of the sorted tile, so warps run one
// material each except at the few material boundaries.  Inputs and outputs
// stay in their original slots.
constexpr int kBatchTile = 256;

__global__ void __launch_bounds__(kBatchTile) bsdfBatchKernel(BsdfBatchArgs a) {
    __shared__ uint32_t sCount[8];
    __shared__ uint32_t sOffset[8];
    __shared__ uint16_t sOrder[kBatchTile];
    const int64_t numTiles = (a.n + kBatchTile - 1) / kBatchTile;
    for (int64_t tile = blockIdx.x; tile < numTiles; tile += gridDim.x) {
        const int64_t base = tile * kBatchTile;
        if (threadIdx.x < 8) sCount[threadIdx.x] = 0;
        __syncthreads();
        const int64_t mine = base + threadIdx.x;
        uint32_t key = 7;   // slots past the end of the batch sort last
        if (mine < a.n) key = min(__ldg(a.mat + mine), 6u);
        const uint32_t rank = atomicAdd(&sCount[key], 1u);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (int k = 0; k < 8; ++k) { sOffset[k] = run; run += sCount[k]; }
        }
        __syncthreads();
        sOrder[sOffset[key] + rank] = static_cast<uint16_t>(threadIdx.x);
        __syncthreads();
        const int64_t i = base + sOrder[threadIdx.x];
        __syncthreads();
        if (i >= a.n) continue;
        float wlPdf;
        WLS wls = WLS::equalOffsets(__ldg(a.wl + 2 * i + 0), __ldg(a.wl + 2 * i + 1), &wlPdf);
        Bsdf B = buildBatchBsdf(a, i, wls);
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
}

static int g_numSMs = 0;

cudaError_t launchBsdfBatch(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs) {
    if (b.count <= 0)
        return cudaSuccess;
    if (g_numSMs == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_numSMs, cudaDevAttrMultiProcessorCount, dev);
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
    // Grid: enough resident 256-thread CTAs to fill every SM several times
    // over, grid-striding beyond that.
    const int64_t blocksNeeded = (b.count + 255) / 256;
    const int64_t maxBlocks = static_cast<int64_t>(g_numSMs) * 8;
    const int blocks = static_cast<int>(blocksNeeded < maxBlocks ? blocksNeeded : maxBlocks);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernelMs) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    bsdfBatchKernel<<<blocks, 256, 0, stream>>>(a);
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

} // namespace vlrb
