// BSDF shading batch: each query = Meng upsampling of the query's RGB albedo
// and grey IOR, construction of one of the six BSDFs, then sample + evaluate
// + evaluatePDF at the sampled direction.
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
// K is the material id (ids above kUE4 build the UE4 BSDF, as the
// reference's default branch does).
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

// Queries arrive in random material order.  One launch per material: each
// warp scans the material ids 32 at a time, collects the indices of its
// material in shared memory (ballot + popcount, no block barriers) and
// shades them 32 at a time, so every warp runs one BSDF with full lanes and
// each launch's code is one BSDF's, which keeps the instruction cache warm.
// Inputs and outputs stay in their original slots.
constexpr int kBatchThreads = 256;

template <uint32_t K>
__global__ void __launch_bounds__(kBatchThreads) bsdfBatchKernel(BsdfBatchArgs a) {
    __shared__ uint32_t sIdx[kBatchThreads / 32][64];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t warpId = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t numWarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    uint32_t pending = 0;
    for (int64_t base = warpId * 32; base < a.n; base += numWarps * 32) {
        const int64_t i = base + lane;
        bool match = false;
        if (i < a.n) {
            const uint32_t m = __ldg(a.mat + i);
            match = K == kUE4 ? m >= kUE4 : m == K;
        }
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, match);
        if (match) sIdx[w][pending + __popc(bal & ((1u << lane) - 1u))] = static_cast<uint32_t>(i);
        pending += __popc(bal);
        __syncwarp();
        if (pending >= 32) {
            shadeQuery<K>(a, sIdx[w][lane]);
            __syncwarp();
            pending -= 32;
            if (lane < pending) sIdx[w][lane] = sIdx[w][32 + lane];
            __syncwarp();
        }
    }
    if (lane < pending) shadeQuery<K>(a, sIdx[w][lane]);
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
    const int64_t blocksNeeded = (b.count + kBatchThreads - 1) / kBatchThreads;
    const int64_t maxBlocks = static_cast<int64_t>(g_numSMs) * 8;
    const int blocks = static_cast<int>(blocksNeeded < maxBlocks ? blocksNeeded : maxBlocks);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (kernelMs) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    // indices are kept as 32-bit in shared memory: chunks of at most 2^31 queries
    const int64_t chunk = int64_t(1) << 31;
    for (int64_t first = 0; first < b.count; first += chunk) {
        BsdfBatchArgs c = a;
        c.n = b.count - first < chunk ? b.count - first : chunk;
        c.wo += 3 * first; c.mat += first; c.rough += 2 * first; c.ior += first; c.rgb += 3 * first;
        c.metallic += first; c.u += 3 * first; c.wl += 2 * first;
        c.value += 4 * first; c.pdf += first; c.wi += 3 * first; c.evalValue += 4 * first; c.evalPdf += first;
        bsdfBatchKernel<kMatte><<<blocks, kBatchThreads, 0, stream>>>(c);
        bsdfBatchKernel<kSpecularBRDF><<<blocks, kBatchThreads, 0, stream>>>(c);
        bsdfBatchKernel<kMicrofacetBRDF><<<blocks, kBatchThreads, 0, stream>>>(c);
        bsdfBatchKernel<kMicrofacetBSDF><<<blocks, kBatchThreads, 0, stream>>>(c);
        bsdfBatchKernel<kLambertianBSDF><<<blocks, kBatchThreads, 0, stream>>>(c);
        bsdfBatchKernel<kUE4><<<blocks, kBatchThreads, 0, stream>>>(c);
    }
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
