// C entry points of the BSDF shading batch (include/vlrb.h).
#include "vlrb_internal.h"
#include "lbvh_build.h"

#include <algorithm>
#include <cstdio>
#include <exception>
#include <map>
#include <mutex>

namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes > 0 ? bytes : 1); }
};

bool validBatch(const VLRBBsdfBatch* b) {
    if (!b || b->count < 0)
        return false;
    if (b->count == 0)
        return true;
    return b->wo && b->material && b->roughness && b->ior && b->albedo && b->metallic && b->u &&
           b->wavelengthU && b->value && b->pdf && b->wi && b->evalValue && b->evalPdf;
}

} // namespace

extern "C" const char* vlrbVersion(void) {
    return "vlr_b200 sm_100a";
}

extern "C" VLRResult vlrbBsdfBatch(const VLRBBsdfBatch* batch, CUstream stream) {
    if (!validBatch(batch))
        return VLRResult_InvalidArgument;
    try {
        cudaError_t e = vlrb::launchBsdfBatch(*batch, reinterpret_cast<cudaStream_t>(stream), nullptr);
        return e == cudaSuccess ? VLRResult_NoError : VLRResult_InternalError;
    }
    catch (const std::exception &ex) {
        std::fprintf(stderr, "vlrbBsdfBatch: %s\n", ex.what());
        return VLRResult_InternalError;
    }
}

// Device side of the host-buffer entry, kept per device between calls (grown
// to the largest batch, never freed: the driver releases it at exit), with
// its own stream and timing events.  Calls are serialised by the mutex.
struct HostBatchState {
    void* in = nullptr;
    void* out = nullptr;
    size_t inBytes = 0, outBytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
};

static std::mutex g_hostBatchMutex;
static std::map<int, HostBatchState> g_hostBatch;

static cudaError_t growDevice(void** p, size_t* have, size_t want) {
    if (*have >= want) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    const cudaError_t e = cudaMalloc(p, want);
    if (e == cudaSuccess) *have = want;
    return e;
}

static VLRResult bsdfBatchHost(const VLRBBsdfBatch* batch, uint32_t flags, float* kernelMs) {
    if (!validBatch(batch) || (flags & ~VLRB_BSDF_BATCH_CONTRACTED))
        return VLRResult_InvalidArgument;
    if (batch->count == 0) {
        if (kernelMs) *kernelMs = 0.0f;
        return VLRResult_NoError;
    }
    try {
        const size_t n = static_cast<size_t>(batch->count);
        std::lock_guard<std::mutex> lock(g_hostBatchMutex);
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess) return VLRResult_InternalError;
        HostBatchState &st = g_hostBatch[device];
        if (!st.stream) {
            if (cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreate(&st.e0) != cudaSuccess || cudaEventCreate(&st.e1) != cudaSuccess)
                return VLRResult_InternalError;
        }
        // Inputs: wo 3, material 1 (u32), roughness 2, ior 1, albedo 3,
        // metallic 1, u 3, wavelengthU 2  -> 16 words per query.
        // Outputs: value 4, pdf 1, wi 3, evalValue 4, evalPdf 1 -> 13 words.
        if (growDevice(&st.in, &st.inBytes, n * 16 * 4) != cudaSuccess ||
            growDevice(&st.out, &st.outBytes, n * 13 * 4) != cudaSuccess)
            return VLRResult_InternalError;
        char* ib = static_cast<char*>(st.in);
        char* ob = static_cast<char*>(st.out);
        cudaStream_t s = st.stream;
        VLRBBsdfBatch d = *batch;
        size_t off = 0;
        cudaError_t e = cudaSuccess;
        auto place = [&](const void* src, size_t words, const void** dst) {
            *dst = ib + off;
            if (e == cudaSuccess) e = cudaMemcpyAsync(ib + off, src, n * words * 4, cudaMemcpyHostToDevice, s);
            off += n * words * 4;
        };
        place(batch->wo, 3, reinterpret_cast<const void**>(&d.wo));
        place(batch->material, 1, reinterpret_cast<const void**>(&d.material));
        place(batch->roughness, 2, reinterpret_cast<const void**>(&d.roughness));
        place(batch->ior, 1, reinterpret_cast<const void**>(&d.ior));
        place(batch->albedo, 3, reinterpret_cast<const void**>(&d.albedo));
        place(batch->metallic, 1, reinterpret_cast<const void**>(&d.metallic));
        place(batch->u, 3, reinterpret_cast<const void**>(&d.u));
        place(batch->wavelengthU, 2, reinterpret_cast<const void**>(&d.wavelengthU));
        // value first so its float4 stores stay 16-byte aligned.
        d.value = reinterpret_cast<float*>(ob);
        d.evalValue = reinterpret_cast<float*>(ob + n * 16);
        d.pdf = reinterpret_cast<float*>(ob + n * 32);
        d.wi = reinterpret_cast<float*>(ob + n * 36);
        d.evalPdf = reinterpret_cast<float*>(ob + n * 48);
        if (e != cudaSuccess) return VLRResult_InternalError;
        cudaEventRecord(st.e0, s);
        e = (flags & VLRB_BSDF_BATCH_CONTRACTED) ? vlrb::launchBsdfBatchContracted(d, s, nullptr)
                                                 : vlrb::launchBsdfBatch(d, s, nullptr);
        cudaEventRecord(st.e1, s);
        if (e != cudaSuccess)
            return VLRResult_InternalError;
        const struct { void* dst; const void* src; size_t bytes; } back[5] = {
            { batch->value, d.value, n * 16 }, { batch->evalValue, d.evalValue, n * 16 },
            { batch->pdf, d.pdf, n * 4 }, { batch->wi, d.wi, n * 12 }, { batch->evalPdf, d.evalPdf, n * 4 } };
        for (const auto &b : back)
            if (e == cudaSuccess) e = cudaMemcpyAsync(b.dst, b.src, b.bytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e == cudaSuccess && kernelMs) e = cudaEventElapsedTime(kernelMs, st.e0, st.e1);
        return e == cudaSuccess ? VLRResult_NoError : VLRResult_InternalError;
    }
    catch (const std::exception &ex) {
        std::fprintf(stderr, "vlrbBsdfBatchHost: %s\n", ex.what());
        return VLRResult_InternalError;
    }
}

extern "C" VLRResult vlrbBsdfBatchHost(const VLRBBsdfBatch* batch, float* kernelMs) {
    return bsdfBatchHost(batch, 0u, kernelMs);
}

extern "C" VLRResult vlrbBsdfBatchHostEx(const VLRBBsdfBatch* batch, uint32_t flags, float* kernelMs) {
    return bsdfBatchHost(batch, flags, kernelMs);
}

static VLRResult bvhBuildHost(const float* triVerts, uint32_t n, uint32_t treeletRounds, uint32_t* sortedCodes,
                              uint32_t* sortedPrims, int32_t* children, float* nodeBoxes, uint32_t* restructured,
                              float* buildMs) {
    if (!triVerts || !sortedCodes || !sortedPrims || (n > 1 && (!children || !nodeBoxes)))
        return VLRResult_InvalidArgument;
    if (restructured) *restructured = 0;
    if (n == 0) return VLRResult_NoError;
    try {
        const size_t N = n;
        auto a256 = [](size_t x) { return (x + 255) & ~size_t(255); };
        const size_t sizes[7] = { N * 36, N * 4, N * 4, N * 8, N * 24, N * sizeof(vlrb::BvhNode), N * sizeof(vlrb::BvhTri) };
        size_t off[7], total = 0;
        for (int i = 0; i < 7; ++i) { off[i] = total; total += a256(sizes[i]); }
        DevBuf out, scratch, optScratch;
        if (out.alloc(total) != cudaSuccess || scratch.alloc(vlrb::lbvhScratchBytes(n)) != cudaSuccess ||
            optScratch.alloc(vlrb::lbvhOptimizeScratchBytes(n) + 256) != cudaSuccess)
            return VLRResult_InternalError;
        uint32_t* dRestructured = reinterpret_cast<uint32_t*>(static_cast<char*>(optScratch.p) +
                                                              vlrb::lbvhOptimizeScratchBytes(n));
        char* b = static_cast<char*>(out.p);
        cudaMemcpy(b + off[0], triVerts, N * 36, cudaMemcpyHostToDevice);
        vlrb::LbvhOutput lo{ reinterpret_cast<uint32_t*>(b + off[1]), reinterpret_cast<uint32_t*>(b + off[2]),
                             reinterpret_cast<int32_t*>(b + off[3]), reinterpret_cast<float*>(b + off[4]),
                             reinterpret_cast<vlrb::BvhNode*>(b + off[5]), reinterpret_cast<vlrb::BvhTri*>(b + off[6]) };
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, nullptr);
        vlrb::lbvhBuild(reinterpret_cast<const float*>(b + off[0]), n, scratch.p, &lo, nullptr);
        if (treeletRounds > 0) vlrb::lbvhOptimize(n, treeletRounds, optScratch.p, &lo, dRestructured, nullptr);
        cudaEventRecord(e1, nullptr);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (buildMs) *buildMs = ms;
        cudaMemcpy(sortedCodes, lo.sortedCodes, N * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(sortedPrims, lo.sortedPrims, N * 4, cudaMemcpyDeviceToHost);
        if (n > 1) {
            cudaMemcpy(children, lo.children, (N - 1) * 8, cudaMemcpyDeviceToHost);
            cudaMemcpy(nodeBoxes, lo.nodeBoxes, (N - 1) * 24, cudaMemcpyDeviceToHost);
        }
        if (restructured && treeletRounds > 0 && n >= 3)
            cudaMemcpy(restructured, dRestructured, 4, cudaMemcpyDeviceToHost);
        return cudaGetLastError() == cudaSuccess ? VLRResult_NoError : VLRResult_InternalError;
    }
    catch (const std::exception &ex) {
        std::fprintf(stderr, "vlrbBvhBuildHost: %s\n", ex.what());
        return VLRResult_InternalError;
    }
}

namespace {
__global__ void traceRaysKernel(vlrb::Bvh bvh, const float4* rays, uint32_t count, bool anyHit, float4* hits) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float4 o = rays[2 * i], d = rays[2 * i + 1];
        const vlrb::V3 org(o.x, o.y, o.z), dir(d.x, d.y, d.z);
        const vlrb::Hit h = anyHit ? vlrb::traceBvh<true>(bvh, org, dir, o.w) : vlrb::traceBvh<false>(bvh, org, dir, o.w);
        hits[i] = make_float4(h.t, h.b1, h.b2, __uint_as_float(h.prim));
    }
}
} // namespace

extern "C" VLRResult vlrbTraceRaysHost(const float* triVerts, uint32_t n, uint32_t treeletRounds, const float* rays,
                                       uint32_t count, uint32_t anyHit, float* hits, float* kernelMs) {
    if (!triVerts || n == 0 || (count > 0 && (!rays || !hits)) || treeletRounds > 8) return VLRResult_InvalidArgument;
    try {
        const size_t N = n;
        auto a256 = [](size_t x) { return (x + 255) & ~size_t(255); };
        const size_t sizes[9] = { N * 36, N * 4, N * 4, N * 8, N * 24, N * sizeof(vlrb::BvhNode),
                                  N * sizeof(vlrb::BvhTri), size_t(count) * 32 + 16, size_t(count) * 16 + 16 };
        size_t off[10], total = 0;
        for (int i = 0; i < 9; ++i) { off[i] = total; total += a256(sizes[i]); }
        off[9] = total;
        total += 256;
        const size_t scratchBytes = vlrb::lbvhTraversableScratchBytes(n);
        DevBuf out, scratch;
        if (out.alloc(total) != cudaSuccess || scratch.alloc(scratchBytes) != cudaSuccess)
            return VLRResult_InternalError;
        char* b = static_cast<char*>(out.p);
        cudaMemset(b + off[9], 0, 256);
        cudaMemcpy(b + off[0], triVerts, N * 36, cudaMemcpyHostToDevice);
        if (count) cudaMemcpy(b + off[7], rays, size_t(count) * 32, cudaMemcpyHostToDevice);
        vlrb::LbvhOutput lo{ reinterpret_cast<uint32_t*>(b + off[1]), reinterpret_cast<uint32_t*>(b + off[2]),
                             reinterpret_cast<int32_t*>(b + off[3]), reinterpret_cast<float*>(b + off[4]),
                             reinterpret_cast<vlrb::BvhNode*>(b + off[5]), reinterpret_cast<vlrb::BvhTri*>(b + off[6]) };
        uint32_t* flags = reinterpret_cast<uint32_t*>(b + off[9]);
        vlrb::lbvhBuildTraversable(reinterpret_cast<const float*>(b + off[0]), n, treeletRounds, scratch.p, &lo,
                                   nullptr, nullptr);
        const vlrb::Bvh bvh{ lo.nodes, lo.tris, n, flags };
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, nullptr);
        if (count) {
            const uint32_t blocks = std::min<uint32_t>((count + 255) / 256, 148u * 16u);
            traceRaysKernel<<<blocks, 256>>>(bvh, reinterpret_cast<const float4*>(b + off[7]), count, anyHit != 0,
                                             reinterpret_cast<float4*>(b + off[8]));
        }
        cudaEventRecord(e1, nullptr);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (kernelMs) *kernelMs = ms;
        if (count) cudaMemcpy(hits, b + off[8], size_t(count) * 16, cudaMemcpyDeviceToHost);
        uint32_t err = 0;
        cudaMemcpy(&err, flags, 4, cudaMemcpyDeviceToHost);
        if (cudaGetLastError() != cudaSuccess || err != 0) return VLRResult_InternalError;
        return VLRResult_NoError;
    }
    catch (const std::exception &ex) {
        cudaGetLastError();
        std::fprintf(stderr, "vlrbTraceRaysHost: %s\n", ex.what());
        return VLRResult_InternalError;
    }
}

extern "C" VLRResult vlrbBvhBuildHost(const float* triVerts, uint32_t n, uint32_t* sortedCodes, uint32_t* sortedPrims,
                                      int32_t* children, float* nodeBoxes, float* buildMs) {
    return bvhBuildHost(triVerts, n, 0, sortedCodes, sortedPrims, children, nodeBoxes, nullptr, buildMs);
}

extern "C" VLRResult vlrbBvhBuildOptimizedHost(const float* triVerts, uint32_t n, uint32_t treeletRounds,
                                               uint32_t* sortedCodes, uint32_t* sortedPrims, int32_t* children,
                                               float* nodeBoxes, uint32_t* restructured, float* buildMs) {
    return bvhBuildHost(triVerts, n, treeletRounds, sortedCodes, sortedPrims, children, nodeBoxes, restructured,
                        buildMs);
}
