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
// its own streams and timing events.  Calls are serialised by the mutex.
//
// A batch moves in chunks of queries on kHostStreams streams in turn: each
// chunk's inputs go up, its kernel runs, its outputs come back, all on its
// stream, so the upload of one chunk, the kernels of another and the
// download of a third overlap (the bus carries both directions at once).
// Each query's result depends only on its own inputs, so the outputs are
// those of one launch over the whole batch.
constexpr int kHostStreams = 3;
constexpr int kMaxHostChunks = 16;
// 2^20 queries between pinned arrays: 0.42 G queries/s in one piece, 0.45,
// 0.49 and 0.49 in chunks of 2^17, 2^18 and 2^19 (the link overlaps the two
// directions only in part on this machine).
constexpr size_t kMinHostChunk = size_t(1) << 18;

struct HostBatchState {
    void* in = nullptr;
    void* out = nullptr;
    size_t inBytes = 0, outBytes = 0;
    cudaStream_t streams[kHostStreams] = {};
    cudaEvent_t e0[kMaxHostChunks] = {}, e1[kMaxHostChunks] = {};
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
        if (!st.streams[0]) {
            for (int i = 0; i < kHostStreams; ++i)
                if (cudaStreamCreateWithFlags(&st.streams[i], cudaStreamNonBlocking) != cudaSuccess)
                    return VLRResult_InternalError;
            for (int i = 0; i < kMaxHostChunks; ++i)
                if (cudaEventCreate(&st.e0[i]) != cudaSuccess || cudaEventCreate(&st.e1[i]) != cudaSuccess)
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
        // the device batch: the SoA arrays back to back (value first so its
        // float4 stores stay 16-byte aligned)
        VLRBBsdfBatch d = *batch;
        {
            size_t off = 0;
            auto at = [&](size_t words) { void* p = ib + off; off += n * words * 4; return p; };
            d.wo = static_cast<const float*>(at(3));
            d.material = static_cast<const uint32_t*>(at(1));
            d.roughness = static_cast<const float*>(at(2));
            d.ior = static_cast<const float*>(at(1));
            d.albedo = static_cast<const float*>(at(3));
            d.metallic = static_cast<const float*>(at(1));
            d.u = static_cast<const float*>(at(3));
            d.wavelengthU = static_cast<const float*>(at(2));
        }
        d.value = reinterpret_cast<float*>(ob);
        d.evalValue = reinterpret_cast<float*>(ob + n * 16);
        d.pdf = reinterpret_cast<float*>(ob + n * 32);
        d.wi = reinterpret_cast<float*>(ob + n * 36);
        d.evalPdf = reinterpret_cast<float*>(ob + n * 48);
        // chunks of at least kMinHostChunk queries, at most kMaxHostChunks,
        // a multiple of 8 queries each
        size_t chunk = std::max(kMinHostChunk, (n + kMaxHostChunks - 1) / kMaxHostChunks);
        chunk = (chunk + 7) & ~size_t(7);
        const int numChunks = static_cast<int>((n + chunk - 1) / chunk);
        cudaError_t e = cudaSuccess;
        for (int c = 0; c < numChunks && e == cudaSuccess; ++c) {
            const size_t first = size_t(c) * chunk, m = std::min(chunk, n - first);
            cudaStream_t s = st.streams[c % kHostStreams];
            struct Part { const void* host; const void* dev; size_t words; };
            const Part in[8] = { { batch->wo, d.wo, 3 }, { batch->material, d.material, 1 },
                                 { batch->roughness, d.roughness, 2 }, { batch->ior, d.ior, 1 },
                                 { batch->albedo, d.albedo, 3 }, { batch->metallic, d.metallic, 1 },
                                 { batch->u, d.u, 3 }, { batch->wavelengthU, d.wavelengthU, 2 } };
            for (const Part &p : in) {
                if (e != cudaSuccess) break;
                const size_t o = first * p.words * 4;
                e = cudaMemcpyAsync(static_cast<char*>(const_cast<void*>(p.dev)) + o,
                                    static_cast<const char*>(p.host) + o, m * p.words * 4,
                                    cudaMemcpyHostToDevice, s);
            }
            if (e != cudaSuccess) break;
            VLRBBsdfBatch dc = d;
            dc.count = static_cast<int64_t>(m);
            dc.wo += first * 3; dc.material += first; dc.roughness += first * 2; dc.ior += first;
            dc.albedo += first * 3; dc.metallic += first; dc.u += first * 3; dc.wavelengthU += first * 2;
            dc.value += first * 4; dc.evalValue += first * 4; dc.pdf += first; dc.wi += first * 3;
            dc.evalPdf += first;
            cudaEventRecord(st.e0[c], s);
            e = (flags & VLRB_BSDF_BATCH_CONTRACTED) ? vlrb::launchBsdfBatchContracted(dc, s, nullptr)
                                                     : vlrb::launchBsdfBatch(dc, s, nullptr);
            cudaEventRecord(st.e1[c], s);
            const struct { void* host; const void* dev; size_t bytes; } back[5] = {
                { batch->value + first * 4, dc.value, m * 16 }, { batch->evalValue + first * 4, dc.evalValue, m * 16 },
                { batch->pdf + first, dc.pdf, m * 4 }, { batch->wi + first * 3, dc.wi, m * 12 },
                { batch->evalPdf + first, dc.evalPdf, m * 4 } };
            for (const auto &b : back)
                if (e == cudaSuccess) e = cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, s);
        }
        for (int i = 0; i < kHostStreams; ++i) {
            const cudaError_t es = cudaStreamSynchronize(st.streams[i]);
            if (e == cudaSuccess) e = es;
        }
        if (e == cudaSuccess && kernelMs) {
            float total = 0.0f;
            for (int c = 0; c < numChunks && e == cudaSuccess; ++c) {
                float ms = 0.0f;
                e = cudaEventElapsedTime(&ms, st.e0[c], st.e1[c]);
                total += ms;
            }
            *kernelMs = total;
        }
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
