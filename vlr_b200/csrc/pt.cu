// Wavefront spectral path tracer with MIS next-event estimation.
//
// Per launch (one or more samples per pixel):
//   cameraKernel      camera rays for every path slot (path_tracing.cu:30-77)
//   per bounce b:
//     traceKernel     closest hit of the active rays, then the path index is
//                     appended to the queue of the hit material's BSDF kind
//                     (or the miss queue): material-sorted shading
//     shadeKernel     walks the sorted queues; implicit emission with MIS,
//                     Russian roulette, NEE light sample, BSDF sample
//                     (path_tracing.cu:133-259, miss :266-337)
//     shadowKernel    any-hit visibility of the NEE rays; adds their
//                     contribution when unoccluded
//   filmKernel        bins each path's 4-wavelength contribution into 16 FP64
//                     strata of its pixel (spectrum_types.h:674-684)
// Queue lengths live in device counters, so a launch never synchronises with
// the host and its fixed kernel sequence can be captured in a CUDA graph.
#include "pt.cuh"
#include <cuda_fp16.h>
#include "guide_mlp.cuh"
#include "tables.cuh"
#include "wavefront.cuh"
#include "pt_shade.cuh"

#include <random>
#include <stdexcept>
#include <string>

namespace vlrb {

namespace {

__device__ __forceinline__ WLS loadWls(const PathBuffers &pb, uint32_t p) {
    float4 l = pb.lambda[p];
    uint32_t f = pb.flags[p];
    WLS w;
    w.lambda[0] = l.x; w.lambda[1] = l.y; w.lambda[2] = l.z; w.lambda[3] = l.w;
    w.selected = f & 0xFu;
    w.single = (f >> 4) & 1u;
    return w;
}

__global__ void __launch_bounds__(256) cameraKernel(SceneGPU S, PathBuffers pb, FrameParams fp) {
    const uint32_t P = fp.numPaths;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const uint32_t pixel = pixelOfPath(p, fp.width, fp.height);
        PCG32 rng{ pb.rng[p] };
        const CameraRay cr = cameraSample(S, pixel % fp.width, pixel / fp.width, fp.width, fp.height, rng);
        pb.rng[p] = rng.state;
        pb.lambda[p] = make_float4(cr.wls.lambda[0], cr.wls.lambda[1], cr.wls.lambda[2], cr.wls.lambda[3]);
        pb.flags[p] = cr.wls.selected;
        pb.alpha[p] = toF4(cr.alpha);
        pb.contrib[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        pb.initImportance[p] = cr.initImportance;
        pb.prevDirPDF[p] = cr.dirPDF;
        pb.prevType[p] = dir::Acquisition | dir::LowFreq;
        pb.rayOrg[p] = make_float4(cr.org.x, cr.org.y, cr.org.z, FLT_MAX);
        pb.rayDir[p] = make_float4(cr.dir.x, cr.dir.y, cr.dir.z, 0.0f);
        pb.active[0][p] = p;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) bounceCounters(pb, 0)[kCntActive] = P;
}

__global__ void __launch_bounds__(256) traceKernel(SceneGPU S, PathBuffers pb, FrameParams fp) {
    uint32_t* ctr = bounceCounters(pb, fp.bounce);
    const uint32_t n = ctr[kCntActive];
    const uint32_t* queue = pb.active[fp.bounce & 1];
    const uint32_t P = fp.numPaths;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = queue[i];
        float4 o = pb.rayOrg[p], d = pb.rayDir[p];
        Hit h = traceClosest(S, V3(o.x, o.y, o.z), V3(d.x, d.y, d.z), o.w, S.hasAlphaMaps ? pb.rng[p] : 0ull);
        pb.hit[p] = make_float4(h.t, h.b1, h.b2, __uint_as_float(h.prim));
        uint32_t key = kNumBsdfKinds;
        if (h.prim != 0xFFFFFFFFu) {
            const uint32_t mi = __ldg(S.triMaterial + h.prim);
            key = S.mats[mi].bsdfKind;
            if (key == kMultiBSDF) {
                float scale;
                key = S.mats[bsdfMaterial(S, mi, pb.rng[p], h.prim, &scale)].bsdfKind;
            }
        }
        uint32_t slot = appendSlot(ctr + kCntBucket0 + key, key);
        pb.buckets[key * P + slot] = p;
    }
}

// Environment contribution for a ray that left the scene
// (path_tracing.cu:266-337).
__device__ __forceinline__ void shadeMiss(const SceneGPU &S, const PathBuffers &pb, uint32_t p, const WLS &wls,
                                          uint32_t pathLength, S4 &contrib) {
    if (S.envInst < 0) return;
    const float4 d4 = pb.rayDir[p];
    envMissContribution(S, V3(d4.x, d4.y, d4.z), wls, toS4(pb.alpha[p]), PrevFromBuffers{ &pb, p }, pathLength,
                        contrib);
}

__device__ __forceinline__ float4* recField(const GuideFrame &gf, uint32_t P, uint32_t b, uint32_t f) {
    return gf.rec + (static_cast<size_t>(b) * kRecFields + f) * P;
}

// Completes the training record of the previous bounce with the path's
// contribution so far (everything gathered after the snapshot is the
// indirect light the previous vertex received along its sampled direction).
__device__ __forceinline__ void completeRecord(const GuideFrame &gf, uint32_t P, uint32_t bounce, uint32_t p,
                                               uint32_t flags, const S4 &contrib) {
    if (!(flags & kFlagRecordPending) || bounce == 0) return;
    const uint32_t b = bounce - 1;
    recField(gf, P, b, 5)[p] = toF4(contrib);
    gf.recStamp[static_cast<size_t>(b) * P + p] = gf.counts[kCountStamp];
}

__device__ __forceinline__ uint32_t packHalf2(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float2 unpackHalf2(uint32_t u) {
    return __half22float2(*reinterpret_cast<const __half2*>(&u));
}

// The stored mixture (112 B per path): directions, concentrations and
// weights in half precision, and per lobe the FP32 factor that turns
// exp(kappa (mu.w - 1)) into density, computed from the rounded values the
// sampler uses, so sampling and pdf stay one density.
__device__ __forceinline__ void loadMixture(const GuideFrame &gf, uint32_t P, uint32_t p, guide::Mixture &m) {
#pragma unroll
    for (int k = 0; k < guide::kLobes; ++k) {
        const uint2 q = gf.lobes[static_cast<size_t>(k) * P + p];
        const float2 a = unpackHalf2(q.x), b = unpackHalf2(q.y);
        const float inv = rsqrtf(a.x * a.x + a.y * a.y + b.x * b.x);
        m.lobe[k] = make_float4(a.x * inv, a.y * inv, b.x * inv, b.y);
    }
    const uint2 w0 = gf.lobeWeights[p], w1 = gf.lobeWeights[static_cast<size_t>(P) + p];
    const float2 a = unpackHalf2(w0.x), b = unpackHalf2(w0.y), c = unpackHalf2(w1.x), d = unpackHalf2(w1.y);
    m.weight[0] = a.x; m.weight[1] = a.y; m.weight[2] = b.x; m.weight[3] = b.y;
    m.weight[4] = c.x; m.weight[5] = c.y; m.weight[6] = d.x; m.weight[7] = d.y;
    const float4 s0 = gf.lobeScales[p], s1 = gf.lobeScales[static_cast<size_t>(P) + p];
    m.scale[0] = s0.x; m.scale[1] = s0.y; m.scale[2] = s0.z; m.scale[3] = s0.w;
    m.scale[4] = s1.x; m.scale[5] = s1.y; m.scale[6] = s1.z; m.scale[7] = s1.w;
}

template <bool kGuide, bool kMaps>
__global__ void __launch_bounds__(256, 3) shadeKernel(SceneGPU S, PathBuffers pb, FrameParams fp, GuideFrame gf) {
    uint32_t* ctr = bounceCounters(pb, fp.bounce);
    uint32_t* next = bounceCounters(pb, fp.bounce + 1);
    __shared__ uint32_t sOff[kNumShadeBuckets + 1];
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < kNumShadeBuckets; ++k) { sOff[k] = run; run += ctr[kCntBucket0 + k]; }
        sOff[kNumShadeBuckets] = run;
    }
    __syncthreads();
    const uint32_t total = sOff[kNumShadeBuckets];
    const uint32_t P = fp.numPaths;
    uint32_t* nextQueue = pb.active[(fp.bounce + 1) & 1];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        uint32_t k = 0;
        while (j >= sOff[k + 1]) ++k;
        const uint32_t p = pb.buckets[k * P + (j - sOff[k])];
        WLS wls = loadWls(pb, p);
        uint32_t flags = pb.flags[p];
        uint32_t pathLength = ((flags >> 8) & 0xFFFFu) + 1;
        bool maxLengthTerminate = pathLength >= fp.maxPathLength;
        S4 contrib = toS4(pb.contrib[p]);
        const uint32_t flagsIn = flags;
        flags = (flags & 0x1Fu) | (pathLength << 8) | (maxLengthTerminate ? 0x20u : 0u);
        if (k == kNumBsdfKinds) {
            shadeMiss(S, pb, p, wls, pathLength, contrib);
            if constexpr (kGuide) completeRecord(gf, P, fp.bounce, p, flagsIn, contrib);
            pb.contrib[p] = toF4(contrib);
            pb.flags[p] = flags;
            continue;
        }
        float4 h = pb.hit[p];
        const uint32_t prim = __float_as_uint(h.w);
        SurfPt sp;
        float hypAreaPDF;
        decodeHit<kMaps>(S, prim, h.y, h.z, &sp, &hypAreaPDF);
        const uint32_t matIndex = __ldg(S.triMaterial + prim);
        const MatDesc &mat = S.mats[matIndex];
        float bsdfScale = 1.0f;
        const uint32_t bsdfIndex =
            mat.bsdfKind == kMultiBSDF ? bsdfMaterial(S, matIndex, pb.rng[p], prim, &bsdfScale) : matIndex;
        Bsdf bsdf = buildBsdf<-1, kMaps>(S.meng, S.mats[bsdfIndex], wls, sp.tu, sp.tv);
        float4 o4 = pb.rayOrg[p], d4 = pb.rayDir[p];
        V3 rayOrg(o4.x, o4.y, o4.z), rayDir(d4.x, d4.y, d4.z);
        V3 dirOutLocal = sp.frame.toLocal(-rayDir);
        S4 alpha = toS4(pb.alpha[p]);
        // implicit light sampling
        implicitEmission(S, mat, wls, sp, dirOutLocal, rayOrg, hypAreaPDF, PrevFromBuffers{ &pb, p }, pathLength,
                         alpha, contrib);
        alpha *= bsdfScale;   // a Multi material's component choice (after the emission)
        // The record of the previous vertex closes after this vertex's
        // emission: light reached directly from there is NEE's job, and the
        // network learns the indirect light NEE cannot sample.
        if constexpr (kGuide) completeRecord(gf, P, fp.bounce, p, flagsIn, contrib);
        pb.contrib[p] = toF4(contrib);
        pb.flags[p] = flags;
        if (maxLengthTerminate) continue;
        PCG32 rng{ pb.rng[p] };
        // Russian roulette on the hero-weighted throughput
        float continueProb = fminf(alpha.importance(wls.selected) / pb.initImportance[p], 1.0f);
        if (rng.uniform() >= continueProb) { pb.rng[p] = rng.state; continue; }
        alpha /= continueProb;
        V3 gnLocal = sp.frame.toLocal(sp.gn);
        BsdfQuery q;
        q.dirLocal = dirOutLocal;
        q.wlHint = wls.selected;
        q.filter = dir::All;
        q.importanceMode = 0;
        bool guided = false;
        guide::Mixture mix;
        if constexpr (kGuide) {
            guided = gf.sample && isGuidedKind(k) && fp.bounce < gf.recBounces;
            if (guided) loadMixture(gf, P, p, mix);
        }
        // next-event estimation
        {
            NeeRay nr;
            if (neeSample<kGuide>(S, sp, bsdf, q, gnLocal, wls, alpha, rng, guided, mix, &nr)) {
                uint32_t slot = appendSlot(ctr + kCntShadow, 0u);
                ShadowRay sr;
                sr.org = make_float4(nr.org.x, nr.org.y, nr.org.z, nr.tmax);
                sr.dir = make_float4(nr.dir.x, nr.dir.y, nr.dir.z, __uint_as_float(p));
                sr.contrib = toF4(nr.contrib);
                pb.shadow[slot] = sr;
            }
        }
        // BSDF sampling (guided kinds: one-sample MIS of BSDF and mixture)
        float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
        BsdfSample bs;
        S4 fs;
        if constexpr (kGuide) {
            if (guided) {
                const float uSel = rng.uniform();
                V3 wiW;
                float pB;
                if (uSel < 0.5f) {
                    wiW = guide::mixtureSample(mix, uc, ud0, ud1);
                    bs.dirLocal = sp.frame.toLocal(wiW);
                    fs = bsdfEval(bsdf, q, gnLocal, bs.dirLocal, nullptr);
                    pB = bsdfPDF(bsdf, q, bs.dirLocal, nullptr);
                    bs.sampledType = dir::LowFreq | (dot(bs.dirLocal, gnLocal) > 0.0f ? dir::Reflection
                                                                                       : dir::Transmission);
                }
                else {
                    fs = bsdfSample(bsdf, q, gnLocal, uc, ud0, ud1, &bs, nullptr);
                    pB = bs.dirPDF;
                    wiW = sp.frame.fromLocal(bs.dirLocal);
                }
                bs.dirPDF = 0.5f * pB + 0.5f * guide::mixturePdf(mix, wiW);
            }
            else fs = bsdfSample(bsdf, q, gnLocal, uc, ud0, ud1, &bs, nullptr);
        }
        else fs = bsdfSample(bsdf, q, gnLocal, uc, ud0, ud1, &bs, nullptr);
        pb.rng[p] = rng.state;
        if (fs.isZero() || !(bs.dirPDF > 0.0f)) continue;
        if (dir::isDispersive(bs.sampledType) && !wls.single) {
            bs.dirPDF /= kNumLambdas;
            flags |= 0x10u;
            pb.flags[p] = flags;
        }
        float cosFactor = dot(bs.dirLocal, gnLocal);
        V3 dirIn = sp.frame.fromLocal(bs.dirLocal);
        if constexpr (kGuide) {
            if (gf.record && fp.bounce < gf.recBounces && isGuidedKind(k)) {
                recField(gf, P, fp.bounce, 0)[p] = make_float4(sp.position.x, sp.position.y, sp.position.z, 0.0f);
                recField(gf, P, fp.bounce, 1)[p] = make_float4(sp.frame.z.x, sp.frame.z.y, sp.frame.z.z, 0.0f);
                recField(gf, P, fp.bounce, 2)[p] = make_float4(-rayDir.x, -rayDir.y, -rayDir.z, 0.0f);
                recField(gf, P, fp.bounce, 3)[p] = make_float4(dirIn.x, dirIn.y, dirIn.z, 0.0f);
                recField(gf, P, fp.bounce, 4)[p] = toF4(alpha);
                flags |= kFlagRecordPending;
                pb.flags[p] = flags;
            }
        }
        alpha *= fs * (fabsf(cosFactor) / bs.dirPDF);
        V3 org = offsetRayOrigin(sp.position, cosFactor > 0.0f ? sp.gn : -sp.gn);
        pb.alpha[p] = toF4(alpha);
        pb.prevDirPDF[p] = bs.dirPDF;
        pb.prevType[p] = bs.sampledType;
        pb.rayOrg[p] = make_float4(org.x, org.y, org.z, FLT_MAX);
        pb.rayDir[p] = make_float4(dirIn.x, dirIn.y, dirIn.z, 0.0f);
        uint32_t slot = appendSlot(next + kCntActive, 0u);
        nextQueue[slot] = p;
    }
}

// Six blocks per SM (40 registers, a few spills): the shadow rays are the
// most divergent rays and gain from the extra warps (terrain shadow stage
// 0.97 -> 0.90 ms per spp; the trace kernel measured slower that way).
__global__ void __launch_bounds__(256, 6) shadowKernel(SceneGPU S, PathBuffers pb, FrameParams fp) {
    const uint32_t n = bounceCounters(pb, fp.bounce)[kCntShadow];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        ShadowRay sr = pb.shadow[i];
        const float vis = shadowVisibility(S, V3(sr.org.x, sr.org.y, sr.org.z), V3(sr.dir.x, sr.dir.y, sr.dir.z),
                                           sr.org.w);
        if (vis != 0.0f) {
            uint32_t p = __float_as_uint(sr.dir.w);
            float4 c = pb.contrib[p];
            c.x += vis * sr.contrib.x; c.y += vis * sr.contrib.y; c.z += vis * sr.contrib.z; c.w += vis * sr.contrib.w;
            pb.contrib[p] = c;
        }
    }
}

// ---- learned guiding: network queries straight from the sorted hit queues
struct GuidedHitSrc {
    SceneGPU S;
    PathBuffers pb;
    FrameParams fp;
    guide::Net net;
    __device__ void counts(uint32_t c[3]) const {
        const uint32_t* ctr = bounceCounters(pb, fp.bounce);
        c[0] = ctr[kCntBucket0 + kMatte];
        c[1] = ctr[kCntBucket0 + kLambertianBSDF];
        c[2] = ctr[kCntBucket0 + kUE4];
    }
    __device__ uint32_t count() const {
        uint32_t c[3];
        counts(c);
        return c[0] + c[1] + c[2];
    }
    __device__ uint32_t pathOf(uint32_t i) const {
        uint32_t c[3];
        counts(c);
        uint32_t k = kMatte;
        if (i >= c[0]) { i -= c[0]; k = kLambertianBSDF; if (i >= c[1]) { i -= c[1]; k = kUE4; } }
        return pb.buckets[k * fp.numPaths + i];
    }
    __device__ bool load(uint32_t i, float3* p01, V3* wo, V3* nrm) const {
        const uint32_t p = pathOf(i);
        const float4 h = pb.hit[p];
        SurfPt sp;
        float hyp;
        decodeHit(S, __float_as_uint(h.w), h.y, h.z, &sp, &hyp);
        const float4 d = pb.rayDir[p];
        *p01 = guide::normalisedPosition(net, sp.position.x, sp.position.y, sp.position.z);
        *wo = V3(-d.x, -d.y, -d.z);
        *nrm = sp.frame.z;
        return true;
    }
};

struct MixtureDst {
    GuidedHitSrc src;
    uint2* lobes;
    uint2* lobeWeights;
    float4* lobeScales;
    __device__ void store(uint32_t i, const float y[guide::kOut]) const {
        const uint32_t p = src.pathOf(i);
        const uint32_t P = src.fp.numPaths;
        guide::Mixture m;
        guide::decodeMixture(y, m);
        // round to half, then derive the density factors from what the
        // sampler will read back: lobe k is chosen with the probability its
        // cumulative-weight test gives (the last lobe takes the remainder)
        float w[guide::kLobes], kap[guide::kLobes];
        float acc = 0.0f, prev = 0.0f;
#pragma unroll
        for (int k = 0; k < guide::kLobes; ++k) {
            const float4 l = m.lobe[k];
            lobes[static_cast<size_t>(k) * P + p] = make_uint2(packHalf2(l.x, l.y), packHalf2(l.z, l.w));
            kap[k] = unpackHalf2(packHalf2(l.w, 0.0f)).x;
            w[k] = unpackHalf2(packHalf2(m.weight[k], 0.0f)).x;
        }
        lobeWeights[p] = make_uint2(packHalf2(w[0], w[1]), packHalf2(w[2], w[3]));
        lobeWeights[static_cast<size_t>(P) + p] = make_uint2(packHalf2(w[4], w[5]), packHalf2(w[6], w[7]));
        float sc[guide::kLobes];
#pragma unroll
        for (int k = 0; k < guide::kLobes; ++k) {
            acc += w[k];
            const float cum = k == guide::kLobes - 1 ? 1.0f : fminf(acc, 1.0f);
            const float prob = fmaxf(cum - prev, 0.0f);
            prev = fmaxf(prev, cum);
            sc[k] = prob * expf(guide::vmfLogNorm(kap[k]));
        }
        lobeScales[p] = make_float4(sc[0], sc[1], sc[2], sc[3]);
        lobeScales[static_cast<size_t>(P) + p] = make_float4(sc[4], sc[5], sc[6], sc[7]);
    }
};

__device__ __forceinline__ uint32_t mixBits(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ c * 0xC2B2AE3Du;
    h ^= h >> 15; h *= 0x2C1B3C6Du; h ^= h >> 12; h *= 0x297A2D39u; h ^= h >> 15;
    return h;
}

// Turns the launch's complete records into training samples: weight =
// mean over the 4 wavelengths of (contribution gathered after the vertex) /
// (throughput at the vertex), i.e. incident radiance x BSDF x cos / pdf of the
// sampled direction.  A random subset of about targetSamples is kept.
__global__ void __launch_bounds__(256) guideFinalizeKernel(PathBuffers pb, FrameParams fp, GuideFrame gf) {
    const uint32_t P = fp.numPaths;
    const uint32_t last = gf.counts[2];
    const uint32_t stamp = gf.counts[kCountStamp];
    const float accept = last > gf.targetSamples ? static_cast<float>(gf.targetSamples) / last : 1.0f;
    // one thread per (bounce, path) record: independent loads in flight
    const size_t total = static_cast<size_t>(P) * gf.recBounces;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const uint32_t b = static_cast<uint32_t>(i / P), p = static_cast<uint32_t>(i % P);
        {
            float w = 0.0f;
            if (gf.recStamp[i] == stamp) {
                const float4 cEnd = pb.contrib[p];
                const float4 beta = recField(gf, P, b, 4)[p];
                const float4 snap = recField(gf, P, b, 5)[p];
                const float bt[4] = { beta.x, beta.y, beta.z, beta.w };
                const float dc[4] = { cEnd.x - snap.x, cEnd.y - snap.y, cEnd.z - snap.z, cEnd.w - snap.w };
                for (int i = 0; i < 4; ++i)
                    if (bt[i] > 0.0f) w += fmaxf(dc[i], 0.0f) / bt[i];
                w *= 0.25f;
            }
            const bool cand = w > 0.0f && isfinite(w);
            const bool keep = cand && (mixBits(p, b, stamp) >> 8) * (1.0f / 16777216.0f) < accept;
            // one atomic per warp for the candidate count and the slots
            const uint32_t active = __activemask();
            const int leader = __ffs(active) - 1;
            const uint32_t lane = threadIdx.x & 31;
            const uint32_t cm = __ballot_sync(active, cand), km = __ballot_sync(active, keep);
            uint32_t base = 0;
            if (static_cast<int>(lane) == leader) {
                if (cm) atomicAdd(gf.counts + 1, static_cast<uint32_t>(__popc(cm)));
                if (km) base = atomicAdd(gf.counts, static_cast<uint32_t>(__popc(km)));
            }
            base = __shfl_sync(active, base, leader);
            const uint32_t slot = base + __popc(km & ((1u << lane) - 1u));
            if (!keep || slot >= gf.sampleCapacity) continue;
            const float4 pos = recField(gf, P, b, 0)[p];
            guide::Sample smp;
            smp.posWeight = make_float4(pos.x, pos.y, pos.z, w);
            smp.nrm = recField(gf, P, b, 1)[p];
            smp.wo = recField(gf, P, b, 2)[p];
            smp.wi = recField(gf, P, b, 3)[p];
            gf.samples[slot] = smp;
        }
    }
}

// Start of a recording launch: accepted = 0, last = this, this = 0, next
// stamp.  All on the device, so a captured launch sequence replays correctly.
__global__ void guideCountsKernel(uint32_t* counts) {
    counts[2] = counts[1] > 0 ? counts[1] : counts[2];
    counts[1] = 0;
    counts[0] = 0;
    counts[kCountStamp] += 1;
}

__global__ void __launch_bounds__(256) filmKernel(PathBuffers pb, Film film, FrameParams fp) {
    const uint32_t P = fp.numPaths;
    const float recBinWidth = kNumStrata / (kWavelengthHigh - kWavelengthLow);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        S4 c = toS4(pb.contrib[p]);
        if (!c.allFinite()) continue;
        float4 l = pb.lambda[p];
        float lam[4] = { l.x, l.y, l.z, l.w };
        const uint32_t pixel = pixelOfPath(p, fp.width, fp.height);
        const uint32_t fi = (pixel / fp.width) * fp.stride + pixel % fp.width;
        double* dst = film.strata + static_cast<size_t>(fi) * kNumStrata;
        for (int i = 0; i < 4; ++i) {
            uint32_t bin = vmin<uint32_t>(static_cast<uint32_t>((lam[i] - kWavelengthLow) /
                                          (kWavelengthHigh - kWavelengthLow) * kNumStrata), kNumStrata - 1);
            float v = c[i] * recBinWidth;
            if (v != 0.0f) atomicAdd(dst + bin, static_cast<double>(v));
        }
    }
}

struct FilmConst {
    float xbar[kNumStrata], ybar[kNumStrata], zbar[kNumStrata];
    float integralCMF;
    float xyzToRgb[9];
};

__global__ void filmAddFramesKernel(uint32_t* frames, uint32_t samples) { *frames += samples; }

__global__ void filmToRGBAKernel(Film film, FilmConst fc, float4* out) {
    const uint32_t n = film.width * film.height;
    const uint32_t frames = *film.frames ? *film.frames : 1u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double* s = film.strata + static_cast<size_t>(i) * kNumStrata;
        double X = 0, Y = 0, Z = 0;
        for (uint32_t k = 0; k < kNumStrata; ++k) {
            double v = s[k];
            X += fc.xbar[k] * v;
            Y += fc.ybar[k] * v;
            Z += fc.zbar[k] * v;
        }
        double scale = static_cast<double>(n) / (static_cast<double>(fc.integralCMF) * frames);
        float xyz[3] = { static_cast<float>(X * scale), static_cast<float>(Y * scale), static_cast<float>(Z * scale) };
        float rgb[3];
        mulColMajor(fc.xyzToRgb, xyz, rgb);
        out[i] = make_float4(rgb[0], rgb[1], rgb[2], 1.0f);
    }
}

// Adds this launch's per-bounce queue lengths to the running totals.
__global__ void statsKernel(PathBuffers pb, uint32_t bounces) {
    unsigned long long seg = 0, sh = 0;
    for (uint32_t b = threadIdx.x; b < bounces; b += 32) {
        seg += bounceCounters(pb, b)[kCntActive];
        sh += bounceCounters(pb, b)[kCntShadow];
    }
    for (int off = 16; off > 0; off >>= 1) {
        seg += __shfl_xor_sync(0xFFFFFFFFu, seg, off);
        sh += __shfl_xor_sync(0xFFFFFFFFu, sh, off);
    }
    if (threadIdx.x == 0) { pb.totals[0] += seg; pb.totals[1] += sh; }
}

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("pt ") + what + ": " + cudaGetErrorString(e));
}

inline size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

} // namespace

size_t pathBufferBytes(uint32_t P) {
    size_t b = 0;
    b += a256(size_t(P) * 8);                 // rng
    b += a256(size_t(P) * 16) * 2;            // lambda, alpha
    b += a256(size_t(P) * 4) * 4;             // flags, initImportance, prevDirPDF, prevType
    b += a256(size_t(P) * 16) * 4;            // contrib, rayOrg, rayDir, hit
    b += a256(size_t(P) * 4) * 2;             // active queues
    b += a256(size_t(P) * 4 * kNumShadeBuckets);
    b += a256(size_t(P) * sizeof(ShadowRay));
    b += a256(size_t(kMaxBounces + 1) * kCountersPerBounce * 4);
    b += a256(16);
    return b;
}

void carvePathBuffers(void* base, uint32_t P, PathBuffers* pb) {
    char* s = static_cast<char*>(base);
    auto take = [&](size_t bytes) { char* r = s; s += a256(bytes); return r; };
    pb->rng = reinterpret_cast<uint64_t*>(take(size_t(P) * 8));
    pb->lambda = reinterpret_cast<float4*>(take(size_t(P) * 16));
    pb->alpha = reinterpret_cast<float4*>(take(size_t(P) * 16));
    pb->flags = reinterpret_cast<uint32_t*>(take(size_t(P) * 4));
    pb->initImportance = reinterpret_cast<float*>(take(size_t(P) * 4));
    pb->prevDirPDF = reinterpret_cast<float*>(take(size_t(P) * 4));
    pb->prevType = reinterpret_cast<uint32_t*>(take(size_t(P) * 4));
    pb->contrib = reinterpret_cast<float4*>(take(size_t(P) * 16));
    pb->rayOrg = reinterpret_cast<float4*>(take(size_t(P) * 16));
    pb->rayDir = reinterpret_cast<float4*>(take(size_t(P) * 16));
    pb->hit = reinterpret_cast<float4*>(take(size_t(P) * 16));
    pb->active[0] = reinterpret_cast<uint32_t*>(take(size_t(P) * 4));
    pb->active[1] = reinterpret_cast<uint32_t*>(take(size_t(P) * 4));
    pb->buckets = reinterpret_cast<uint32_t*>(take(size_t(P) * 4 * kNumShadeBuckets));
    pb->shadow = reinterpret_cast<ShadowRay*>(take(size_t(P) * sizeof(ShadowRay)));
    pb->counters = reinterpret_cast<uint32_t*>(take(size_t(kMaxBounces + 1) * kCountersPerBounce * 4));
    pb->totals = reinterpret_cast<unsigned long long*>(take(16));
}

size_t guideBufferBytes(uint32_t P, uint32_t recBounces, uint32_t sampleCapacity) {
    size_t b = 0;
    b += a256(size_t(P) * 8 * guide::kLobes);
    b += a256(size_t(P) * 8 * 2) + a256(size_t(P) * 16 * 2);
    b += a256(size_t(P) * 16 * kRecFields * recBounces);
    b += a256(size_t(P) * 4 * recBounces);
    b += a256(size_t(sampleCapacity) * sizeof(guide::Sample));
    b += a256(64);
    return b;
}

void carveGuideBuffers(void* base, uint32_t P, uint32_t recBounces, uint32_t sampleCapacity, GuideFrame* gf) {
    char* s = static_cast<char*>(base);
    auto take = [&](size_t bytes) { char* r = s; s += a256(bytes); return r; };
    gf->lobes = reinterpret_cast<uint2*>(take(size_t(P) * 8 * guide::kLobes));
    gf->lobeWeights = reinterpret_cast<uint2*>(take(size_t(P) * 8 * 2));
    gf->lobeScales = reinterpret_cast<float4*>(take(size_t(P) * 16 * 2));
    gf->rec = reinterpret_cast<float4*>(take(size_t(P) * 16 * kRecFields * recBounces));
    gf->recStamp = reinterpret_cast<uint32_t*>(take(size_t(P) * 4 * recBounces));
    gf->samples = reinterpret_cast<guide::Sample*>(take(size_t(sampleCapacity) * sizeof(guide::Sample)));
    gf->counts = reinterpret_cast<uint32_t*>(take(64));
    gf->err = gf->counts + 8;
    gf->recBounces = recBounces;
    gf->sampleCapacity = sampleCapacity;
}

void seedPathRngs(uint64_t* states, uint32_t n, uint64_t seed) {
    std::mt19937_64 gen(seed);
    for (uint32_t i = 0; i < n; ++i) states[i] = gen();
}

void StageTimer::begin(uint32_t stage, cudaStream_t s, size_t params) {
    ++totalLaunches;
    paramBytes += params;
    if (!enabled) return;
    if (used == kSlots) collect();   // every slot recorded: drain before reuse
    if (used == 0)
        for (auto &e : ev) if (!e) cudaEventCreate(&e);
    stageOf[used] = stage;
    cudaEventRecord(ev[2 * used], s);
}

void StageTimer::end(cudaStream_t s) {
    if (!enabled) return;
    cudaEventRecord(ev[2 * used + 1], s);
    ++used;
}

StageTimer::~StageTimer() {
    for (auto &e : ev) if (e) cudaEventDestroy(e);
}

void StageTimer::collect() {
    if (!enabled) return;
    for (uint32_t i = 0; i < used; ++i) {
        float t = 0.0f;
        cudaEventSynchronize(ev[2 * i + 1]);
        cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
        ms[stageOf[i]] += t;
        launches[stageOf[i]] += 1;
    }
    used = 0;
}

void ptRenderLaunch(const SceneGPU &scene, const PathBuffers &pb, const Film &film, const FrameParams &fpIn,
                    int numSMs, cudaStream_t stream, StageTimer* timer, const GuideFrame* gfp) {
    FrameParams fp = fpIn;
    if (fp.maxPathLength == 0 || fp.maxPathLength > kMaxBounces)
        throw std::runtime_error("maxPathLength out of range");
    StageTimer dummy;
    StageTimer &T = timer ? *timer : dummy;
    ck(cudaMemsetAsync(pb.counters, 0, size_t(kMaxBounces + 1) * kCountersPerBounce * 4, stream), "counters");
    const int grid = numSMs * static_cast<int>(fp.blocksPerSM ? fp.blocksPerSM : 8);
    const size_t pMain = sizeof(SceneGPU) + sizeof(PathBuffers) + sizeof(FrameParams);
    T.begin(kStageCamera, stream, pMain);
    cameraKernel<<<grid, 256, 0, stream>>>(scene, pb, fp);
    T.end(stream);
    const bool guiding = gfp && (gfp->sample || gfp->record);
    if (guiding && gfp->record) {
        T.begin(kStageGuide, stream, sizeof(void*));
        guideCountsKernel<<<1, 1, 0, stream>>>(gfp->counts);
        T.end(stream);
    }
    for (uint32_t b = 0; b < fp.maxPathLength; ++b) {
        fp.bounce = b;
        T.begin(kStageTrace, stream, pMain);
        traceKernel<<<grid, 256, 0, stream>>>(scene, pb, fp);
        T.end(stream);
        if (guiding && gfp->sample && b < gfp->recBounces) {
            GuidedHitSrc src{ scene, pb, fp, gfp->net };
            MixtureDst dst{ src, gfp->lobes, gfp->lobeWeights, gfp->lobeScales };
            auto kern = guide::guideInferKernel<GuidedHitSrc, MixtureDst>;
            ck(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, guide::kInferSmemBytes),
               "infer smem");
            T.begin(kStageGuide, stream, sizeof(guide::Net) + 2 * sizeof(GuidedHitSrc));
            kern<<<numSMs * 3, guide::kInferThreads, guide::kInferSmemBytes, stream>>>(gfp->net, src, dst, gfp->err);
            T.end(stream);
        }
        T.begin(kStageShade, stream, pMain + (guiding ? sizeof(GuideFrame) : 0));
        // the kMaps variants: normal maps, and float3 textures on scalar parameters
        const bool maps = scene.geomMaps != nullptr || scene.hasScalarTextures != 0;
        // the guided variant only where guiding acts: bounces that sample or
        // record, and the one after the last recorded bounce, which closes
        // its records; later bounces only add to the path's contribution,
        // which the plain variant (fewer registers) does the same way
        const bool guideShade = guiding && (b < gfp->recBounces || (gfp->record && b == gfp->recBounces));
        if (guideShade && maps) shadeKernel<true, true><<<grid, 256, 0, stream>>>(scene, pb, fp, *gfp);
        else if (guideShade) shadeKernel<true, false><<<grid, 256, 0, stream>>>(scene, pb, fp, *gfp);
        else if (maps) shadeKernel<false, true><<<grid, 256, 0, stream>>>(scene, pb, fp, GuideFrame{});
        else shadeKernel<false, false><<<grid, 256, 0, stream>>>(scene, pb, fp, GuideFrame{});
        T.end(stream);
        T.begin(kStageShadow, stream, pMain);
        shadowKernel<<<grid, 256, 0, stream>>>(scene, pb, fp);
        T.end(stream);
    }
    if (guiding && gfp->record) {
        T.begin(kStageGuide, stream, sizeof(PathBuffers) + sizeof(FrameParams) + sizeof(GuideFrame));
        guideFinalizeKernel<<<grid, 256, 0, stream>>>(pb, fp, *gfp);
        T.end(stream);
    }
    T.begin(kStageFilm, stream, sizeof(PathBuffers) + sizeof(Film) + sizeof(FrameParams));
    filmKernel<<<grid, 256, 0, stream>>>(pb, film, fp);
    T.end(stream);
    T.begin(kStageFilm, stream, sizeof(PathBuffers) + 4);
    statsKernel<<<1, 32, 0, stream>>>(pb, fp.maxPathLength);
    T.end(stream);
    ck(cudaGetLastError(), "launch");
    T.collect();
}

void launchTraceSorted(const SceneGPU &scene, const PathBuffers &pb, const FrameParams &fp, int grid,
                       cudaStream_t stream) {
    traceKernel<<<grid, 256, 0, stream>>>(scene, pb, fp);
}

void filmClear(const Film &film, cudaStream_t stream) {
    ck(cudaMemsetAsync(film.strata, 0, size_t(film.width) * film.height * kNumStrata * 8, stream), "film clear");
    ck(cudaMemsetAsync(film.frames, 0, 4, stream), "film frames");
}

void filmAddFrames(const Film &film, uint32_t samples, cudaStream_t stream) {
    filmAddFramesKernel<<<1, 1, 0, stream>>>(film.frames, samples);
    ck(cudaGetLastError(), "film frames");
}

void filmToRGBA(const Film &film, float4* out, cudaStream_t stream) {
    FilmConst fc;
    const CmfStrata &cs = hostCmfStrata();
    for (uint32_t k = 0; k < kNumStrata; ++k) { fc.xbar[k] = cs.xbar[k]; fc.ybar[k] = cs.ybar[k]; fc.zbar[k] = cs.zbar[k]; }
    fc.integralCMF = cs.integralCMF;
    for (int k = 0; k < 9; ++k) fc.xyzToRgb[k] = hostColorMatrices().xyzToRec709D65[k];
    const uint32_t n = film.width * film.height;
    filmToRGBAKernel<<<(n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096, 256, 0, stream>>>(film, fc, out);
    ck(cudaGetLastError(), "film convert");
}

} // namespace vlrb
