// Persistent path tracing of many scenes in one launch.
//
// The wavefront kernels (pt.cu) render one scene per launch sequence; a batch
// of uneven scenes then either serialises or competes for the GPU.  Here one
// kernel holds every SM for the whole batch: each lane takes a pixel of some
// scene from one global counter over the pixels of all scenes (scenes in the
// order the host lays them out, smallest work first), renders all of that
// pixel's samples with the pixel's own RNG stream, one path segment per loop
// step, and takes the next pixel when done.  Lanes fetch with one atomic per
// warp (warp-aggregated), so the warps stay full until the counter runs out,
// and a scene's pixels are spread over the whole GPU.  Shading uses the same
// steps as the wavefront kernels (pt_shade.cuh) in the same order, and a
// pixel's samples draw from its stream one after another, so a batch renders
// what the wavefront path tracer renders at one sample per pixel per launch
// (the reference's per-pixel sequence, path_tracing.cu:30-259).
//
// Each scene's completion time is stamped from the GPU's global timer by the
// lane that finishes its last pixel, which also adds the samples to the
// scene's film count.  The kernel waits on nothing: lanes only count.
#include "pt_shade.cuh"

#include <stdexcept>
#include <string>

namespace vlrb {

namespace {

constexpr int kPersistentThreads = 128;
// Six blocks of 128 threads per SM (80 registers, a few hundred bytes of
// spills): measured on the 32-scene batch at 0.52, 0.54, 0.57 and 0.62 G
// segments/s for 3 (unbounded, 146 registers), 4, 5 and 6 blocks per SM.
constexpr int kPersistentMinBlocks = 6;

__device__ __forceinline__ unsigned long long globalTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <bool kMaps>
__global__ void __launch_bounds__(kPersistentThreads, kPersistentMinBlocks) persistentPtKernel(PersistentWork w) {
    const uint32_t lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) atomicMin(w.startNs, globalTimerNs());
    uint32_t sc = 0;                    // the lane's scene (units arrive in increasing order)
    uint32_t slot = 0, pixel = 0, samplesLeft = 0;
    bool haveUnit = false, finished = false, alive = false;
    PCG32 rng{ 0ull };
    WLS wls{};
    S4 alpha(0.0f), contrib(0.0f);
    float initImportance = 1.0f, prevDirPDF = 0.0f;
    uint32_t prevType = 0, pathLength = 0;
    V3 rayOrg(0.0f), rayDir(0.0f, 0.0f, 1.0f);
    unsigned long long segs = 0, shadows = 0;
    while (true) {
        // lanes without a pixel take the next ones, one atomic per warp
        const bool need = !finished && !haveUnit;
        const uint32_t needMask = __ballot_sync(0xFFFFFFFFu, need);
        if (needMask) {
            const int leader = __ffs(needMask) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader)
                base = atomicAdd(w.next, static_cast<unsigned long long>(__popc(needMask)));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (need) {
                const unsigned long long unit = base + __popc(needMask & ((1u << lane) - 1u));
                if (unit >= w.totalUnits) finished = true;
                else {
                    while (sc + 1 < w.numScenes && unit >= w.scenes[sc + 1].firstUnit) ++sc;
                    const PersistentScene &PS = w.scenes[sc];
                    slot = static_cast<uint32_t>(unit - PS.firstUnit);
                    pixel = pixelOfPath(slot, PS.width, PS.height);
                    rng.state = PS.rng[slot];
                    samplesLeft = PS.spp;
                    haveUnit = true;
                }
            }
        }
        if (__all_sync(0xFFFFFFFFu, finished)) break;
        if (finished) continue;
        const PersistentScene &PS = w.scenes[sc];
        const SceneGPU &S = PS.scene;
        if (!alive) {
            const CameraRay cr = cameraSample(S, pixel % PS.width, pixel / PS.width, PS.width, PS.height, rng);
            wls = cr.wls;
            alpha = cr.alpha;
            contrib = S4(0.0f);
            initImportance = cr.initImportance;
            prevDirPDF = cr.dirPDF;
            prevType = dir::Acquisition | dir::LowFreq;
            rayOrg = cr.org;
            rayDir = cr.dir;
            pathLength = 0;
            alive = true;
        }
        // one path segment: trace, then shade the hit or the miss
        ++pathLength;
        ++segs;
        bool end = false;
        const Hit h = traceClosest(S, rayOrg, rayDir, FLT_MAX, S.hasAlphaMaps ? rng.state : 0ull);
        if (h.prim == 0xFFFFFFFFu) {
            envMissContribution(S, rayDir, wls, alpha, PrevInRegisters{ prevType, prevDirPDF }, pathLength, contrib);
            end = true;
        }
        else {
            SurfPt sp;
            float hypAreaPDF;
            decodeHit<kMaps>(S, h.prim, h.b1, h.b2, &sp, &hypAreaPDF);
            const uint32_t matIndex = __ldg(S.triMaterial + h.prim);
            const MatDesc &mat = S.mats[matIndex];
            float bsdfScale = 1.0f;
            const uint32_t bsdfIndex =
                mat.bsdfKind == kMultiBSDF ? bsdfMaterial(S, matIndex, rng.state, h.prim, &bsdfScale) : matIndex;
            Bsdf bsdf = buildBsdf<-1, kMaps>(S.meng, S.mats[bsdfIndex], wls, sp.tu, sp.tv);
            const V3 dirOutLocal = sp.frame.toLocal(-rayDir);
            implicitEmission(S, mat, wls, sp, dirOutLocal, rayOrg, hypAreaPDF, PrevInRegisters{ prevType, prevDirPDF },
                             pathLength, alpha, contrib);
            alpha *= bsdfScale;
            if (pathLength >= PS.maxPathLength) end = true;
            else {
                // Russian roulette on the hero-weighted throughput
                const float continueProb = fminf(alpha.importance(wls.selected) / initImportance, 1.0f);
                if (rng.uniform() >= continueProb) end = true;
                else {
                    alpha /= continueProb;
                    const V3 gnLocal = sp.frame.toLocal(sp.gn);
                    BsdfQuery q;
                    q.dirLocal = dirOutLocal;
                    q.wlHint = wls.selected;
                    q.filter = dir::All;
                    q.importanceMode = 0;
                    guide::Mixture noMixture;
                    NeeRay nr;
                    if (neeSample<false>(S, sp, bsdf, q, gnLocal, wls, alpha, rng, false, noMixture, &nr)) {
                        ++shadows;
                        const float vis = shadowVisibility(S, nr.org, nr.dir, nr.tmax);
                        if (vis != 0.0f) contrib += nr.contrib * vis;
                    }
                    const float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
                    BsdfSample bs;
                    const S4 fs = bsdfSample(bsdf, q, gnLocal, uc, ud0, ud1, &bs, nullptr);
                    if (fs.isZero() || !(bs.dirPDF > 0.0f)) end = true;
                    else {
                        if (dir::isDispersive(bs.sampledType) && !wls.single) {
                            bs.dirPDF /= kNumLambdas;
                            wls.single = 1;
                        }
                        const float cosFactor = dot(bs.dirLocal, gnLocal);
                        const V3 dirIn = sp.frame.fromLocal(bs.dirLocal);
                        alpha *= fs * (fabsf(cosFactor) / bs.dirPDF);
                        rayOrg = offsetRayOrigin(sp.position, cosFactor > 0.0f ? sp.gn : -sp.gn);
                        rayDir = dirIn;
                        prevDirPDF = bs.dirPDF;
                        prevType = bs.sampledType;
                    }
                }
            }
        }
        if (!end) continue;
        // the path is done: its film sample (filmKernel's binning), then the
        // pixel's next sample or the next pixel
        alive = false;
        if (contrib.allFinite()) {
            const uint32_t fi = (pixel / PS.width) * PS.stride + pixel % PS.width;
            filmAdd(PS.film.strata + static_cast<size_t>(fi) * kNumStrata, wls.lambda, contrib);
        }
        if (--samplesLeft > 0) continue;
        PS.rng[slot] = rng.state;
        haveUnit = false;
        atomicAdd(PS.totals, segs);
        atomicAdd(PS.totals + 1, shadows);
        segs = shadows = 0;
        if (atomicAdd(w.pixelsDone + sc, 1u) + 1 == PS.width * PS.height) {
            w.endNs[sc] = globalTimerNs();
            *PS.film.frames += PS.spp;
        }
    }
}

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("persistent pt ") + what + ": " + cudaGetErrorString(e));
}

} // namespace

size_t persistentCounterBytes(uint32_t numScenes) {
    return 256 + size_t(numScenes) * 4 + 256 + size_t(numScenes) * 8 + 256;
}

PersistentWork persistentWorkDesc(const PersistentScene* devScenes, uint32_t numScenes,
                                  unsigned long long totalUnits, void* counters) {
    char* c = static_cast<char*>(counters);
    PersistentWork w;
    w.scenes = devScenes;
    w.numScenes = numScenes;
    w.totalUnits = totalUnits;
    w.next = reinterpret_cast<unsigned long long*>(c);
    w.startNs = reinterpret_cast<unsigned long long*>(c + 8);
    w.pixelsDone = reinterpret_cast<uint32_t*>(c + 256);
    w.endNs = reinterpret_cast<unsigned long long*>(c + 256 + ((size_t(numScenes) * 4 + 255) & ~size_t(255)));
    return w;
}

int persistentGrid(int numSMs, bool maps) {
    int perSM = 0;
    ck(maps ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, persistentPtKernel<true>, kPersistentThreads, 0)
            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, persistentPtKernel<false>, kPersistentThreads, 0),
       "occupancy");
    return numSMs * (perSM > 0 ? perSM : 1);
}

void persistentPtLaunch(const PersistentWork &w, bool maps, int grid, cudaStream_t stream) {
    // counters: next = 0, start = max, pixels done = 0, end stamps = 0
    ck(cudaMemsetAsync(w.next, 0, 8, stream), "counter");
    ck(cudaMemsetAsync(w.startNs, 0xFF, 8, stream), "start stamp");
    ck(cudaMemsetAsync(w.pixelsDone, 0, size_t(w.numScenes) * 4, stream), "pixels done");
    ck(cudaMemsetAsync(w.endNs, 0, size_t(w.numScenes) * 8, stream), "end stamps");
    if (maps) persistentPtKernel<true><<<grid, kPersistentThreads, 0, stream>>>(w);
    else persistentPtKernel<false><<<grid, kPersistentThreads, 0, stream>>>(w);
    ck(cudaGetLastError(), "launch");
}

} // namespace vlrb
