// Wavefront path tracer: device buffers and host launch interface.
#pragma once

#include "scene_gpu.cuh"
#include "guide.cuh"
#include <cuda_runtime.h>

namespace vlrb {

constexpr uint32_t kNumShadeBuckets = kNumBsdfKinds + 1;  // + miss
constexpr uint32_t kCountersPerBounce = 16;
constexpr uint32_t kMaxBounces = 64;

// Counter slots within one bounce's block of kCountersPerBounce words.
enum : uint32_t {
    kCntActive = 0,          // rays to trace this bounce
    kCntShadow = 1,          // shadow rays emitted by this bounce's shading
    kCntBucket0 = 2,         // material-sorted hit queues (kNumShadeBuckets)
};

// Pixel of path slot p: the slots of one sample cover the image in 8x4-pixel
// tiles, one warp per tile, when it divides into them (row-major otherwise),
// so a warp's camera rays leave neighbouring pixels in both directions.
// Slot p of every launch renders this pixel, so its RNG state is that
// pixel's stream (seeded in pixel order, as the reference seeds them).
VLRB_HD uint32_t pixelOfPath(uint32_t p, uint32_t W, uint32_t H) {
    const uint32_t i = p % (W * H);
    if ((W & 7u) || (H & 3u)) return i;
    const uint32_t tile = i >> 5, lane = i & 31u, tilesX = W >> 3;
    return ((tile / tilesX) * 4 + (lane >> 3)) * W + (tile % tilesX) * 8 + (lane & 7u);
}

struct ShadowRay {
    float4 org;      // xyz, w = tmax
    float4 dir;      // xyz, w = path index (bits)
    float4 contrib;  // contribution if unoccluded
};

// Per-path state, structure of arrays (P = number of path slots).
struct PathBuffers {
    uint64_t* rng;
    float4* lambda;
    uint32_t* flags;          // bits 0-3 hero index, 4 single, 5 max-length, 8-23 path length
    float4* alpha;
    float4* contrib;
    float* initImportance;
    float* prevDirPDF;
    uint32_t* prevType;
    float4* rayOrg;
    float4* rayDir;
    float4* hit;              // t, b1, b2, prim bits
    uint32_t* active[2];
    uint32_t* buckets;        // [kNumShadeBuckets][P]
    ShadowRay* shadow;        // [P]
    uint32_t* counters;       // [kMaxBounces + 1][kCountersPerBounce]
    unsigned long long* totals;  // [0] extension rays traced, [1] shadow rays (never reset)
};

struct FrameParams {
    uint32_t width, height;   // the image being rendered (the film's top-left region when shrunk)
    uint32_t stride;          // film row length in pixels
    uint32_t sppPerLaunch;    // paths per pixel in this launch
    uint32_t numPaths;        // width * height * sppPerLaunch
    uint32_t maxPathLength;   // hits after which a path stops scattering
    uint32_t bounce;          // current bounce (0-based)
    uint32_t blocksPerSM;     // grid of the wavefront kernels = SMs x this (0: 8)
};

// Film: 16 FP64 strata per pixel, [pixel][16], and the device count of
// samples per pixel it holds (kept on the device so that a captured launch
// sequence replays with the right normalisation).
struct Film {
    double* strata;
    uint32_t width, height;
    uint32_t* frames;
};

// Learned guiding for one launch, at the first recBounces bounces.
// `sample`: guided kinds (Matte, LambertianScattering, UE4) draw their next
// direction from the network's vMF mixture or the BSDF with probability 1/2
// each and weight by the combined density (one-sample MIS).  `record`: every
// guided-kind vertex stores a training record; after the launch
// each record becomes a training sample (position, directions, weight =
// radiance carried back along wi x BSDF x cos / pdf, per path).
constexpr uint32_t kMaxRecBounces = 8;
constexpr uint32_t kRecFields = 6;          // pos, normal, wo, wi, throughput, contribution snapshot
constexpr uint32_t kFlagRecordPending = 1u << 24;
constexpr uint32_t kCountStamp = 3;

struct GuideFrame {
    bool sample;
    bool record;
    uint32_t recBounces;
    guide::Net net;
    uint2* lobes;              // [kLobes][P]  (mu, kappa) as 4 halves
    uint2* lobeWeights;        // [2][P]       mixture weights, 4 halves each
    float4* lobeScales;        // [2][P]       sampling probability x vMF normalisation (FP32)
    float4* rec;               // [recBounces][kRecFields][P]
    uint32_t* recStamp;        // [recBounces][P] launch stamp once a record is complete
    guide::Sample* samples;    // training-sample buffer
    uint32_t sampleCapacity;
    uint32_t targetSamples;    // samples wanted per launch
    uint32_t* counts;          // [0] accepted, [1] candidates this launch, [2] candidates last launch,
                               // [kCountStamp] launch stamp
    uint32_t* err;
};

__host__ __device__ constexpr bool isGuidedKind(uint32_t k) {
    return k == kMatte || k == kLambertianBSDF || k == kUE4;
}

size_t guideBufferBytes(uint32_t numPaths, uint32_t recBounces, uint32_t sampleCapacity);
// Carves the per-path guiding buffers (lobes, records, samples, counters).
void carveGuideBuffers(void* base, uint32_t numPaths, uint32_t recBounces, uint32_t sampleCapacity, GuideFrame* gf);

size_t pathBufferBytes(uint32_t numPaths);
void carvePathBuffers(void* base, uint32_t numPaths, PathBuffers* pb);

// Seeds every path slot's PCG32 state from std::mt19937_64 in slot order, the
// reference's per-pixel seeding (context.cpp:1176-1190) for one slot per pixel.
void seedPathRngs(uint64_t* hostStates, uint32_t numSlots, uint64_t seed);

struct PTStats {
    uint64_t segments;        // extension rays traced
    uint64_t shadowRays;
};

// Render one launch of sppPerLaunch samples per pixel and accumulate the film.
// counterHost (pinned, optional) receives the per-bounce counters after the
// launch for statistics.
// Optional per-stage timing with CUDA events on the launching stream.
enum PtStage : uint32_t { kStageCamera = 0, kStageTrace, kStageShade, kStageShadow, kStageFilm, kStageGuide,
                          kNumPtStages };
struct StageTimer {
    bool enabled = false;
    static constexpr uint32_t kSlots = 3 * kMaxBounces + 4;
    cudaEvent_t ev[2 * kSlots] = {};
    uint32_t stageOf[kSlots] = {};
    uint32_t used = 0;
    double ms[kNumPtStages] = {};
    uint64_t launches[kNumPtStages] = {};
    uint64_t totalLaunches = 0;
    uint64_t paramBytes = 0;   // kernel parameter bytes sent with the launches
    void begin(uint32_t stage, cudaStream_t s, size_t params = 0);
    void end(cudaStream_t s);
    void collect();   // synchronises on the recorded events and accumulates
    StageTimer() = default;
    StageTimer(const StageTimer &) = delete;
    StageTimer &operator=(const StageTimer &) = delete;
    ~StageTimer();
};

void ptRenderLaunch(const SceneGPU &scene, const PathBuffers &pb, const Film &film, const FrameParams &fp,
                    int numSMs, cudaStream_t stream, StageTimer* timer = nullptr, const GuideFrame* guide = nullptr);

// Convert the FP64 film to RGBA32F: XYZ / frames * (W*H) -> Rec.709 D65
// (post_process.cu:93-163).
// Closest-hit trace of bounce fp.bounce's active queue with material-sorted
// output queues (used by both integrators).
void launchTraceSorted(const SceneGPU &scene, const PathBuffers &pb, const FrameParams &fp, int grid,
                       cudaStream_t stream);

void filmToRGBA(const Film &film, float4* out, cudaStream_t stream);

// One scene of a persistent batch launch (pt_persistent.cu): a rendered
// context's scene, RNG states, film and statistics, and how much to render.
struct PersistentScene {
    SceneGPU scene;
    uint64_t* rng;                 // path-slot RNG states: slot p renders pixel pixelOfPath(p)
    Film film;
    unsigned long long* totals;    // running [segments, shadow rays] of the context
    uint32_t width, height;        // the image
    uint32_t stride;               // film row length in pixels
    uint32_t spp;                  // samples per pixel of this launch
    uint32_t maxPathLength;
    unsigned long long firstUnit;  // pixels of the scenes laid out before this one
};

// The batch of one persistent launch and its device counters.
struct PersistentWork {
    const PersistentScene* scenes;   // device array
    uint32_t numScenes;
    unsigned long long totalUnits;   // pixels of all scenes
    unsigned long long* next;        // next pixel to hand out
    unsigned long long* startNs;     // global timer at the launch's start
    uint32_t* pixelsDone;            // per scene
    unsigned long long* endNs;       // global timer when each scene's last pixel finished
};

size_t persistentCounterBytes(uint32_t numScenes);
PersistentWork persistentWorkDesc(const PersistentScene* devScenes, uint32_t numScenes,
                                  unsigned long long totalUnits, void* counters);
// Blocks of the persistent grid: every SM filled to the kernel's occupancy.
int persistentGrid(int numSMs, bool maps);
// Resets the counters and launches (maps: the normal-map / scalar-texture
// shading variant).  Enqueued on `stream`; capturable.
void persistentPtLaunch(const PersistentWork &w, bool maps, int grid, cudaStream_t stream);
void filmClear(const Film &film, cudaStream_t stream);
void filmAddFrames(const Film &film, uint32_t samples, cudaStream_t stream);

} // namespace vlrb
