// Rendering context: owns the API objects, the flattened device scene, the
// path buffers, the FP64 film and the output image.
#pragma once

#include "api_objects.h"
#include "pt.cuh"
#include "bpt.cuh"
#include "post.cuh"
#include "guide_net.h"

#include <memory>

#include <cuda.h>
#include <cuda_runtime.h>
#include <random>

namespace vlrb {
namespace api {

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer() { release(); }
    void release();
    void resize(size_t b);     // discards contents
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

struct RenderOptions {
    uint32_t maxPathLength = 25;      // path_tracing.cu:78, lvc_bpt.cu:216,513
    uint32_t maxPathsInFlight = 1u << 22;
    uint32_t lightPathsPerFrame = 0;  // 0: width * height
    uint64_t rngSeed = 0;             // 0: 591842031321323413 (context.cpp:1176-1190)
    bool consistentDielectricPdf = false;   // see mfBsdfPDF; false = the reference's pdf
    uint32_t blocksPerSM = 8;         // wavefront kernel grid = SMs x blocksPerSM
    uint32_t bvhTreeletRounds = 3;    // treelet restructuring rounds after the LBVH build
    bool auxBuffers = false;          // fill the denoiser's guide buffers on every render
};

struct AutotuneTrial {
    uint32_t maxPathsInFlight, blocksPerSM;
    double segmentsPerSecond;
};

// Learned guiding of the path tracer (vlrbContextSetGuiding).
struct GuidingOptions {
    bool enabled = false;             // guided sampling at Matte / LambertianScattering / UE4 vertices
    bool train = false;               // record samples and train after every launch
    uint32_t log2TableSize = 19;
    float learningRate = 1e-2f;
    uint32_t samplesPerStep = 1u << 18;
    uint32_t stepsPerLaunch = 1;
    uint32_t recordBounces = 2;
    uint32_t warmupLaunches = 4;      // launches that train on plain BSDF sampling first
    float weightClamp = 0.0f;         // > 0: clip training weights above this multiple of the batch mean
    uint32_t trainInterval = 1;       // after warm-up, record and train on every n-th launch
};

struct GuidingStats {
    float lastLoss = 0.0f;
    uint64_t trainingSteps = 0;
    uint64_t guidedLaunches = 0;
};

struct RenderStats {
    uint64_t segments = 0;            // extension rays traced
    uint64_t shadowRays = 0;
    uint64_t frames = 0;
    uint32_t lightVertexOverflow = 0;
};

class Context : public Object {
public:
    explicit Context(CUcontext cu, bool logging);
    ~Context() override;

    // object registry (handle validation)
    std::set<Object*> objects;
    template <typename T> T* adopt(T* o) { o->ctx = this; objects.insert(o); return o; }
    bool owns(const Object* o) const { return o && objects.count(const_cast<Object*>(o)) != 0; }
    void destroy(Object* o);

    void bindOutput(uint32_t w, uint32_t h);
    void setScene(Scene* s) { scene = s; markDirty(); }
    void markDirty() { ++generation; }
    // shrink: on a first frame, render the image at 1/shrink of the output
    // size into the film's top-left region until the next first frame
    // (vlrContextRender's shrinkCoeff, context.cpp:1414)
    // denoise: fill the guide buffers (as options.auxBuffers does) and
    // replace the output image by its denoised version.
    void render(cudaStream_t stream, const Camera* cam, bool firstFrame, uint32_t limitFrames,
                uint32_t samples, uint32_t* numAccumFrames, uint32_t shrink = 1, bool denoise = false);
    // Times short renders over a grid of (paths in flight, blocks per SM),
    // keeps the fastest in `options`, and returns every trial.  Leaves the
    // film holding the last trial (the next firstFrame render clears it).
    std::vector<AutotuneTrial> autotune(cudaStream_t stream, const Camera* cam, uint32_t samplesPerTrial);
    void readOutput(float* host);
    void readFilm(double* host);
    // Linear guide images (Rec.709 albedo, camera-space normal), width x
    // height float4 each; false when no render has filled them.
    bool readAux(float* albedo, float* normal);
    void readStats(RenderStats* out);
    CUarray outputArray();
    void* outputDevicePtr() const { return output.ptr; }
    void* filmDevicePtr() const { return film.ptr; }
    Film filmDesc() const {
        return Film{ film.as<double>(), width, height,
                     reinterpret_cast<uint32_t*>(static_cast<char*>(film.ptr) + size_t(width) * height * kNumStrata * 8) };
    }
    uint32_t numTriangles() const { return sg.numTris; }
    uint32_t bvhDepth() const { return bvhMaxDepth; }
    uint32_t guideSamplesRecorded() const;

    CUcontext cuContext;
    bool logging;
    int device = 0, numSMs = 148;
    uint32_t width = 0, height = 0;
    uint32_t imgW = 0, imgH = 0;    // the image being rendered (width, height unless shrunk)
    Scene* scene = nullptr;
    VLRRenderer renderer = VLRRenderer_PathTracing;
    RenderOptions options;
    GuidingOptions guiding;
    GuidingStats guidingStats;
    RenderStats stats;
    StageTimer timer;
    uint32_t numAccumFrames = 0;
    uint64_t generation = 1, builtGeneration = 0;

    // Path tracer RNG states of the first sample's slots in pixel order
    // (pixel y*imgW+x), count <= imgW*imgH; false if the path buffers do not
    // hold that many.
    bool readPixelRngStates(uint64_t* states, uint32_t count);
    // The path tracer's queue counters of its last launch, kCountersPerBounce
    // words per bounce (pt.cuh: rays traced, shadow rays, then one hit queue
    // per BSDF kind and the miss queue) for the first `bounces` bounces.
    bool readBounceCounters(uint32_t* counters, uint32_t bounces);

    // For a persistent batch launch (after a render of this image): the
    // scene, path RNG states, film and totals, rendering `spp` samples per
    // pixel; false when the path buffers do not hold one slot per pixel.
    bool persistentScene(uint32_t spp, PersistentScene* out) const;
    bool shadingNeedsMaps() const { return sg.geomMaps != nullptr || sg.hasScalarTextures != 0; }
    void clearFilm(cudaStream_t stream) { filmClear(filmDesc(), stream); }
    void convertFilm(cudaStream_t stream) { filmToRGBA(filmDesc(), output.as<float4>(), stream); }

private:
    void buildScene(cudaStream_t stream);
    void setupCamera(const Camera* cam);
    void ensurePathBuffers(uint32_t paths, uint32_t imageW, uint32_t imageH);
    void ensureGuiding(uint32_t paths);
    void trainGuide(cudaStream_t stream);

public:
    std::unique_ptr<guide::GuideNet> guideNet;
private:
    DeviceBuffer guideMem;
    GuideFrame gframe{};
    uint32_t guideCapacityPaths = 0, guideLaunches = 0, guideRecBounces = 0, guideSampleCapacity = 0;

    SceneGPU sg{};
    std::vector<std::unique_ptr<DeviceBuffer>> sceneBufs;
    // Image2DTexture nodes of the bound scene: each image in a CUDA array
    // read through a texture object with the node's filter and wrap modes
    struct SceneTexture {
        cudaArray_t array = nullptr;
        cudaTextureObject_t tex = 0;
        SceneTexture() = default;
        SceneTexture(const SceneTexture &) = delete;
        SceneTexture &operator=(const SceneTexture &) = delete;
        ~SceneTexture();
    };
    std::vector<std::unique_ptr<SceneTexture>> sceneTextures;
    DeviceBuffer film, output, pathMem, lbvhScratch, bptMem, auxMem;
    uint32_t bvhMaxDepth = 0;          // deepest leaf of the scene's hierarchy (internal nodes on its path)
    AuxBuffers aux{};
    uint32_t auxSamples = 0;       // guide samples accumulated since the buffers were cleared
    uint64_t auxSeed = 0;
    bool auxCurrent = false;       // the guide buffers follow the current accumulation
    PathBuffers pb{};
    PathBuffers lightPb{};
    std::mt19937_64 bptRng{ 459182033132123413ull };
    uint64_t bptLightSeed = 459182033132123413ull, ltLightSeed = 459182033132123413ull;
    static uint64_t lightSeedOf(uint64_t rngSeed);
    BptBuffers bb{};
    uint32_t pathCapacity = 0;
    uint64_t pathSeed = 0;
    uint32_t pathSeedW = 0, pathSeedH = 0;   // image layout the path RNG states were seeded for
    unsigned long long totalsBase[2] = { 0, 0 };
    uint32_t bptCapacityPaths = 0, bptCapacityVerts = 0, bptEyeCapacity = 0;
    // light tracing: light subpaths of one frame and their lens connections
    DeviceBuffer ltMem;
    PathBuffers ltPb{};
    void* ltConn = nullptr;
    uint32_t ltCapacity = 0;
    CUarray outArray = nullptr;
    uint32_t* hostCounters = nullptr;
    std::vector<float> envPixelsCache;
    template <typename T> T* upload(const std::vector<T> &v, cudaStream_t stream);
};

// Many contexts rendered together: each item's launch sequence runs on its
// own stream forked from the caller's, and the whole batch is captured once
// into one CUDA graph that every launch replays.  Per-item device times come
// from event nodes around each branch.  Path tracing only (plain or guided):
// LVC-BPT draws its per-frame wavelengths on the host, which a replayed graph
// would freeze.
struct BatchItem {
    Context* ctx;
    const Camera* cam;
    uint32_t samples;
    bool firstFrame;
};

class RenderBatch {
public:
    // persistent: the plain (unguided) items render in one persistent kernel
    // launch (pt_persistent.cu), laid out smallest work (pixels x samples)
    // first; guided items keep their own launch sequences beside it.
    RenderBatch(std::vector<BatchItem> items, cudaStream_t stream, bool persistent = false);
    ~RenderBatch();
    RenderBatch(const RenderBatch &) = delete;
    RenderBatch &operator=(const RenderBatch &) = delete;
    void launch(cudaStream_t stream);
    // device milliseconds of each item in the latest launch
    void itemTimes(std::vector<float>* ms) const;

    std::vector<BatchItem> items;
private:
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> evBegin, evEnd, evJoin;
    cudaEvent_t fork = nullptr;
    cudaStream_t captureStream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // persistent mode
    bool persistent = false;
    std::vector<uint32_t> plainOrder;        // item indices in the order of the persistent layout
    std::vector<uint32_t> slotOfItem;        // item -> position in plainOrder, or ~0u
    DeviceBuffer scenesBuf, countersBuf;
    PersistentWork work{};
    bool maps = false;
    int grid = 0;
    cudaStream_t pStream = nullptr;
    cudaEvent_t pJoin = nullptr;
};

} // namespace api
} // namespace vlrb
