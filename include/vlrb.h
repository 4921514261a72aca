/* libvlr_b200 extension API: entry points with no counterpart in the
 * reference's vlr.h, added for workloads the reference runs only inside its
 * renderer.  All are plain C: pointers, sizes, VLRResult codes.
 */
#ifndef VLRB_VLRB_H
#define VLRB_VLRB_H

#include "vlr/vlr.h"

#if defined(__cplusplus)
extern "C" {
#endif

/* Library build identifier, e.g. "vlr_b200 sm_100a". */
const char* vlrbVersion(void);

/* ------------------------------------------------------------------------
 * BSDF shading batch.
 *
 * One query = the reference's BSDF sample, then evaluate and evaluatePDF at
 * the sampled direction, for one of seven BSDFs built from immediate values
 * the way the reference's setupBSDF callables build them
 * (libVLR/GPU_kernels/materials.cu:584-1994).  Arrays are AoS float tuples.
 *   material: 0 Matte, 1 SpecularReflection, 2 MicrofacetReflection,
 *             3 MicrofacetScattering, 4 LambertianScattering, 5 UE4,
 *             6 SpecularScattering (dispersive ideal dielectric, exterior
 *             IOR 1); any other id builds UE4.
 *   roughness[2]: per-axis roughness r; alpha = max(0.001, r^2) for the GGX
 *             materials, roughness = max(0.01, r.x) for UE4.
 *   ior: grey index of refraction (interior for the dielectric, eta of the
 *             conductors with k = 0).
 *   albedo[3]: linear Rec.709 reflectance, Meng-upsampled.
 *   u[3] = (uComponent, uDir0, uDir1); wavelengthU[2] = (offset, uSelect).
 * Outputs: value[4], pdf, wi[3], evalValue[4], evalPdf.  Queries whose sample
 * fails (pdf 0) write zeros everywhere.
 * ---------------------------------------------------------------------- */
typedef struct VLRBBsdfBatch {
    int64_t count;
    const float* wo;
    const uint32_t* material;
    const float* roughness;
    const float* ior;
    const float* albedo;
    const float* metallic;
    const float* u;
    const float* wavelengthU;
    float* value;
    float* pdf;
    float* wi;
    float* evalValue;
    float* evalPdf;
} VLRBBsdfBatch;

/* All pointers are device pointers; enqueued on `stream`, asynchronous. */
VLRResult vlrbBsdfBatch(const VLRBBsdfBatch* batch, CUstream stream);

/* All pointers are host pointers; copies in, runs, copies out, returns when
 * done.  The batch moves in chunks on three streams, so uploads, kernels and
 * downloads of different chunks overlap; the outputs are those of one launch
 * over the whole batch.  kernelMs (may be NULL) receives the kernels' device
 * time summed over the chunks.  The device buffers and streams it uses are
 * kept per device between calls (grown to the largest batch so far, released
 * at process exit), and calls are serialised; pinned host arrays copy at the
 * link's full rate and overlap, pageable ones are staged by the driver. */
VLRResult vlrbBsdfBatchHost(const VLRBBsdfBatch* batch, float* kernelMs);

/* vlrbBsdfBatchHost with options.  VLRB_BSDF_BATCH_CONTRACTED runs the copy
 * of the kernel compiled with fused multiply-add contraction, the arithmetic
 * the renderers' shading kernels use; without it the kernel rounds every
 * operation like the reference's host build.  Other bits: InvalidArgument. */
#define VLRB_BSDF_BATCH_CONTRACTED 1u
VLRResult vlrbBsdfBatchHostEx(const VLRBBsdfBatch* batch, uint32_t flags, float* kernelMs);


/* ------------------------------------------------------------------------
 * Rendering extensions.
 * ---------------------------------------------------------------------- */

/* Render `samples` samples per pixel in as few launches as the path budget
 * allows (vlrContextRender renders exactly one per call, as the reference
 * does: libVLR/context.cpp:1423-1442).  Same film, accumulation and
 * firstFrame semantics as vlrContextRender; limitNumAccumFrames caps the
 * total. */
VLRResult vlrbContextRenderSamples(VLRContext context, CUstream stream, VLRCameraConst camera, bool firstFrame,
                                   uint32_t samples, uint32_t limitNumAccumFrames, uint32_t* numAccumFrames);

typedef struct VLRBRenderOptions {
    uint32_t maxPathLength;       /* hits after which a path stops scattering (reference: 25) */
    uint32_t maxPathsInFlight;    /* path slots per launch (memory ~ 200 B each) */
    uint32_t lightPathsPerFrame;  /* light subpaths per frame of LVC-BPT and the light tracer;
                                     0 = the pixel count (one per pixel path); the LVC-BPT
                                     cache holds 10 vertices per light subpath */
    uint64_t rngSeed;             /* seed of the per-path RNG states, 0 = the reference's
                                     591842031321323413 (context.cpp:1176-1190); any other
                                     seed also gives LVC-BPT's and the light tracer's light
                                     subpaths and per-frame wavelengths their own seed
                                     (otherwise the reference's 459182033132123413) */
    uint32_t consistentDielectricPdf;  /* 0: MicrofacetScattering pdf exactly as the reference,
                                     which is 0 for every transmission out of the medium
                                     (materials.cu:1448-1513), so MIS double-counts NEE
                                     through exits; 1: pdf consistent with the sampled
                                     density and the value (unbiased MIS) */
    uint32_t blocksPerSM;         /* grid of the wavefront kernels = SMs x this (0 = 8) */
    uint32_t bvhTreeletRounds;    /* treelet restructuring rounds after the LBVH build
                                     (vlrbBvhBuildOptimizedHost), 0..8; default 3 */
    uint32_t auxBuffers;          /* 1: fill the denoiser's guide buffers (first-hit albedo and
                                     normal) with every render, as vlrContextRender(denoise = true)
                                     does for its own call; read with vlrbContextReadAuxBuffers */
} VLRBRenderOptions;

VLRResult vlrbContextSetRenderOptions(VLRContext context, const VLRBRenderOptions* options);
VLRResult vlrbContextGetRenderOptions(VLRContext context, VLRBRenderOptions* options);

/* Autotuner: times `samplesPerTrial`-spp renders of the bound scene and camera
 * over paths in flight {2^20 .. 2^25} x blocks per SM {4, 8, 16, 32}, keeps
 * the fastest pair in the render options and writes up to maxTrials trials
 * (paths in flight, blocks per SM, segments/s).  Path counts above what one
 * trial renders (pixels x samplesPerTrial) or above half the free device
 * memory (~256 bytes a path) are not tried: give the trial the samples per
 * call the application renders.  The film holds the last trial afterwards;
 * the next render with firstFrame clears it. */
typedef struct VLRBAutotuneTrial {
    uint32_t maxPathsInFlight;
    uint32_t blocksPerSM;
    double segmentsPerSecond;
} VLRBAutotuneTrial;
VLRResult vlrbContextAutotune(VLRContext context, CUstream stream, VLRCameraConst camera, uint32_t samplesPerTrial,
                              VLRBAutotuneTrial* trials, uint32_t maxTrials, uint32_t* numTrials);

typedef struct VLRBRenderStats {
    uint64_t pathSegments;        /* extension rays traced (camera rays included) */
    uint64_t shadowRays;
    uint64_t frames;              /* samples per pixel rendered since context creation */
    uint32_t lightVertexOverflow; /* LVC-BPT cache appends dropped for lack of capacity */
    uint32_t numTriangles;
    uint32_t bvhMaxDepth;         /* internal nodes on the deepest root-to-leaf path of the scene's
                                     hierarchy; never above the traversal stack (64) */
} VLRBRenderStats;

VLRResult vlrbContextGetStats(VLRContext context, VLRBRenderStats* stats);

/* The path tracer's per-pixel RNG states (PCG32 state words) after the last
 * render, in pixel order (y * width + x of the rendered image), for the first
 * `count` pixels.  Pixel i's stream starts at the i-th output of
 * std::mt19937_64(rngSeed), as the reference seeds its per-pixel RNG buffer
 * (context.cpp:1176-1190), and is advanced by that pixel's samples exactly as
 * the reference's when every launch renders one sample per pixel
 * (maxPathsInFlight = pixel count).  InvalidArgument if count exceeds the
 * pixels or no path tracer render has seeded the states for this image. */
VLRResult vlrbContextReadPixelRngStates(VLRContext context, uint64_t* states, uint32_t count);

/* The path tracer's queue lengths in its last launch (no counterpart in the
 * reference, whose OptiX launch keeps no queues): 16 words per bounce for the
 * first `bounces` bounces (at most 65): [0] rays traced, [1] shadow rays
 * appended, [2 + k] hits appended to the shading queue of BSDF kind k (0
 * Matte, 1 SpecularReflection, 2 MicrofacetReflection, 3
 * MicrofacetScattering, 4 LambertianScattering, 5 UE4, 6 SpecularScattering,
 * 7 emitter without BSDF), [10] misses; the rest 0. */
VLRResult vlrbContextReadBounceCounters(VLRContext context, uint32_t* counters, uint32_t bounces);

/* Learned path guiding of the path tracer (no counterpart in the reference).
 * With `train`, a launch records training samples at the Matte,
 * LambertianScattering and UE4 vertices of its first `recordBounces` bounces
 * and is followed by `stepsPerLaunch` Adam steps on about `samplesPerStep` of
 * them (every launch during the warm-up, then every `trainInterval`-th).  With `enabled`, those vertices sample the next direction from the
 * network's vMF mixture or the BSDF with probability 1/2 each and weight by
 * the combined density (one-sample MIS: unbiased whatever the network
 * learned); when training too, guided sampling starts after `warmupLaunches`
 * launches.  The network is created on first use and kept across frames. */
typedef struct VLRBGuidingOptions {
    bool enabled;
    bool train;
    uint32_t log2TableSize;       /* hash-grid entries per level = 2^log2TableSize (8..24, default 19) */
    float learningRate;           /* default 1e-2 */
    uint32_t samplesPerStep;      /* default 2^18 */
    uint32_t stepsPerLaunch;      /* default 1 */
    uint32_t recordBounces;       /* bounces that are guided and recorded, 1..8, default 2 */
    uint32_t warmupLaunches;      /* default 4 */
    float weightClamp;            /* > 0: training weights above this multiple of the batch
                                     mean are clipped (0 = off, the default) */
    uint32_t trainInterval;       /* after the warm-up, record and train on every n-th launch
                                     (0 or 1 = every launch) */
} VLRBGuidingOptions;

typedef struct VLRBGuidingStats {
    float lastLoss;               /* batch loss of the latest training step */
    uint64_t trainingSteps;
    uint64_t guidedLaunches;
    uint32_t lastSamples;         /* training samples the latest launch recorded */
} VLRBGuidingStats;

typedef struct VLRBGuideNet_API* VLRBGuideNet;
VLRResult vlrbContextSetGuiding(VLRContext context, const VLRBGuidingOptions* options);
VLRResult vlrbContextGetGuiding(VLRContext context, VLRBGuidingOptions* options);
VLRResult vlrbContextGetGuidingStats(VLRContext context, VLRBGuidingStats* stats);
/* A handle to the context's network (created by its first guided or
 * training render) for the vlrbGuideNet* calls below; release it with
 * vlrbGuideNetDestroy, which leaves the context's network alone.  The handle
 * is valid while the context lives and keeps its guiding table size. */
VLRResult vlrbContextGetGuideNet(VLRContext context, VLRBGuideNet* net);

/* Copies the FP64 spectral film (width * height * 16 doubles, strata of
 * 29.375 nm over 360-830 nm, sum over accumulated samples) to host memory. */
VLRResult vlrbContextReadFilm(VLRContext context, double* strata);

/* The denoiser's guide images of the current accumulation (the reference's
 * linearAlbedoBuffer / linearNormalBuffer, post_process.cu:33-91): first-hit
 * base colour in linear Rec.709 and the shading normal in the camera frame
 * (x negated), width * height RGBA32F each; either pointer may be NULL.
 * InvalidArgument until a render with VLRBRenderOptions::auxBuffers or
 * denoise has filled them since the accumulation started. */
VLRResult vlrbContextReadAuxBuffers(VLRContext context, float* albedo, float* normal);

/* Writes <pathWithoutExtension>.png (8-bit RGBA: max(0), x brightnessCoeff,
 * 1 - exp(-x), sRGB gamma, as HostProgram/main.cpp:120-168 tone-maps) and
 * <pathWithoutExtension>.exr (linear, half-float A/B/G/R, no compression)
 * from a width * height RGBA32F image in host memory.  Host-only. */
VLRResult vlrbWriteOutputImages(const float* rgba, uint32_t width, uint32_t height,
                                const char* pathWithoutExtension, float brightnessCoeff);

/* vlrbWriteOutputImages of the context's output image. */
VLRResult vlrbContextSaveOutputImages(VLRContext context, const char* pathWithoutExtension, float brightnessCoeff);

/* Device address of the RGBA32F output image (width * height * 16 bytes). */
VLRResult vlrbContextGetOutputDevicePointer(VLRContext context, void** devicePtr);

/* ------------------------------------------------------------------------
 * LBVH build over world-space triangles (replaces the OptiX acceleration
 * structure builds of libVLR/scene.cpp:1318-1328).
 * triVerts: n triangles x 3 vertices x xyz (host).  Outputs (host):
 *   sortedCodes[n]  30-bit Morton codes in BVH order
 *   sortedPrims[n]  primitive index of each sorted slot
 *   children[2(n-1)] child references of each internal node (>= 0 internal,
 *                   ~i leaf i in sorted order)
 *   nodeBoxes[6(n-1)] box (min xyz, max xyz) of each internal node
 * buildMs (may be NULL) receives the GPU build time.
 * ---------------------------------------------------------------------- */
VLRResult vlrbBvhBuildHost(const float* triVerts, uint32_t n, uint32_t* sortedCodes, uint32_t* sortedPrims,
                           int32_t* children, float* nodeBoxes, float* buildMs);

/* The LBVH build followed by `treeletRounds` rounds of treelet restructuring
 * (7-leaf treelets, least-SAH topology by dynamic programming; the hierarchy
 * the renderer traverses, VLRBRenderOptions::bvhTreeletRounds).  Same outputs
 * as vlrbBvhBuildHost, children and nodeBoxes after restructuring;
 * restructured (may be NULL) receives the number of treelets rebuilt.
 * treeletRounds = 0 is vlrbBvhBuildHost. */
/* Ray queries against a hierarchy built here (the traversal the renderers
 * use; replaces optixTrace, path_tracing.cu:89-93 and
 * light_transport_common.h:169-172, for callers with rays of their own).
 * triVerts as above (host); the hierarchy is the LBVH after `treeletRounds`
 * rounds of restructuring.  rays: count x 8 floats (origin xyz, tmax,
 * direction xyz, unused); hits: count x 4 floats (t, b1, b2, primitive index
 * bits; 0xFFFFFFFF and t = tmax for a miss).  anyHit: stop at the first hit
 * found.  kernelMs (may be NULL) receives the trace kernel's device time. */
VLRResult vlrbTraceRaysHost(const float* triVerts, uint32_t n, uint32_t treeletRounds, const float* rays,
                            uint32_t count, uint32_t anyHit, float* hits, float* kernelMs);

VLRResult vlrbBvhBuildOptimizedHost(const float* triVerts, uint32_t n, uint32_t treeletRounds,
                                    uint32_t* sortedCodes, uint32_t* sortedPrims, int32_t* children,
                                    float* nodeBoxes, uint32_t* restructured, float* buildMs);

/* ------------------------------------------------------------------------
 * The same LBVH build with caller-owned DEVICE buffers that allocates no
 * device memory (no counterpart in the reference, whose acceleration
 * structures OptiX builds).  Its scratch is a static device array sized for
 * VLRB_BVH_NO_ALLOC_MAX_TRIANGLES triangles; a larger n returns
 * VLRResult_InvalidArgument.  The arrays are those of vlrbBvhBuildHost plus
 *   nodes[(n-1) x 64 bytes]  traversal nodes,
 *   tris[n x 48 bytes]       triangles in sorted order.
 * Work is enqueued on `stream`.  One scratch per device: calls on the same
 * device must not overlap (serialise them on one stream or synchronise
 * between them).  The first call on a device does a one-time set-up (it
 * looks up the scratch's device address, which loads this library's device
 * code).  No scratch byte needs an initial value.  The set-up is kept for the
 * process: no cudaDeviceReset between calls.  For
 * n == 1 children, nodeBoxes and nodes are not written and may be NULL.
 * ---------------------------------------------------------------------- */
#define VLRB_BVH_NO_ALLOC_MAX_TRIANGLES 65536u
VLRResult vlrbBvhBuildNoAlloc(const float* triVerts, uint32_t n, uint32_t* sortedCodes, uint32_t* sortedPrims,
                              int32_t* children, float* nodeBoxes, void* nodes, void* tris, CUstream stream);

/* ------------------------------------------------------------------------
 * Spectral utilities (host-side, no GPU needed).
 * ---------------------------------------------------------------------- */

/* Meng-Simon RGB -> spectrum upsampling (the reference's UpsampledSpectrum
 * constructor, libVLR/shared/spectrum_types.cpp:162-228).
 * spectrumType: 0 Reflectance, 1 Light Source, 2 IndexOfRefraction, 3 NA.
 * colorSpace: 0 Rec709(D65) sRGB Gamma, 1 Rec709(D65), 2 XYZ, 3 xyY.
 * packed receives the 12-byte representation {adjacent indices, s, t, scale}. */
VLRResult vlrbUpsampleSpectrum(uint32_t spectrumType, uint32_t colorSpace, float e0, float e1, float e2,
                               uint32_t packed[3]);

/* Evaluate an upsampled spectrum at four wavelengths (nm)
 * (spectrum_types.cpp:273-322). */
VLRResult vlrbEvaluateSpectrum(const uint32_t packed[3], const float lambdas[4], float values[4]);

/* The same spectrum evaluated the way the renderers evaluate material
 * colours: tabulated once on the 95-sample wavelength grid with its point
 * weights and scale applied, then interpolated (equal to
 * vlrbEvaluateSpectrum up to float rounding). */
VLRResult vlrbEvaluateSpectrumTabulated(const uint32_t packed[3], const float lambdas[4], float values[4]);

/* The CIE 1931 colour-matching functions integrated over the 16 film strata
 * (xyz[0..15] = xbar, [16..31] = ybar, [32..47] = zbar) and the Y integral
 * (spectrum_types.cpp:634-680). */
VLRResult vlrbCmfStrata(float xyz[48], float* integralCMF);

/* ------------------------------------------------------------------------
 * Kernel timing.  With profiling on, every wavefront stage is bracketed by
 * CUDA events on the render stream (adds a host synchronisation per render
 * call); times accumulate until reset.  Stages: 0 camera, 1 trace
 * (closest hit + material sort), 2 shade, 3 shadow rays, 4 film, 5 guiding
 * (network inference, training records, training steps).
 * launchCount counts every kernel this library launched for rendering,
 * profiling on or off.
 * ---------------------------------------------------------------------- */
VLRResult vlrbContextSetProfiling(VLRContext context, bool enabled);
VLRResult vlrbContextGetKernelTimes(VLRContext context, double stageMs[6], uint64_t stageLaunches[6],
                                    uint64_t* launchCount);
VLRResult vlrbContextResetKernelTimes(VLRContext context);
/* Bytes of kernel parameters passed host-to-device with the counted launches
 * (the per-launch inputs: scene, path-buffer and frame descriptors). */
VLRResult vlrbContextGetLaunchParamBytes(VLRContext context, uint64_t* bytes);

/* Device address of the FP64 film (width * height * 16 doubles). */
VLRResult vlrbContextGetFilmDevicePointer(VLRContext context, void** devicePtr);

/* ------------------------------------------------------------------------
 * Batched rendering of many contexts (no counterpart in the reference).
 * vlrbRenderBatchCreate renders every item once (scene build, buffers,
 * guiding warm-up), then captures all items' launch sequences, each on its
 * own stream forked from `stream`, into one CUDA graph.  Every
 * vlrbRenderBatchLaunch replays it: item i renders samples[i] spp (restarting
 * its accumulation when firstFrame) and all items run concurrently.  Path
 * tracing only (plain or guided).  itemMs (may be NULL) receives each item's
 * device time of the latest launch (waits for it).
 * ---------------------------------------------------------------------- */
typedef struct VLRBBatchItem {
    VLRContext context;
    VLRCameraConst camera;
    uint32_t samples;
    bool firstFrame;
} VLRBBatchItem;
typedef struct VLRBRenderBatch_API* VLRBRenderBatch;
VLRResult vlrbRenderBatchCreate(const VLRBBatchItem* items, uint32_t numItems, CUstream stream,
                                VLRBRenderBatch* batch);
/* flags: VLRB_BATCH_PERSISTENT renders the plain (unguided) items in ONE
 * persistent kernel launch instead of one launch sequence each: every SM
 * stays busy with pixels taken from one counter over all those items, laid
 * out smallest work (pixels x samples) first, each pixel's samples drawn from
 * its own RNG stream one after another (the images equal the path tracer's at
 * one sample per pixel per launch).  Guided items keep their own launch
 * sequences beside it.  itemMs of a persistent item is the time from the
 * kernel's start to the end of the item's last pixel.  Persistent items do
 * not fill the denoiser's guide buffers. */
#define VLRB_BATCH_PERSISTENT 1u
VLRResult vlrbRenderBatchCreateEx(const VLRBBatchItem* items, uint32_t numItems, CUstream stream, uint32_t flags,
                                  VLRBRenderBatch* batch);
VLRResult vlrbRenderBatchLaunch(VLRBRenderBatch batch, CUstream stream);
VLRResult vlrbRenderBatchItemTimes(VLRBRenderBatch batch, float* itemMs);
VLRResult vlrbRenderBatchDestroy(VLRBRenderBatch batch);

/* ------------------------------------------------------------------------
 * Learned path-guiding network (no counterpart in the reference, which has
 * no guiding).  A hash-grid position encoding (16 levels x 2 features,
 * 2^log2TableSize entries per level) and spherical-harmonic encodings of the
 * outgoing direction and shading normal feed a 64-64-64-64-48 BF16 MLP on
 * the tensor cores; its 40 used outputs are 8 von Mises-Fisher lobes, 5 raw
 * values each: direction (3, normalised), log concentration, mixture logit.
 *
 * Parameters: numWeights FP32 weights, layers back to back, each row-major
 * [out][in] (64x64, 64x64, 64x64, 48x64; output rows 40..47 are padding and
 * stay zero), and numGridFloats FP32 grid features [level][entry][2].
 * Positions are normalised to [0,1]^3 by the box given to SetBounds.
 * Training samples: 16 floats each = position xyz, weight (radiance / pdf),
 * outgoing direction (xyz, pad), shading normal (xyz, pad), incident
 * direction (xyz, pad).  The loss is sum_j (w_j / sum w) * -log q(wi_j).
 * ---------------------------------------------------------------------- */
VLRResult vlrbGuideNetCreate(uint32_t log2TableSize, uint64_t seed, VLRBGuideNet* net);
VLRResult vlrbGuideNetDestroy(VLRBGuideNet net);
VLRResult vlrbGuideNetSetBounds(VLRBGuideNet net, const float* lo, const float* hi);
VLRResult vlrbGuideNetGetSizes(VLRBGuideNet net, uint32_t* numWeights, uint64_t* numGridFloats);
VLRResult vlrbGuideNetGetParams(VLRBGuideNet net, float* weights, float* grid);
VLRResult vlrbGuideNetSetParams(VLRBGuideNet net, const float* weights, const float* grid);
/* raw[n x 40] network outputs for n queries (host arrays of n x 3 floats). */
VLRResult vlrbGuideNetInferHost(VLRBGuideNet net, uint32_t n, const float* pos, const float* wo,
                                const float* nrm, float* raw);
/* Gradients of the batch loss (no parameter update); loss may be NULL. */
VLRResult vlrbGuideNetGradientsHost(VLRBGuideNet net, uint32_t n, const float* samples, float* weightGrad,
                                    float* gridGrad, float* loss);
/* `steps` Adam steps on the same batch; lossPerStep[steps] may be NULL. */
VLRResult vlrbGuideNetTrainHost(VLRBGuideNet net, uint32_t n, const float* samples, float learningRate,
                                uint32_t steps, float* lossPerStep);

#if defined(__cplusplus)
}
#endif

#endif /* VLRB_VLRB_H */
