// Post-processing after the film: the denoiser's guide buffers (first-hit
// albedo and shading normal per pixel), the linear colour / albedo / normal
// images built from them, and an edge-avoiding wavelet denoiser.
//
// The reference fills the guide buffers with its auxBufferGenerator pipeline
// (GPU_kernels/aux_buffer_generator.cu), converts them in copyBuffers
// (post_process.cu:33-91) and hands them to the OptiX denoiser
// (context.cpp:1545-1570), a closed library.  The denoiser here is the
// spatial filter of SVGF (Schied et al., "Spatiotemporal Variance-Guided
// Filtering", HPG 2017), itself the edge-avoiding a-trous wavelet transform
// of Dammertz et al. (HPG 2010): illumination (colour / albedo) is filtered
// with a 5x5 B3-spline kernel at strides 1, 2, 4, 8, 16, each tap weighted
// by normal, albedo and luminance similarity, the luminance stop scaled by
// the locally estimated standard deviation; then remodulated by the albedo.
#pragma once

#include "pt.cuh"
#include "scene_gpu.cuh"

namespace vlrb {

struct AuxBuffers {
    double* albedo;       // [stride * height][kNumStrata] accumulated first-hit base colour x white
    float4* normal;       // [stride * height] accumulated world shading normal
    float4* linAlbedo;    // [stride * height] Rec.709 albedo
    float4* linNormal;    // [stride * height] camera-space normal (x flipped, as the reference)
    float4* work[3];      // [stride * height] denoiser ping-pong buffers + variance
    uint4* guide;         // [stride * height] albedo rgb + normal xyz as halves (the a-trous taps)
    uint32_t stride;      // pixels per row (the output buffer's width)
};

size_t auxBufferBytes(uint32_t stride, uint32_t height);
void carveAuxBuffers(void* base, uint32_t stride, uint32_t height, AuxBuffers* out);
void auxClear(const AuxBuffers &ab, uint32_t height, cudaStream_t stream);

// `samples` first-hit samples per pixel of the width x height image,
// accumulated into ab.albedo / ab.normal.  seed varies per call.
void auxLaunch(const SceneGPU &scene, const AuxBuffers &ab, uint32_t width, uint32_t height, uint32_t samples,
               uint64_t seed, cudaStream_t stream);

// ab.linAlbedo / ab.linNormal from the accumulated buffers (auxSamples: the
// number of samples accumulated so far).
void auxToLinear(const SceneGPU &scene, const AuxBuffers &ab, uint32_t width, uint32_t height, uint32_t auxSamples,
                 cudaStream_t stream);

// Denoises `color` (linear Rec.709, stride layout) in place over the
// width x height region with the guide buffers of ab.
void denoiseLaunch(const AuxBuffers &ab, float4* color, uint32_t width, uint32_t height, cudaStream_t stream);

} // namespace vlrb
