// Guide buffers, their linear images and the wavelet denoiser (post.cuh).
#include "post.cuh"
#include "tables.cuh"
#include "wavefront.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <stdexcept>

namespace vlrb {
namespace {

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// getBaseColor of each BSDF (materials.cu:537-539, 592-594, 677-679,
// 805-807, 1077-1081, 1261-1263, 1551-1553, 1702-1704): the albedo or
// coefficient, the conductor's Fresnel reflectance at normal incidence,
// UE4's diffuse + specular F0 colours, zero for emitters.
__device__ __forceinline__ S4 baseColor(const Bsdf &B) {
    switch (B.kind) {
    case kMatte:
    case kLambertianBSDF:
    case kSpecularBRDF:
    case kSpecularBSDF:
    case kMicrofacetBSDF:
        return B.a;
    case kMicrofacetBRDF: {
        FresnelConductor fr{ B.b, B.c };
        return fr.eval(1.0f);
    }
    case kUE4:
        return B.a + B.b;
    default:
        return S4::zero();
    }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct AuxArgs {
    SceneGPU S;
    AuxBuffers ab;
    uint32_t width, height, samples;
    uint64_t seed;
    UpSpec white;   // LightSource Rec.709 (1, 1, 1): the albedo's white point
};

// auxBufferGenerator (aux_buffer_generator.cu:21-69): a camera ray per sample
// through the pixel, its first hit's base colour x the white point's
// spectrum / wavelength pdf into the albedo strata, the shading normal
// (normal maps applied) into the normal sum; misses add nothing.  Unlike the
// reference (one hero-wavelength set per sample), each sample evaluates the
// base colour at 16 stratified wavelengths: the denoiser's albedo term needs
// a guide that is smooth after a few samples.
__global__ void __launch_bounds__(256) auxKernel(AuxArgs a) {
    const SceneGPU &S = a.S;
    const Camera &C = S.cam;
    const uint32_t n = a.width * a.height;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t px = i % a.width, py = i / a.width;
        const size_t fi = static_cast<size_t>(py) * a.ab.stride + px;
        V3 nsum(0.0f, 0.0f, 0.0f);
        for (uint32_t s = 0; s < a.samples; ++s) {
            PCG32 rng{ mix64(a.seed + (static_cast<uint64_t>(i) * a.samples + s) * 0x9E3779B97F4A7C15ULL) };
            const float fx = px + rng.uniform(), fy = py + rng.uniform();
            const float wo = rng.uniform(), ws = rng.uniform();
            float lx, ly;
            const float l0 = rng.uniform(), l1 = rng.uniform();
            concentricDisk(l0, l1, &lx, &ly);
            Frame camFrame;
            camFrame.z = normalize(C.forward);
            camFrame.x = normalize(C.right);
            camFrame.y = cross(camFrame.z, camFrame.x);
            const V3 lensPos = C.right * (C.lensRadius * lx) + C.up * (C.lensRadius * ly) + C.position;
            float dirPDF;
            const V3 dirLocal = cameraSampleDir(C, C.lensRadius * lx, C.lensRadius * ly, fx / a.width,
                                                fy / a.height, &dirPDF);
            const V3 dir = camFrame.fromLocal(dirLocal);
            const Hit h = traceClosest(S, lensPos, dir, FLT_MAX, rng.state);
            if (h.prim == 0xFFFFFFFFu) continue;
            SurfPt sp;
            decodeHit(S, h.prim, h.b1, h.b2, &sp, nullptr);
            const MatDesc &m = S.mats[__ldg(S.triMaterial + h.prim)];
            const uint32_t parts = m.bsdfKind == kMultiBSDF ? m.numSub : 1u;
            // four wavelength sets at offsets (j + wo) / 4: 16 stratified
            // wavelengths per sample, so the guide is nearly free of
            // spectral noise after a few samples
            for (int j = 0; j < 4; ++j) {
                float selectWLPDF;
                const WLS wls = WLS::equalOffsets((j + wo) * 0.25f, ws, &selectWLPDF);
                // a Multi material's base colour is the sum of its components'
                // (MultiBSDF::getBaseColor, materials.cu:2307-2319)
                S4 base = S4::zero();
                for (uint32_t c = 0; c < parts; ++c) {
                    const MatDesc &mc = m.bsdfKind == kMultiBSDF ? S.mats[m.sub[c]] : m;
                    base += baseColor(buildBsdf(S.meng, mc, wls, sp.tu, sp.tv));
                }
                const S4 v = base * mengEvaluate(S.meng, a.white, wls) / (4.0f * selectWLPDF);
                const float lam[4] = { wls.lambda[0], wls.lambda[1], wls.lambda[2], wls.lambda[3] };
                filmAdd(a.ab.albedo + fi * kNumStrata, lam, v);
            }
            nsum += sp.frame.z;
        }
        float4 acc = a.ab.normal[fi];
        a.ab.normal[fi] = make_float4(acc.x + nsum.x, acc.y + nsum.y, acc.z + nsum.z, 0.0f);
    }
}

struct LinearArgs {
    AuxBuffers ab;
    uint32_t width, height;
    float xbar[kNumStrata], ybar[kNumStrata], zbar[kNumStrata];
    float xyzToRgb[9];
    double scale;             // 1 / (integral of the CMF x samples)
    V3 right, up, forward;    // camera axes (the orientation's matrix columns)
};

// copyBuffers (post_process.cu:33-91) for the guides: albedo XYZ / samples ->
// Rec.709; the normal sum into the camera frame (inverse orientation), x
// negated, normalised unless zero.
__global__ void __launch_bounds__(256) auxLinearKernel(LinearArgs a) {
    const uint32_t n = a.width * a.height;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t fi = static_cast<size_t>(i / a.width) * a.ab.stride + i % a.width;
        const double* s = a.ab.albedo + fi * kNumStrata;
        double X = 0, Y = 0, Z = 0;
        for (uint32_t k = 0; k < kNumStrata; ++k) {
            X += a.xbar[k] * s[k];
            Y += a.ybar[k] * s[k];
            Z += a.zbar[k] * s[k];
        }
        const float xyz[3] = { static_cast<float>(X * a.scale), static_cast<float>(Y * a.scale),
                               static_cast<float>(Z * a.scale) };
        float rgb[3];
        mulColMajor(a.xyzToRgb, xyz, rgb);
        a.ab.linAlbedo[fi] = make_float4(rgb[0], rgb[1], rgb[2], 1.0f);
        const float4 w4 = a.ab.normal[fi];
        const V3 w(w4.x, w4.y, w4.z);
        V3 c(-dot(w, a.right), dot(w, a.up), dot(w, a.forward));
        if (c.x != 0.0f || c.y != 0.0f || c.z != 0.0f) c = normalize(c);
        a.ab.linNormal[fi] = make_float4(c.x, c.y, c.z, 1.0f);
    }
}

// ---------------------------------------------------------------- denoiser
constexpr float kAlbedoEps = 1e-3f;
constexpr float kSigmaLuminance = 4.0f;
// exponent of the normal term: 128 = 2^7 (computed by squaring)
constexpr float kSigmaAlbedo2 = 0.02f;     // 2 x (0.1)^2
constexpr int kWaveletPasses = 5;

struct DenoiseArgs {
    const float4* color;
    const float4* albedo;
    const float4* normal;
    uint4* guide;
    uint32_t width, height, stride;
};

__device__ __forceinline__ uint32_t packHalf2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    uint32_t u;
    memcpy(&u, &h, 4);
    return u;
}
__device__ __forceinline__ float2 unpackHalf2(uint32_t u) {
    __half2 h;
    memcpy(&h, &u, 4);
    return __half22float2(h);
}

__device__ __forceinline__ bool isGuided(const float4 &a) {
    return a.x + a.y + a.z > kAlbedoEps;
}
__device__ __forceinline__ float luminance(const float4 &c) {
    return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
}

// Illumination = colour / albedo (pixels with no albedo, misses and
// emitters, pass through unfiltered), and its luminance variance over the
// 3x3 neighbourhood of guided pixels in .w.
__global__ void demodulateKernel(DenoiseArgs a, float4* illum) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= static_cast<int>(a.width) || y >= static_cast<int>(a.height)) return;
    const size_t p = static_cast<size_t>(y) * a.stride + x;
    const float4 ap = a.albedo[p];
    // the taps' guide record: albedo rgb, normal xyz as halves; albedo r
    // negative marks a pixel that is not filtered
    // (albedo clamped to the largest finite half: an unclamped texture or
    // plug value above it would pack to inf and turn tap weights into NaN)
    const float4 np = a.normal[p];
    constexpr float kHalfMax = 65504.0f;
    a.guide[p] = make_uint4(packHalf2(isGuided(ap) ? fminf(ap.x, kHalfMax) : -1.0f, fminf(ap.y, kHalfMax)),
                            packHalf2(fminf(ap.z, kHalfMax), np.x),
                            packHalf2(np.y, np.z), 0u);
    if (!isGuided(ap)) { illum[p] = make_float4(0.f, 0.f, 0.f, 0.f); return; }
    float sum = 0.0f, sum2 = 0.0f, cnt = 0.0f;
    float4 mine = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int qx = x + dx, qy = y + dy;
            if (qx < 0 || qy < 0 || qx >= static_cast<int>(a.width) || qy >= static_cast<int>(a.height)) continue;
            const size_t q = static_cast<size_t>(qy) * a.stride + qx;
            const float4 aq = a.albedo[q];
            if (!isGuided(aq)) continue;
            const float4 cq = a.color[q];
            const float4 iq = make_float4(cq.x / fmaxf(aq.x, kAlbedoEps), cq.y / fmaxf(aq.y, kAlbedoEps),
                                          cq.z / fmaxf(aq.z, kAlbedoEps), 0.0f);
            if (dx == 0 && dy == 0) mine = iq;
            const float l = luminance(iq);
            sum += l;
            sum2 += l * l;
            cnt += 1.0f;
        }
    const float mean = sum / cnt;
    mine.w = fmaxf(sum2 / cnt - mean * mean, 0.0f);
    illum[p] = mine;
}

// One a-trous pass at `step`: 5x5 B3-spline taps at step spacing, each
// weighted by normal agreement, albedo similarity and the luminance
// difference relative to the centre's standard deviation; the variance is
// filtered with the squared weights.
__global__ void __launch_bounds__(256) waveletKernel(DenoiseArgs a, const float4* in, float4* out, int step) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= static_cast<int>(a.width) || y >= static_cast<int>(a.height)) return;
    const size_t p = static_cast<size_t>(y) * a.stride + x;
    const uint4 gp = a.guide[p];
    const float4 ip = in[p];
    const float2 g0 = unpackHalf2(gp.x), g1 = unpackHalf2(gp.y), g2 = unpackHalf2(gp.z);
    if (g0.x < 0.0f) { out[p] = ip; return; }
    const float4 ap = make_float4(g0.x, g0.y, g1.x, 0.0f);
    const float4 np = make_float4(g1.y, g2.x, g2.y, 0.0f);
    const float lp = luminance(ip);
    const float recSigmaL = 1.0f / (kSigmaLuminance * sqrtf(ip.w) + 1e-6f);
    const float kernel[3] = { 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f };
    float sr = 0.f, sg = 0.f, sb = 0.f, wsum = 0.f, vsum = 0.f;
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            const int qx = x + dx * step, qy = y + dy * step;
            if (qx < 0 || qy < 0 || qx >= static_cast<int>(a.width) || qy >= static_cast<int>(a.height)) continue;
            const size_t q = static_cast<size_t>(qy) * a.stride + qx;
            const uint4 gq = a.guide[q];
            const float2 h0 = unpackHalf2(gq.x), h1 = unpackHalf2(gq.y), h2 = unpackHalf2(gq.z);
            if (h0.x < 0.0f) continue;
            const float4 aq = make_float4(h0.x, h0.y, h1.x, 0.0f);
            const float4 nq = make_float4(h1.y, h2.x, h2.y, 0.0f);
            const float4 iq = in[q];
            const float h = kernel[dx < 0 ? -dx : dx] * kernel[dy < 0 ? -dy : dy];
            // normal term max(0, n.n')^128 by seven squarings; the albedo and
            // luminance terms in one exponential (one special-function op a tap)
            float wn = fmaxf(0.0f, np.x * nq.x + np.y * nq.y + np.z * nq.z);
            for (int k = 0; k < 7; ++k) wn *= wn;
            const float da = sq(ap.x - aq.x) + sq(ap.y - aq.y) + sq(ap.z - aq.z);
            const float wal = __expf(-da * (1.0f / kSigmaAlbedo2) - fabsf(lp - luminance(iq)) * recSigmaL);
            const float w = (dx == 0 && dy == 0) ? h : h * wn * wal;
            sr += w * iq.x; sg += w * iq.y; sb += w * iq.z;
            wsum += w;
            vsum += w * w * iq.w;
        }
    out[p] = make_float4(sr / wsum, sg / wsum, sb / wsum, vsum / (wsum * wsum));
}

// Colour = filtered illumination x albedo; unguided pixels keep their colour.
__global__ void remodulateKernel(DenoiseArgs a, const float4* illum, float4* color) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= static_cast<int>(a.width) || y >= static_cast<int>(a.height)) return;
    const size_t p = static_cast<size_t>(y) * a.stride + x;
    const float4 ap = a.albedo[p];
    if (!isGuided(ap)) return;
    const float4 ip = illum[p];
    const float w = color[p].w;
    color[p] = make_float4(ip.x * fmaxf(ap.x, kAlbedoEps), ip.y * fmaxf(ap.y, kAlbedoEps),
                           ip.z * fmaxf(ap.z, kAlbedoEps), w);
}

int numSMsOf() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

} // namespace

size_t auxBufferBytes(uint32_t stride, uint32_t height) {
    const size_t px = static_cast<size_t>(stride) * height;
    return align256(px * kNumStrata * sizeof(double)) + 7 * align256(px * sizeof(float4));
}

void carveAuxBuffers(void* base, uint32_t stride, uint32_t height, AuxBuffers* out) {
    const size_t px = static_cast<size_t>(stride) * height;
    char* c = static_cast<char*>(base);
    out->albedo = reinterpret_cast<double*>(c);
    c += align256(px * kNumStrata * sizeof(double));
    float4** f4[6] = { &out->normal, &out->linAlbedo, &out->linNormal, &out->work[0], &out->work[1], &out->work[2] };
    for (float4** f : f4) {
        *f = reinterpret_cast<float4*>(c);
        c += align256(px * sizeof(float4));
    }
    out->guide = reinterpret_cast<uint4*>(c);
    out->stride = stride;
}

void auxClear(const AuxBuffers &ab, uint32_t height, cudaStream_t stream) {
    const size_t px = static_cast<size_t>(ab.stride) * height;
    ck(cudaMemsetAsync(ab.albedo, 0, px * kNumStrata * sizeof(double), stream), "aux clear");
    ck(cudaMemsetAsync(ab.normal, 0, px * sizeof(float4), stream), "aux clear");
    ck(cudaMemsetAsync(ab.linAlbedo, 0, px * sizeof(float4), stream), "aux clear");
    ck(cudaMemsetAsync(ab.linNormal, 0, px * sizeof(float4), stream), "aux clear");
}

void auxLaunch(const SceneGPU &scene, const AuxBuffers &ab, uint32_t width, uint32_t height, uint32_t samples,
               uint64_t seed, cudaStream_t stream) {
    static const UpSpec white = mengUpsample(hostMengTables(), hostColorMatrices(), SpType::LightSource,
                                             ColorSp::Rec709, 1.0f, 1.0f, 1.0f);
    AuxArgs a;
    a.S = scene;
    a.ab = ab;
    a.width = width;
    a.height = height;
    a.samples = samples;
    a.seed = seed;
    a.white = white;
    const uint32_t n = width * height;
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, static_cast<uint32_t>(numSMsOf()) * 8);
    if (grid == 0) return;
    auxKernel<<<grid, 256, 0, stream>>>(a);
    ck(cudaGetLastError(), "aux kernel");
}

void auxToLinear(const SceneGPU &scene, const AuxBuffers &ab, uint32_t width, uint32_t height, uint32_t auxSamples,
                 cudaStream_t stream) {
    LinearArgs a;
    a.ab = ab;
    a.width = width;
    a.height = height;
    const CmfStrata &cs = hostCmfStrata();
    for (uint32_t k = 0; k < kNumStrata; ++k) { a.xbar[k] = cs.xbar[k]; a.ybar[k] = cs.ybar[k]; a.zbar[k] = cs.zbar[k]; }
    for (int k = 0; k < 9; ++k) a.xyzToRgb[k] = hostColorMatrices().xyzToRec709D65[k];
    a.scale = 1.0 / (static_cast<double>(cs.integralCMF) * std::max<uint32_t>(auxSamples, 1u));
    a.right = scene.cam.right;
    a.up = scene.cam.up;
    a.forward = scene.cam.forward;
    const uint32_t n = width * height;
    const uint32_t grid = std::min<uint32_t>((n + 255) / 256, static_cast<uint32_t>(numSMsOf()) * 8);
    if (grid == 0) return;
    auxLinearKernel<<<grid, 256, 0, stream>>>(a);
    ck(cudaGetLastError(), "aux linear");
}

void denoiseLaunch(const AuxBuffers &ab, float4* color, uint32_t width, uint32_t height, cudaStream_t stream) {
    if (width == 0 || height == 0) return;
    DenoiseArgs a{ color, ab.linAlbedo, ab.linNormal, ab.guide, width, height, ab.stride };
    const dim3 block(16, 16), grid((width + 15) / 16, (height + 15) / 16);
    demodulateKernel<<<grid, block, 0, stream>>>(a, ab.work[0]);
    const float4* in = ab.work[0];
    float4* out = ab.work[1];
    for (int pass = 0; pass < kWaveletPasses; ++pass) {
        waveletKernel<<<grid, block, 0, stream>>>(a, in, out, 1 << pass);
        in = out;
        out = out == ab.work[1] ? ab.work[2] : ab.work[1];
    }
    remodulateKernel<<<grid, block, 0, stream>>>(a, in, color);
    ck(cudaGetLastError(), "denoise");
}

} // namespace vlrb
