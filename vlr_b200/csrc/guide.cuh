// Learned path guiding: a small network maps a shading point (position,
// outgoing direction, shading normal) to an 8-lobe von Mises-Fisher mixture
// over incident directions.  The reference renderer has no guiding; this is
// an addition beside its BSDF sampling, combined with it by one-sample MIS.
//
// Network (all sizes fixed at compile time):
//   inputs   64 features: a multi-resolution hash grid over the position
//            normalised to the scene box (16 levels x 2 features, trilinear;
//            Mueller et al., "Instant Neural Graphics Primitives", 2022) and
//            real spherical harmonics up to degree 3 of the outgoing direction
//            (16) and of the shading normal (16);
//   layers   64 -> 64 -> 64 -> 64 -> 48 (ReLU after the first three, no
//            biases), BF16 operands with FP32 accumulation on the tensor
//            cores (tcgen05.mma, accumulators in TMEM);
//   output   40 raw values used (the last 8 columns stay zero): per lobe k a
//            direction v_k (normalised to the mean mu_k), a log-concentration
//            s_k (kappa_k = exp(clamp(s_k, -4, 8))) and a logit (softmax over
//            the 8 lobes gives the mixture weights).
// Training minimises the KL divergence from the incident-radiance
// distribution to the mixture, estimated with the renderer's own samples:
// loss = mean_j  -w_j log q(wi_j), with w_j = L_j / p_j normalised to mean 1
// over the batch (Mueller et al., "Neural Importance Sampling", 2019).
#pragma once

#include "core.cuh"
#include <cuda_bf16.h>

namespace vlrb {
namespace guide {

constexpr int kLevels = 16;
constexpr int kFeatPerLevel = 2;
constexpr int kGridFeatures = kLevels * kFeatPerLevel;   // 32
constexpr int kIn = 64;
constexpr int kHidden = 64;
constexpr int kOut = 48;            // padded output width
constexpr int kRaw = 40;            // used outputs: 8 lobes x 5
constexpr int kLobes = 8;
constexpr int kRows = 128;          // samples per tensor-core tile
constexpr int kNumLayers = 4;

// FP32 master weights, row-major [out][in] per layer, layers back to back.
__host__ __device__ constexpr int layerOut(int l) { return l == kNumLayers - 1 ? kOut : kHidden; }
__host__ __device__ constexpr int weightOffset(int l) { return l < kNumLayers ? l * kHidden * kIn : 3 * kHidden * kIn + kOut * kHidden; }
constexpr int kNumWeights = weightOffset(kNumLayers);                  // 15360
// BF16 weight tiles in the chunk-major shared-memory layout (umma.cuh),
// layer l occupying layerOut(l) rows x 64 columns.
__host__ __device__ constexpr int tileOffset(int l) { return l < kNumLayers ? l * kHidden * kIn * 2 : 30720; }
constexpr int kWeightTileBytes = tileOffset(kNumLayers);               // 30720

struct Net {
    // hash grid: kLevels x tableSize x kFeatPerLevel FP32
    float* grid;
    float* gridGrad;
    float* gridM;
    float* gridV;
    uint32_t log2Table;
    float levelScale[kLevels];     // grid resolution of each level
    // MLP
    float* w;                      // kNumWeights FP32 master weights
    float* wGrad;
    float* wM;
    float* wV;
    uint8_t* wTiles;               // kWeightTileBytes BF16 tile image
    // position normalisation to [0,1]^3
    float3 lo;
    float3 invExtent;
};

// One training sample: position (xyz) + weight, outgoing direction, shading
// normal, sampled incident direction (all world space).
struct Sample {
    float4 posWeight;
    float4 wo;
    float4 nrm;
    float4 wi;
};

// Per-query mixture: lobe k = (mu_k, kappa_k), mixture weight pi_k.
// Per-query mixture: lobe k = (mu_k, kappa_k), mixture weight pi_k, and
// scale_k = pi_k * kappa_k / (2 pi (1 - exp(-2 kappa_k))) so that
// q(w) = sum_k scale_k exp(kappa_k (mu_k . w - 1)) costs one exp per lobe.
struct Mixture {
    float4 lobe[kLobes];
    float weight[kLobes];
    float scale[kLobes];
};

// ------------------------------------------------------------ encoding
__device__ __forceinline__ uint32_t hashCorner(uint32_t x, uint32_t y, uint32_t z, uint32_t res, uint32_t mask,
                                               bool dense) {
    if (dense) return x + (res + 1) * (y + (res + 1) * z);
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & mask;
}

// Visits the 8 trilinear corners of level l at position p in [0,1]^3:
// fn(tableIndex, weight).
template <class Fn>
__device__ __forceinline__ void forEachCorner(const Net &net, int l, float px, float py, float pz, Fn fn) {
    const float res = net.levelScale[l];
    const uint32_t ires = static_cast<uint32_t>(res);
    const uint32_t T = 1u << net.log2Table;
    const bool dense = static_cast<double>(ires + 1) * (ires + 1) * (ires + 1) <= static_cast<double>(T);
    float x = px * res, y = py * res, z = pz * res;
    float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    uint32_t cx = static_cast<uint32_t>(fx), cy = static_cast<uint32_t>(fy), cz = static_cast<uint32_t>(fz);
    cx = cx > ires - 1 ? ires - 1 : cx;
    cy = cy > ires - 1 ? ires - 1 : cy;
    cz = cz > ires - 1 ? ires - 1 : cz;
    float tx = x - static_cast<float>(cx), ty = y - static_cast<float>(cy), tz = z - static_cast<float>(cz);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const uint32_t dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        const float w = (dx ? tx : 1.0f - tx) * (dy ? ty : 1.0f - ty) * (dz ? tz : 1.0f - tz);
        fn(hashCorner(cx + dx, cy + dy, cz + dz, ires, T - 1, dense), w);
    }
}

// Real spherical harmonics, degrees 0-3, of a unit vector (16 values).
__device__ __forceinline__ void sphericalHarmonics(float x, float y, float z, float out[16]) {
    const float xx = x * x, yy = y * y, zz = z * z;
    out[0] = 0.28209479177f;
    out[1] = 0.48860251190f * y;
    out[2] = 0.48860251190f * z;
    out[3] = 0.48860251190f * x;
    out[4] = 1.09254843059f * x * y;
    out[5] = 1.09254843059f * y * z;
    out[6] = 0.31539156525f * (3.0f * zz - 1.0f);
    out[7] = 1.09254843059f * x * z;
    out[8] = 0.54627421529f * (xx - yy);
    out[9] = 0.59004358992f * y * (3.0f * xx - yy);
    out[10] = 2.89061144264f * x * y * z;
    out[11] = 0.45704579946f * y * (5.0f * zz - 1.0f);
    out[12] = 0.37317633259f * z * (5.0f * zz - 3.0f);
    out[13] = 0.45704579946f * x * (5.0f * zz - 1.0f);
    out[14] = 1.44530572132f * z * (xx - yy);
    out[15] = 0.59004358992f * x * (xx - 3.0f * yy);
}

__device__ __forceinline__ float3 normalisedPosition(const Net &net, float x, float y, float z) {
    auto c = [](float v) { return fminf(fmaxf(v, 0.0f), 1.0f); };
    return make_float3(c((x - net.lo.x) * net.invExtent.x), c((y - net.lo.y) * net.invExtent.y),
                       c((z - net.lo.z) * net.invExtent.z));
}

// ------------------------------------------------------------ vMF mixture
constexpr float kLogKappaMin = -4.0f;
constexpr float kLogKappaMax = 8.0f;

// log of the vMF normalisation kappa / (2 pi (1 - exp(-2 kappa))).
__device__ __forceinline__ float vmfLogNorm(float kappa) {
    return logf(kappa) - logf(2.0f * kPi) - log1pf(-expf(-2.0f * kappa));
}

__device__ __forceinline__ float mixturePdf(const Mixture &m, const V3 &w) {
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const float4 l = m.lobe[k];
        const float cosT = l.x * w.x + l.y * w.y + l.z * w.z;
        q += m.scale[k] * expf(l.w * (cosT - 1.0f));
    }
    return q;
}

// Samples the mixture: lobe by its weight (uLobe), then the direction of a
// vMF lobe by inverting its cosine CDF (W. Jakob, "Numerically stable
// sampling of the von Mises Fisher distribution on S^2", 2012).
__device__ __forceinline__ V3 mixtureSample(const Mixture &m, float uLobe, float u0, float u1) {
    int k = 0;
    float acc = 0.0f;
    for (; k < kLobes - 1; ++k) {
        acc += m.weight[k];
        if (uLobe < acc) break;
    }
    const float4 l = m.lobe[k];
    const float kappa = l.w;
    const float cosT = 1.0f + logf(u0 + (1.0f - u0) * expf(-2.0f * kappa)) / kappa;
    const float c = fminf(fmaxf(cosT, -1.0f), 1.0f);
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    float sp, cp;
    sincosf(2.0f * kPi * u1, &sp, &cp);
    V3 mu(l.x, l.y, l.z);
    V3 t = fabsf(mu.x) > 0.9f ? V3(0.0f, 1.0f, 0.0f) : V3(1.0f, 0.0f, 0.0f);
    V3 bx = normalize(cross(t, mu));
    V3 by = cross(mu, bx);
    return bx * (sinT * cp) + by * (sinT * sp) + mu * c;
}

// Decode the 40 raw outputs into a mixture (no gradients).
__device__ __forceinline__ void decodeMixture(const float raw[kRaw], Mixture &m) {
    float mx = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, raw[5 * k + 4]);
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        float e = expf(raw[5 * k + 4] - mx);
        m.weight[k] = e;
        sum += e;
        const float vx = raw[5 * k], vy = raw[5 * k + 1], vz = raw[5 * k + 2];
        const float len = sqrtf(vx * vx + vy * vy + vz * vz);
        const float inv = len > 1e-12f ? 1.0f / len : 0.0f;
        const float kappa = expf(fminf(fmaxf(raw[5 * k + 3], kLogKappaMin), kLogKappaMax));
        m.lobe[k] = len > 1e-12f ? make_float4(vx * inv, vy * inv, vz * inv, kappa) : make_float4(0.f, 0.f, 1.f, kappa);
    }
    const float inv = 1.0f / sum;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        m.weight[k] *= inv;
        m.scale[k] = m.weight[k] * expf(vmfLogNorm(m.lobe[k].w));
    }
}

} // namespace guide
} // namespace vlrb
