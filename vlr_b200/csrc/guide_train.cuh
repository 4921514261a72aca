// Training step of the guiding network: forward, KL-loss gradient at the
// mixture outputs, backward through the MLP on the tensor cores, weight
// gradients accumulated in TMEM across the CTA's tiles, hash-grid gradients
// scattered with atomics.
//
// Per 128-sample tile (sample row t = TMEM lane t):
//   forward   X -> A1 -> A2 -> A3 -> Y as in inference, keeping X and the
//             three hidden activation tiles in shared memory;
//   output    dY = d loss / d raw outputs per row (FP32 in registers, stored
//             as BF16, columns 40..63 zero);
//   per layer l = 3..0 (two products per commit):
//             dA_in  = dZ_l x W_l        (M 128, dZ read K-major, W MN-major)
//             dW_l  += dZ_l^T x A_in     (M 64, both tiles read MN-major)
//             dZ_{l-1} = dA_in * (A_in > 0)
//   grid      dX[0..31] (layer 0 only needs its first 32 columns) is spread
//             over the 8 trilinear corners of every level with atomics.
// TMEM: columns 0..63 for the M = 128 products, 64 + 64 l for dW_l.
// At the end each CTA writes its four dW partial sums to a global slab;
// a second kernel sums the slabs in a fixed order.
#pragma once

#include "guide_mlp.cuh"

namespace vlrb {
namespace guide {

constexpr uint32_t kTrainSmemBytes = kWeightTileBytes + 6 * kActTileBytes + 64;
constexpr uint32_t kTrainTmemCols = 512;
constexpr uint32_t kDwSlabFloats = kNumLayers * kHidden * kHidden;   // per CTA

struct TrainArgs {
    const Sample* samples;
    uint32_t count;            // buffer capacity (or the exact count when countDev is null)
    const uint32_t* countDev;  // device sample count (clamped to count), or null
    const float* weightSum;    // device: sum of the batch's sample weights
    float weightClamp;         // > 0: weights above this multiple of the batch mean are clipped
    float* dwSlabs;            // [gridDim.x][4][64][64]
    float* lossSum;            // device accumulator of the batch loss
    uint32_t* err;
};

// d(-w log q)/d raw outputs for one sample; returns -w log q.
__device__ __forceinline__ float mixtureLossGrad(const float raw[kOut], const V3 &wi, float w, float dy[kOut]) {
    float logit[kLobes], logComp[kLobes], kappa[kLobes], cosT[kLobes], len[kLobes];
    V3 mu[kLobes];
    float mx = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) mx = fmaxf(mx, raw[5 * k + 4]);
    float se = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) { logit[k] = raw[5 * k + 4] - mx; se += expf(logit[k]); }
    const float logSe = logf(se);
    float lmax = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const V3 v(raw[5 * k], raw[5 * k + 1], raw[5 * k + 2]);
        len[k] = v.length();
        mu[k] = len[k] > 1e-12f ? v / len[k] : V3(0.0f, 0.0f, 1.0f);
        kappa[k] = expf(fminf(fmaxf(raw[5 * k + 3], kLogKappaMin), kLogKappaMax));
        cosT[k] = dot(mu[k], wi);
        logComp[k] = (logit[k] - logSe) + vmfLogNorm(kappa[k]) + kappa[k] * (cosT[k] - 1.0f);
        lmax = fmaxf(lmax, logComp[k]);
    }
    float sq = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) sq += expf(logComp[k] - lmax);
    const float logQ = lmax + logf(sq);
#pragma unroll
    for (int i = 0; i < kOut; ++i) dy[i] = 0.0f;
#pragma unroll
    for (int k = 0; k < kLobes; ++k) {
        const float r = expf(logComp[k] - logQ);             // responsibility
        const float pi = expf(logit[k] - logSe);
        dy[5 * k + 4] = -w * (r - pi);
        const float s = raw[5 * k + 3];
        if (s > kLogKappaMin && s < kLogKappaMax) {
            const float dLogPdfDKappa = 1.0f / kappa[k] - 2.0f / expm1f(2.0f * kappa[k]) + (cosT[k] - 1.0f);
            dy[5 * k + 3] = -w * r * kappa[k] * dLogPdfDKappa;
        }
        if (len[k] > 1e-12f) {
            // d/dmu = -w r kappa wi; through mu = v / |v|
            const V3 g = wi * (-w * r * kappa[k]);
            const V3 gv = (g - mu[k] * dot(mu[k], g)) / len[k];
            dy[5 * k + 0] = gv.x;
            dy[5 * k + 1] = gv.y;
            dy[5 * k + 2] = gv.z;
        }
    }
    return -w * logQ;
}

// Row r of a chunk-major tile: `nchunks` 8-column chunks starting at c0.
__device__ __forceinline__ void loadChunks(const uint8_t* tile, uint32_t R, uint32_t r, float* v, int c0,
                                           int nchunks) {
#pragma unroll
    for (int c = 0; c < nchunks; ++c) {
        uint4 q = *reinterpret_cast<const uint4*>(tile + (c0 + c) * R * 16u + r * 16u);
        const uint32_t w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[i]));
            v[8 * c + 2 * i] = f.x;
            v[8 * c + 2 * i + 1] = f.y;
        }
    }
}

// 256 threads per 128-row tile, as in inference: thread t works on row
// t mod 128 and half h = t / 128.  Each half encodes 8 grid levels and one SH
// block, handles 32 of the 64 columns after every product, and scatters the
// hash-grid gradient of its 8 levels; half 0 computes the loss gradient.
constexpr uint32_t kTrainThreads = 2 * kRows;

__global__ void __launch_bounds__(kTrainThreads, 1) guideTrainKernel(Net net, TrainArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sW = smem;
    uint8_t* sX = smem + kWeightTileBytes;
    uint8_t* sA[3] = { sX + kActTileBytes, sX + 2 * kActTileBytes, sX + 3 * kActTileBytes };
    uint8_t* sDY = sX + 4 * kActTileBytes;
    uint8_t* sDZ = sX + 5 * kActTileBytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sX + 6 * kActTileBytes);
    uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t r = tid & (kRows - 1), half = tid / kRows, lane0 = 32 * (warp & 3);

    loadWeightTiles(net, sW);
    if (warp == 0) umma::tmemAlloc(slot, kTrainTmemCols);
    if (tid == 0) umma::mbarInit(mbar, 1);
    umma::fenceProxyAsync();
    umma::fenceBeforeSync();
    __syncthreads();
    umma::fenceAfterSync();
    const uint32_t tmem = *slot;
    const uint32_t wAddr = umma::smemAddr(sW);
    const uint32_t xAddr = umma::smemAddr(sX);
    const uint32_t aAddr[3] = { umma::smemAddr(sA[0]), umma::smemAddr(sA[1]), umma::smemAddr(sA[2]) };
    const uint32_t dyAddr = umma::smemAddr(sDY), dzAddr = umma::smemAddr(sDZ);
    const float invWeightSum = 1.0f / fmaxf(*a.weightSum, 1e-30f);
    uint32_t phase = 0;
    bool ok = true;
    uint32_t tilesDone = 0;
    float lossAcc = 0.0f;

    // Bounded wait by all threads for the latest commit; false on timeout.
    auto sync = [&]() -> bool {
        const bool done = umma::mbarWait(mbar, phase);
        phase ^= 1u;
        umma::fenceAfterSync();
        if (!__syncthreads_and(done)) {
            if (tid == 0) atomicOr(a.err, kErrMmaTimeout);
            return false;
        }
        return true;
    };
    auto beforeIssue = [&]() {
        umma::fenceProxyAsync();
        umma::fenceBeforeSync();
        __syncthreads();
    };

    const uint32_t count = a.countDev ? min(*a.countDev, a.count) : a.count;
    for (uint32_t tile = blockIdx.x; ok && tile * kRows < count; tile += gridDim.x) {
        const uint32_t row = tile * kRows + r;
        const bool valid = row < count;
        Sample s;
        if (valid) s = a.samples[row];
        else s = Sample{ make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 1.f, 0.f),
                         make_float4(0.f, 0.f, 1.f, 0.f), make_float4(0.f, 0.f, 1.f, 0.f) };
        const float3 p = normalisedPosition(net, s.posWeight.x, s.posWeight.y, s.posWeight.z);
        const V3 wi(s.wi.x, s.wi.y, s.wi.z);
        {
            float f[16];
            if (valid) encodeLevels(net, p, 8 * half, f);
            else {
#pragma unroll
                for (int i = 0; i < 16; ++i) f[i] = 0.0f;
            }
            storeChunks(sX, kRows, r, f, 2 * half, 2);
            const float4 d = half ? s.nrm : s.wo;
            sphericalHarmonics(d.x, d.y, d.z, f);
            if (!valid) {
#pragma unroll
                for (int i = 0; i < 16; ++i) f[i] = 0.0f;
            }
            storeChunks(sX, kRows, r, f, 4 + 2 * half, 2);
        }
        // ---- forward
        uint32_t in = xAddr;
        for (int l = 0; l < kNumLayers && ok; ++l) {
            beforeIssue();
            if (tid == 0) {
                umma::fenceAfterSync();
                issueGemm(tmem, in, kRows, false, wAddr + tileOffset(l), layerOut(l), false, kRows, layerOut(l),
                          kIn / 16, false);
                umma::commit(mbar);
            }
            if (!(ok = sync())) break;
            if (l < kNumLayers - 1) {
                float h[32];
                umma::tmemLoad16(umma::tmemAt(tmem, lane0, 32 * half), h);
                umma::tmemLoad16(umma::tmemAt(tmem, lane0, 32 * half + 16), h + 16);
#pragma unroll
                for (int i = 0; i < 32; ++i) h[i] = fmaxf(h[i], 0.0f);
                storeChunks(sA[l], kRows, r, h, 4 * half, 4);
                in = aAddr[l];
            }
        }
        if (!ok) break;
        // ---- loss gradient at the outputs (half 0)
        if (half == 0) {
            float y[kOut], dy[kHidden];
#pragma unroll
            for (int c = 0; c < kOut; c += 16) umma::tmemLoad16(umma::tmemAt(tmem, lane0, c), y + c);
            float w = valid ? s.posWeight.w * invWeightSum : 0.0f;
            // clipping the rare huge weights (sum-normalised: mean = 1/count)
            if (a.weightClamp > 0.0f) w = fminf(w, a.weightClamp / fmaxf(static_cast<float>(count), 1.0f));
            if (w > 0.0f) lossAcc += mixtureLossGrad(y, wi, w, dy);
            else {
#pragma unroll
                for (int i = 0; i < kOut; ++i) dy[i] = 0.0f;
            }
#pragma unroll
            for (int i = kOut; i < kHidden; ++i) dy[i] = 0.0f;
            storeRow(sDY, kRows, r, dy, kHidden);
        }
        // ---- backward, layer 3 .. 0
        const bool accumulate = tilesDone > 0;
        uint32_t dzTile = dyAddr;
        for (int l = kNumLayers - 1; l >= 0; --l) {
            const uint32_t inTile = l == 0 ? xAddr : aAddr[l - 1];
            const uint32_t nIn = l == 0 ? kGridFeatures : kHidden;
            beforeIssue();
            if (tid == 0) {
                umma::fenceAfterSync();
                // dA_in[m][k] = sum_n dZ[m][n] W[n][k]
                issueGemm(tmem, dzTile, kRows, false, wAddr + tileOffset(l), layerOut(l), true, kRows, nIn,
                          layerOut(l) / 16, false);
                // dW[n][k] += sum_m dZ[m][n] A_in[m][k]
                issueGemm(tmem + 64 + 64 * l, dzTile, kRows, true, inTile, kRows, true, 64, kHidden, kRows / 16,
                          accumulate);
                umma::commit(mbar);
            }
            if (!(ok = sync())) break;
            if (l > 0) {
                float g[32], act[32];
                umma::tmemLoad16(umma::tmemAt(tmem, lane0, 32 * half), g);
                umma::tmemLoad16(umma::tmemAt(tmem, lane0, 32 * half + 16), g + 16);
                loadChunks(sA[l - 1], kRows, r, act, 4 * half, 4);
#pragma unroll
                for (int i = 0; i < 32; ++i) g[i] = act[i] > 0.0f ? g[i] : 0.0f;
                storeChunks(sDZ, kRows, r, g, 4 * half, 4);
                dzTile = dzAddr;
            }
            else {
                float g[16];
                umma::tmemLoad16(umma::tmemAt(tmem, lane0, 16 * half), g);
                if (valid) {
#pragma unroll 1
                    for (int j = 0; j < 8; ++j) {
                        const int lv = 8 * half + j;
                        const float g0 = g[2 * j], g1 = g[2 * j + 1];
                        if (g0 == 0.0f && g1 == 0.0f) continue;
                        float* table = net.gridGrad + (static_cast<size_t>(lv) << net.log2Table) * kFeatPerLevel;
                        forEachCorner(net, lv, p.x, p.y, p.z, [&](uint32_t idx, float cw) {
                            atomicAdd(table + 2 * idx, cw * g0);
                            atomicAdd(table + 2 * idx + 1, cw * g1);
                        });
                    }
                }
            }
        }
        if (!ok) break;
        ++tilesDone;
    }
    // ---- weight-gradient partial sums of this CTA -> its slab; the M = 64
    // accumulator keeps row 16 q + i in lane 32 q + i (i < 16)
    umma::fenceBeforeSync();
    __syncthreads();
    umma::fenceAfterSync();
    float* slab = a.dwSlabs + static_cast<size_t>(blockIdx.x) * kDwSlabFloats;
    const bool holdsRow = (tid & 31) < 16;
    const uint32_t row64 = 16 * (warp & 3) + (tid & 31);
    for (int l = 0; l < kNumLayers; ++l) {
        for (int c = 32 * half; c < 32 * half + 32; c += 16) {
            float v[16];
            umma::tmemLoad16(umma::tmemAt(tmem, lane0, 64 + 64 * l + c), v);
            if (holdsRow) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    slab[l * kHidden * kHidden + row64 * kHidden + c + i] = (tilesDone > 0 && ok) ? v[i] : 0.0f;
            }
        }
    }
    // loss: block reduction then one atomic
    for (int off = 16; off > 0; off >>= 1) lossAcc += __shfl_xor_sync(0xFFFFFFFFu, lossAcc, off);
    __shared__ float sLoss[kTrainThreads / 32];
    if ((tid & 31) == 0) sLoss[warp] = lossAcc;
    umma::fenceBeforeSync();
    __syncthreads();
    if (tid == 0) {
        float t = 0.0f;
        for (uint32_t i = 0; i < kTrainThreads / 32; ++i) t += sLoss[i];
        atomicAdd(a.lossSum, t);
    }
    if (warp == 0) umma::tmemFree(tmem, kTrainTmemCols);
}

// wGrad[layer][row][col] = sum over slabs (fixed order).  Rows beyond the
// layer's output width (layer 3: 48) are skipped.
__global__ void reduceDwKernel(const float* slabs, uint32_t numSlabs, float* wGrad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kDwSlabFloats) return;
    const uint32_t l = i / (kHidden * kHidden), rc = i % (kHidden * kHidden);
    const uint32_t r = rc / kHidden, c = rc % kHidden;
    if (r >= static_cast<uint32_t>(layerOut(l))) return;
    float s = 0.0f;
    for (uint32_t b = 0; b < numSlabs; ++b) s += slabs[static_cast<size_t>(b) * kDwSlabFloats + i];
    wGrad[weightOffset(l) + r * kIn + c] = s;
}

} // namespace guide
} // namespace vlrb
