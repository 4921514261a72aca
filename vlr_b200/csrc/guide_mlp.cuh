// Guiding network kernels on the sm_100a tensor cores.
//
// A CTA owns one 128-sample tile at a time; sample row t is TMEM lane t of
// the M = 128 accumulators (the 32x32b TMEM load shape gives warp w lanes
// 32 (w mod 4) .. +31).  Per layer:
//   threads write their row of BF16 activations into a chunk-major shared
//   tile -> fence.proxy.async -> barrier -> thread 0 issues the K/16
//   tcgen05.mma steps and a tcgen05.commit on an mbarrier -> every thread
//   waits (bounded), loads its row of FP32 accumulators from TMEM, applies
//   the activation and writes the next tile.
// Weights stay in shared memory for the CTA's lifetime (30 KB of BF16).
#pragma once

#include "guide.cuh"
#include "umma.cuh"

namespace vlrb {
namespace guide {

constexpr uint32_t kActTileBytes = kRows * kIn * 2;   // 16 KB: 128 rows x 64 BF16

__device__ __forceinline__ uint32_t packBf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// Row r of a chunk-major BF16 tile with R rows: ncols values (multiple of 8).
__device__ __forceinline__ void storeRow(uint8_t* tile, uint32_t R, uint32_t r, const float* v, int ncols) {
#pragma unroll
    for (int c = 0; c < ncols / 8; ++c) {
        uint4 q;
        q.x = packBf16x2(v[8 * c + 0], v[8 * c + 1]);
        q.y = packBf16x2(v[8 * c + 2], v[8 * c + 3]);
        q.z = packBf16x2(v[8 * c + 4], v[8 * c + 5]);
        q.w = packBf16x2(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(tile + c * R * 16u + r * 16u) = q;
    }
}

__device__ __forceinline__ void loadRow(const uint8_t* tile, uint32_t R, uint32_t r, float* v, int ncols) {
#pragma unroll
    for (int c = 0; c < ncols / 8; ++c) {
        uint4 q = *reinterpret_cast<const uint4*>(tile + c * R * 16u + r * 16u);
        const uint32_t w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
            float2 f = __bfloat1622float2(h);
            v[8 * c + 2 * i] = f.x;
            v[8 * c + 2 * i + 1] = f.y;
        }
    }
}

// 64 input features of one sample: hash grid (32), SH of wo (16), SH of the
// shading normal (16).
__device__ __forceinline__ void encode(const Net &net, float3 p, const V3 &wo, const V3 &n, float f[kIn]) {
#pragma unroll
    for (int l = 0; l < kLevels; ++l) {
        const float* table = net.grid + (static_cast<size_t>(l) << net.log2Table) * kFeatPerLevel;
        float a = 0.0f, b = 0.0f;
        forEachCorner(net, l, p.x, p.y, p.z, [&](uint32_t idx, float w) {
            const float2 g = __ldg(reinterpret_cast<const float2*>(table) + idx);
            a += w * g.x;
            b += w * g.y;
        });
        f[2 * l] = a;
        f[2 * l + 1] = b;
    }
    sphericalHarmonics(wo.x, wo.y, wo.z, f + kGridFeatures);
    sphericalHarmonics(n.x, n.y, n.z, f + kGridFeatures + 16);
}

// D (TMEM) = A x B over `kSteps` K = 16 steps, issued by one thread.
// A and B are chunk-major tiles read K-major or MN-major (umma.cuh).
__device__ __forceinline__ void issueGemm(uint32_t dTmem, uint32_t aTile, uint32_t aRows, bool aMN, uint32_t bTile,
                                          uint32_t bRows, bool bMN, uint32_t M, uint32_t N, uint32_t kSteps,
                                          bool accumulate) {
    const uint32_t idesc = umma::instrDescBf16(M, N, aMN, bMN);
    for (uint32_t ks = 0; ks < kSteps; ++ks) {
        const uint64_t da = aMN ? umma::descMNMajor(aTile, aRows, ks) : umma::descKMajor(aTile, aRows, ks);
        const uint64_t db = bMN ? umma::descMNMajor(bTile, bRows, ks) : umma::descKMajor(bTile, bRows, ks);
        umma::mmaBf16(dTmem, da, db, idesc, accumulate || ks > 0);
    }
}

// Copies the BF16 weight tile image into shared memory (16-byte vectors).
__device__ __forceinline__ void loadWeightTiles(const Net &net, uint8_t* sW) {
    const uint4* src = reinterpret_cast<const uint4*>(net.wTiles);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    for (uint32_t i = threadIdx.x; i < kWeightTileBytes / 16; i += blockDim.x) dst[i] = src[i];
}

// Error bits reported through the kernels' error word.
constexpr uint32_t kErrMmaTimeout = 1u;

// Row r of a chunk-major tile: `nchunks` 8-column chunks starting at chunk c0.
__device__ __forceinline__ void storeChunks(uint8_t* tile, uint32_t R, uint32_t r, const float* v, int c0,
                                            int nchunks) {
#pragma unroll
    for (int c = 0; c < nchunks; ++c) {
        uint4 q;
        q.x = packBf16x2(v[8 * c + 0], v[8 * c + 1]);
        q.y = packBf16x2(v[8 * c + 2], v[8 * c + 3]);
        q.z = packBf16x2(v[8 * c + 4], v[8 * c + 5]);
        q.w = packBf16x2(v[8 * c + 6], v[8 * c + 7]);
        *reinterpret_cast<uint4*>(tile + (c0 + c) * R * 16u + r * 16u) = q;
    }
}

// Hash-grid features of levels [l0, l0 + 8) (16 values).
__device__ __forceinline__ void encodeLevels(const Net &net, float3 p, int l0, float f[16]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int l = l0 + j;
        const float* table = net.grid + (static_cast<size_t>(l) << net.log2Table) * kFeatPerLevel;
        float a = 0.0f, b = 0.0f;
        forEachCorner(net, l, p.x, p.y, p.z, [&](uint32_t idx, float w) {
            const float2 g = __ldg(reinterpret_cast<const float2*>(table) + idx);
            a += w * g.x;
            b += w * g.y;
        });
        f[2 * j] = a;
        f[2 * j + 1] = b;
    }
}

// Forward pass over tiles of queries.  Src provides
//   uint32_t count() const;
//   bool load(uint32_t i, float3* pos01, V3* wo, V3* nrm) const;   // false: padding row
// and Dst provides  void store(uint32_t i, const float raw[kRaw]) const.
// One thread per row (128 threads): each warp fetches, encodes and writes
// its rows without waiting for the others, which hides the gather latency
// better than splitting rows over two threads (measured: 0.74 vs 1.31 ms for
// the first-bounce queries of a 1024^2 x 4 spp launch).  Shared memory:
// weights (30 KB) + two activation tiles (32 KB) + barrier.
constexpr uint32_t kInferThreads = kRows;
constexpr uint32_t kInferSmemBytes = kWeightTileBytes + 2 * kActTileBytes + 64;

template <class Src, class Dst>
__global__ void __launch_bounds__(kInferThreads) guideInferKernel(Net net, Src src, Dst dst, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sW = smem;
    uint8_t* sT[2] = { smem + kWeightTileBytes, smem + kWeightTileBytes + kActTileBytes };
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kWeightTileBytes + 2 * kActTileBytes);
    uint32_t* slot = reinterpret_cast<uint32_t*>(mbar + 1);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;

    loadWeightTiles(net, sW);
    if (warp == 0) umma::tmemAlloc(slot, 64);
    if (tid == 0) umma::mbarInit(mbar, 1);
    umma::fenceProxyAsync();
    umma::fenceBeforeSync();
    __syncthreads();
    umma::fenceAfterSync();
    const uint32_t tmem = *slot;
    const uint32_t wAddr = umma::smemAddr(sW);
    const uint32_t tAddr[2] = { umma::smemAddr(sT[0]), umma::smemAddr(sT[1]) };
    uint32_t phase = 0;
    const uint32_t n = src.count();
    bool ok = true;
    for (uint32_t tile = blockIdx.x; ok && tile * kRows < n; tile += gridDim.x) {
        const uint32_t row = tile * kRows + tid;
        float f[kIn];
        float3 p;
        V3 wo, nrm;
        bool valid = row < n && src.load(row, &p, &wo, &nrm);
        if (valid) encode(net, p, wo, nrm, f);
        else {
#pragma unroll
            for (int i = 0; i < kIn; ++i) f[i] = 0.0f;
        }
        storeRow(sT[0], kRows, tid, f, kIn);
        int cur = 0;
        for (int l = 0; l < kNumLayers; ++l) {
            umma::fenceProxyAsync();
            umma::fenceBeforeSync();
            __syncthreads();
            if (tid == 0) {
                umma::fenceAfterSync();
                issueGemm(tmem, tAddr[cur], kRows, false, wAddr + tileOffset(l), layerOut(l), false, kRows,
                          layerOut(l), kIn / 16, false);
                umma::commit(mbar);
            }
            const bool done = umma::mbarWait(mbar, phase);
            phase ^= 1u;
            umma::fenceAfterSync();
            if (!__syncthreads_and(done)) {
                if (tid == 0) atomicOr(err, kErrMmaTimeout);
                ok = false;
                break;
            }
            if (l < kNumLayers - 1) {
                float h[kHidden];
#pragma unroll
                for (int c = 0; c < kHidden; c += 16) umma::tmemLoad16(umma::tmemAt(tmem, 32 * warp, c), h + c);
#pragma unroll
                for (int i = 0; i < kHidden; ++i) h[i] = fmaxf(h[i], 0.0f);
                storeRow(sT[cur ^ 1], kRows, tid, h, kHidden);
                cur ^= 1;
            }
            else {
                float y[kOut];
#pragma unroll
                for (int c = 0; c < kOut; c += 16) umma::tmemLoad16(umma::tmemAt(tmem, 32 * warp, c), y + c);
                if (valid) dst.store(row, y);
                umma::fenceBeforeSync();
                __syncthreads();   // TMEM and tiles free for the next tile
            }
        }
    }
    umma::fenceBeforeSync();
    __syncthreads();
    if (warp == 0) umma::tmemFree(tmem, 64);
}

} // namespace guide
} // namespace vlrb
