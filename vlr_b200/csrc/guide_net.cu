// Guiding network: parameter storage, initialisation, optimiser, and the C
// entry points that run inference and training on host or device buffers.
#include "guide_net.h"
#include "guide_train.cuh"
#include "vlrb_internal.h"

#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace vlrb {
namespace guide {

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("guide ") + what + ": " + cudaGetErrorString(e));
}

namespace {

// FP32 master weights -> BF16 chunk-major tile image.
__global__ void packWeightsKernel(const float* w, uint8_t* tiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kNumWeights) return;
    int l = 0;
    while (i >= weightOffset(l + 1)) ++l;
    const int local = i - weightOffset(l);
    const int r = local / kIn, c = local % kIn;
    __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
    *reinterpret_cast<__nv_bfloat16*>(tiles + tileOffset(l) + umma::chunkOffset(layerOut(l), r, c)) = b;
}

// Adam (Kingma & Ba 2015) with bias correction; the gradient is consumed
// (zeroed).  sparse: entries whose gradient is exactly zero keep their
// parameter and moments (hash-grid entries no sample touched).
__global__ void adamKernel(float* param, float* grad, float* m, float* v, size_t n, float lr, float beta1,
                           float beta2, float eps, float corr1, float corr2, bool sparse, uint32_t rowMask) {
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const float g = grad[i];
        if (sparse && g == 0.0f) continue;
        grad[i] = 0.0f;
        const float mi = beta1 * m[i] + (1.0f - beta1) * g;
        const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
        m[i] = mi;
        v[i] = vi;
        param[i] -= lr * (mi / corr1) / (sqrtf(vi / corr2) + eps);
    }
    (void)rowMask;
}

__global__ void sumWeightsKernel(const Sample* s, uint32_t n, const uint32_t* countDev, float* out) {
    if (countDev) n = min(*countDev, n);
    float acc = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc += s[i].posWeight.w;
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

struct ArraySrc {
    const float* pos;
    const float* wo;
    const float* nrm;
    uint32_t n;
    Net net;
    __device__ uint32_t count() const { return n; }
    __device__ bool load(uint32_t i, float3* p, V3* w, V3* nn) const {
        *p = normalisedPosition(net, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        *w = V3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        *nn = V3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
        return true;
    }
};

struct RawDst {
    float* raw;
    __device__ void store(uint32_t i, const float y[kOut]) const {
        for (int k = 0; k < kRaw; ++k) raw[static_cast<size_t>(i) * kRaw + k] = y[k];
    }
};

} // namespace

GuideNet::GuideNet(uint32_t log2Table, uint64_t seed) {
    if (log2Table < 8 || log2Table > 24) throw std::runtime_error("hash table size out of range");
    ck(cudaGetDevice(&device), "device");
    ck(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device), "SMs");
    net = Net{};
    net.log2Table = log2Table;
    // resolutions 16 .. 2048, geometric
    const double growth = std::exp(std::log(2048.0 / 16.0) / (kLevels - 1));
    for (int l = 0; l < kLevels; ++l) net.levelScale[l] = static_cast<float>(std::floor(16.0 * std::pow(growth, l)));
    net.lo = make_float3(0.f, 0.f, 0.f);
    net.invExtent = make_float3(1.f, 1.f, 1.f);
    const size_t g = gridFloats();
    const size_t bytes = 4 * g * 4 + 4 * size_t(kNumWeights) * 4 + kWeightTileBytes + 256 +
                         size_t(numSMs) * kDwSlabFloats * 4 + 64;
    ck(cudaMalloc(&mem, bytes), "alloc");
    char* p = static_cast<char*>(mem);
    auto take = [&](size_t b) { char* r = p; p += (b + 255) & ~size_t(255); return r; };
    net.grid = reinterpret_cast<float*>(take(g * 4));
    net.gridGrad = reinterpret_cast<float*>(take(g * 4));
    net.gridM = reinterpret_cast<float*>(take(g * 4));
    net.gridV = reinterpret_cast<float*>(take(g * 4));
    net.w = reinterpret_cast<float*>(take(kNumWeights * 4));
    net.wGrad = reinterpret_cast<float*>(take(kNumWeights * 4));
    net.wM = reinterpret_cast<float*>(take(kNumWeights * 4));
    net.wV = reinterpret_cast<float*>(take(kNumWeights * 4));
    net.wTiles = reinterpret_cast<uint8_t*>(take(kWeightTileBytes));
    dwSlabs = reinterpret_cast<float*>(take(size_t(numSMs) * kDwSlabFloats * 4));
    scalars = reinterpret_cast<float*>(take(64));
    err = reinterpret_cast<uint32_t*>(scalars + 8);
    ck(cudaMemset(mem, 0, bytes), "clear");
    // initialisation: grid U(-1e-4, 1e-4); layers U(-sqrt(6/fan_in), +) (He
    // uniform for the ReLU layers), output layer scaled by 0.1
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<float> u01(0.0f, 1.0f);
    std::vector<float> hg(g), hw(kNumWeights, 0.0f);
    for (auto &x : hg) x = (u01(gen) * 2.0f - 1.0f) * 1e-4f;
    for (int l = 0; l < kNumLayers; ++l) {
        const float bound = std::sqrt(6.0f / kIn) * (l == kNumLayers - 1 ? 0.1f : 1.0f);
        const int rows = l == kNumLayers - 1 ? kRaw : layerOut(l);
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < kIn; ++c) hw[weightOffset(l) + r * kIn + c] = (u01(gen) * 2.0f - 1.0f) * bound;
    }
    setParams(hw.data(), hg.data());
}

GuideNet::~GuideNet() {
    if (mem) cudaFree(mem);
}

size_t GuideNet::gridFloats() const { return size_t(kLevels) * kFeatPerLevel << net.log2Table; }

void GuideNet::setBounds(const float lo[3], const float hi[3]) {
    net.lo = make_float3(lo[0], lo[1], lo[2]);
    auto inv = [](float a, float b) { return b > a ? 1.0f / (b - a) : 1.0f; };
    net.invExtent = make_float3(inv(lo[0], hi[0]), inv(lo[1], hi[1]), inv(lo[2], hi[2]));
}

void GuideNet::setParams(const float* w, const float* g) {
    if (w) {
        std::vector<float> hw(w, w + kNumWeights);
        // the padding rows of the output layer stay zero
        for (int r = kRaw; r < kOut; ++r)
            for (int c = 0; c < kIn; ++c) hw[weightOffset(3) + r * kIn + c] = 0.0f;
        ck(cudaMemcpy(net.w, hw.data(), kNumWeights * 4, cudaMemcpyHostToDevice), "weights");
        packWeightsKernel<<<(kNumWeights + 255) / 256, 256>>>(net.w, net.wTiles);
        ck(cudaGetLastError(), "pack");
    }
    if (g) ck(cudaMemcpy(net.grid, g, gridFloats() * 4, cudaMemcpyHostToDevice), "grid");
    ck(cudaDeviceSynchronize(), "set params");
}

void GuideNet::getParams(float* w, float* g) const {
    if (w) ck(cudaMemcpy(w, net.w, kNumWeights * 4, cudaMemcpyDeviceToHost), "weights");
    if (g) ck(cudaMemcpy(g, net.grid, gridFloats() * 4, cudaMemcpyDeviceToHost), "grid");
}

void GuideNet::inferArrays(const float* pos, const float* wo, const float* nrm, uint32_t n, float* raw,
                           cudaStream_t stream) {
    if (n == 0) return;
    ArraySrc src{ pos, wo, nrm, n, net };
    RawDst dst{ raw };
    auto kern = guideInferKernel<ArraySrc, RawDst>;
    ck(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmemBytes), "smem attr");
    const uint32_t tiles = (n + kRows - 1) / kRows;
    const uint32_t grid = tiles < uint32_t(numSMs) * 3 ? tiles : uint32_t(numSMs) * 3;
    kern<<<grid, kInferThreads, kInferSmemBytes, stream>>>(net, src, dst, err);
    ck(cudaGetLastError(), "infer launch");
}

void GuideNet::gradients(const Sample* samples, uint32_t n, cudaStream_t stream, const uint32_t* countDev) {
    ck(cudaMemsetAsync(scalars, 0, 8 * 4, stream), "scalars");
    if (n == 0) return;
    sumWeightsKernel<<<numSMs * 4, 256, 0, stream>>>(samples, n, countDev, scalars);
    ck(cudaFuncSetAttribute(guideTrainKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmemBytes),
       "smem attr");
    const uint32_t tiles = (n + kRows - 1) / kRows;
    const uint32_t grid = tiles < uint32_t(numSMs) ? tiles : uint32_t(numSMs);
    TrainArgs a{ samples, n, countDev, scalars, weightClamp, dwSlabs, scalars + 1, err };
    guideTrainKernel<<<grid, kTrainThreads, kTrainSmemBytes, stream>>>(net, a);
    reduceDwKernel<<<(kDwSlabFloats + 255) / 256, 256, 0, stream>>>(dwSlabs, grid, net.wGrad);
    ck(cudaGetLastError(), "train launch");
}

void GuideNet::step(float lr, cudaStream_t stream) {
    ++adamStep;
    const float b1 = 0.9f, b2 = 0.99f;
    const float c1 = 1.0f - std::pow(b1, float(adamStep)), c2 = 1.0f - std::pow(b2, float(adamStep));
    adamKernel<<<numSMs * 4, 256, 0, stream>>>(net.grid, net.gridGrad, net.gridM, net.gridV, gridFloats(), lr, b1, b2,
                                               1e-15f, c1, c2, true, 0);
    adamKernel<<<(kNumWeights + 255) / 256, 256, 0, stream>>>(net.w, net.wGrad, net.wM, net.wV, kNumWeights, lr, b1,
                                                              b2, 1e-8f, c1, c2, false, 0);
    packWeightsKernel<<<(kNumWeights + 255) / 256, 256, 0, stream>>>(net.w, net.wTiles);
    ck(cudaGetLastError(), "adam launch");
}

uint32_t GuideNet::errorBits() const {
    uint32_t e = 0;
    ck(cudaMemcpy(&e, err, 4, cudaMemcpyDeviceToHost), "err");
    return e;
}

float GuideNet::lastLoss() const {
    float l = 0.0f;
    ck(cudaMemcpy(&l, scalars + 1, 4, cudaMemcpyDeviceToHost), "loss");
    return l;
}

} // namespace guide
} // namespace vlrb

// ------------------------------------------------------------ C entry points
using vlrb::guide::GuideNet;

namespace {

struct DevMem {
    void* p = nullptr;
    ~DevMem() { if (p) cudaFree(p); }
    void alloc(size_t b) {
        cudaError_t e = cudaMalloc(&p, b > 0 ? b : 1);
        if (e != cudaSuccess) throw std::runtime_error(std::string("guide buffer: ") + cudaGetErrorString(e));
    }
};

template <class F>
VLRResult guarded(const char* name, F f) {
    try {
        f();
        return VLRResult_NoError;
    }
    catch (const std::exception &ex) {
        std::fprintf(stderr, "%s: %s\n", name, ex.what());
        return VLRResult_InternalError;
    }
}

} // namespace

extern "C" VLRResult vlrbGuideNetCreate(uint32_t log2TableSize, uint64_t seed, VLRBGuideNet* net) {
    if (!net || log2TableSize < 8 || log2TableSize > 24) return VLRResult_InvalidArgument;
    return guarded("vlrbGuideNetCreate", [&] { *net = new VLRBGuideNet_API{ new GuideNet(log2TableSize, seed), true }; });
}

extern "C" VLRResult vlrbGuideNetDestroy(VLRBGuideNet net) {
    if (!net) return VLRResult_InvalidInstance;
    if (net->owned) delete net->impl;
    delete net;
    return VLRResult_NoError;
}

extern "C" VLRResult vlrbGuideNetSetBounds(VLRBGuideNet net, const float* lo, const float* hi) {
    if (!net) return VLRResult_InvalidInstance;
    if (!lo || !hi) return VLRResult_InvalidArgument;
    net->impl->setBounds(lo, hi);
    return VLRResult_NoError;
}

extern "C" VLRResult vlrbGuideNetGetSizes(VLRBGuideNet net, uint32_t* numWeights, uint64_t* numGridFloats) {
    if (!net) return VLRResult_InvalidInstance;
    if (numWeights) *numWeights = vlrb::guide::kNumWeights;
    if (numGridFloats) *numGridFloats = net->impl->gridFloats();
    return VLRResult_NoError;
}

extern "C" VLRResult vlrbGuideNetGetParams(VLRBGuideNet net, float* weights, float* grid) {
    if (!net) return VLRResult_InvalidInstance;
    return guarded("vlrbGuideNetGetParams", [&] { net->impl->getParams(weights, grid); });
}

extern "C" VLRResult vlrbGuideNetSetParams(VLRBGuideNet net, const float* weights, const float* grid) {
    if (!net) return VLRResult_InvalidInstance;
    return guarded("vlrbGuideNetSetParams", [&] { net->impl->setParams(weights, grid); });
}

extern "C" VLRResult vlrbGuideNetInferHost(VLRBGuideNet net, uint32_t n, const float* pos, const float* wo,
                                           const float* nrm, float* raw) {
    if (!net) return VLRResult_InvalidInstance;
    if (n > 0 && (!pos || !wo || !nrm || !raw)) return VLRResult_InvalidArgument;
    return guarded("vlrbGuideNetInferHost", [&] {
        if (n == 0) return;
        DevMem d;
        const size_t in = size_t(n) * 3 * 4, out = size_t(n) * vlrb::guide::kRaw * 4;
        d.alloc(3 * in + out);
        char* b = static_cast<char*>(d.p);
        cudaMemcpy(b, pos, in, cudaMemcpyHostToDevice);
        cudaMemcpy(b + in, wo, in, cudaMemcpyHostToDevice);
        cudaMemcpy(b + 2 * in, nrm, in, cudaMemcpyHostToDevice);
        net->impl->inferArrays(reinterpret_cast<float*>(b), reinterpret_cast<float*>(b + in),
                               reinterpret_cast<float*>(b + 2 * in), n, reinterpret_cast<float*>(b + 3 * in), nullptr);
        vlrb::guide::ck(cudaMemcpy(raw, b + 3 * in, out, cudaMemcpyDeviceToHost), "raw");
        if (net->impl->errorBits()) throw std::runtime_error("tensor-core wait timed out");
    });
}

extern "C" VLRResult vlrbGuideNetGradientsHost(VLRBGuideNet net, uint32_t n, const float* samples,
                                               float* weightGrad, float* gridGrad, float* loss) {
    if (!net) return VLRResult_InvalidInstance;
    if (n > 0 && !samples) return VLRResult_InvalidArgument;
    return guarded("vlrbGuideNetGradientsHost", [&] {
        GuideNet &G = *net->impl;
        DevMem d;
        d.alloc(size_t(n) * sizeof(vlrb::guide::Sample));
        vlrb::guide::ck(cudaMemcpy(d.p, samples, size_t(n) * sizeof(vlrb::guide::Sample), cudaMemcpyHostToDevice),
                        "samples");
        vlrb::guide::ck(cudaMemset(G.net.gridGrad, 0, G.gridFloats() * 4), "grid grad");
        vlrb::guide::ck(cudaMemset(G.net.wGrad, 0, vlrb::guide::kNumWeights * 4), "w grad");
        G.gradients(static_cast<const vlrb::guide::Sample*>(d.p), n, nullptr);
        vlrb::guide::ck(cudaDeviceSynchronize(), "gradients");
        if (G.errorBits()) throw std::runtime_error("tensor-core wait timed out");
        if (weightGrad)
            vlrb::guide::ck(cudaMemcpy(weightGrad, G.net.wGrad, vlrb::guide::kNumWeights * 4, cudaMemcpyDeviceToHost),
                            "w grad out");
        if (gridGrad)
            vlrb::guide::ck(cudaMemcpy(gridGrad, G.net.gridGrad, G.gridFloats() * 4, cudaMemcpyDeviceToHost),
                            "grid grad out");
        if (loss) *loss = G.lastLoss();
    });
}

extern "C" VLRResult vlrbGuideNetTrainHost(VLRBGuideNet net, uint32_t n, const float* samples, float learningRate,
                                           uint32_t steps, float* lossPerStep) {
    if (!net) return VLRResult_InvalidInstance;
    if (n > 0 && !samples) return VLRResult_InvalidArgument;
    return guarded("vlrbGuideNetTrainHost", [&] {
        GuideNet &G = *net->impl;
        DevMem d;
        d.alloc(size_t(n) * sizeof(vlrb::guide::Sample));
        vlrb::guide::ck(cudaMemcpy(d.p, samples, size_t(n) * sizeof(vlrb::guide::Sample), cudaMemcpyHostToDevice),
                        "samples");
        for (uint32_t s = 0; s < steps; ++s) {
            G.gradients(static_cast<const vlrb::guide::Sample*>(d.p), n, nullptr);
            G.step(learningRate, nullptr);
            if (lossPerStep) lossPerStep[s] = G.lastLoss();
        }
        vlrb::guide::ck(cudaDeviceSynchronize(), "train");
        if (G.errorBits()) throw std::runtime_error("tensor-core wait timed out");
    });
}
