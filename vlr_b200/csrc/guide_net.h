// Host side of the guiding network (implemented in guide_net.cu).
#pragma once

#include "guide.cuh"
#include <cuda_runtime.h>

namespace vlrb {
namespace guide {

class GuideNet {
public:
    GuideNet(uint32_t log2Table, uint64_t seed);
    ~GuideNet();
    GuideNet(const GuideNet &) = delete;
    GuideNet &operator=(const GuideNet &) = delete;

    size_t gridFloats() const;
    void setBounds(const float lo[3], const float hi[3]);
    void setParams(const float* weights, const float* grid);   // host arrays, either may be null
    void getParams(float* weights, float* grid) const;
    // raw[n][40] = network outputs for queries given as device arrays.
    void inferArrays(const float* pos, const float* wo, const float* nrm, uint32_t n, float* raw,
                     cudaStream_t stream);
    // Gradients of the batch loss into net.wGrad / net.gridGrad (the grid
    // gradient accumulates; the optimiser step consumes it).
    // countDev (optional): device word holding the number of valid samples
    // (at most n); the launch then needs no host round trip.
    void gradients(const Sample* samples, uint32_t n, cudaStream_t stream, const uint32_t* countDev = nullptr);
    void step(float lr, cudaStream_t stream);
    uint32_t errorBits() const;
    float lastLoss() const;

    Net net;
    int device = 0;
    int numSMs = 148;
    uint32_t adamStep = 0;
    float weightClamp = 0.0f;   // > 0: clip training weights above this multiple of the batch mean
    float* dwSlabs = nullptr;
    float* scalars = nullptr;   // [0] batch weight sum, [1] batch loss
    uint32_t* err = nullptr;

private:
    void* mem = nullptr;
};

} // namespace guide
} // namespace vlrb

// Handle behind VLRBGuideNet: a network the handle owns, or a context's
// network lent out by vlrbContextGetGuideNet.
struct VLRBGuideNet_API {
    vlrb::guide::GuideNet* impl;
    bool owned;
};
