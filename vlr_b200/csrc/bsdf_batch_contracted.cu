// BSDF shading batch, contracted build: the same kernel as bsdf_batch.cu
// compiled with nvcc's default FMA contraction, as the renderers' shading
// kernels are, so the error of the render path's BSDF arithmetic against the
// reference can be measured query by query.
#define VLRB_BATCH_NS contracted
#include "bsdf_batch.cuh"

namespace vlrb {

cudaError_t launchBsdfBatchContracted(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs) {
    return contracted::launch(b, stream, kernelMs);
}

} // namespace vlrb
