// BSDF shading batch, exact build: this translation unit is compiled with
// -fmad=false so every product and sum is rounded exactly like the
// reference's host build (materials.cu classes compiled by g++ for x86-64,
// which has no fused multiply-add).
#define VLRB_BATCH_NS exact
#include "bsdf_batch.cuh"

namespace vlrb {

cudaError_t launchBsdfBatch(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs) {
    return exact::launch(b, stream, kernelMs);
}

} // namespace vlrb
