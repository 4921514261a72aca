// Internal declarations shared by the library's translation units.
#pragma once

#include "../../include/vlrb.h"
#include <cuda_runtime.h>

namespace vlrb {

// bsdf_batch.cu (no FMA contraction) and bsdf_batch_contracted.cu (FMA)
cudaError_t launchBsdfBatch(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs);
cudaError_t launchBsdfBatchContracted(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs);

} // namespace vlrb
