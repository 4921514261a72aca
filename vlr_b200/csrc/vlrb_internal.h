// Internal declarations shared by the library's translation units.
#pragma once

#include "../../include/vlrb.h"
#include <cuda_runtime.h>

namespace vlrb {

// bsdf_batch.cu
cudaError_t launchBsdfBatch(const VLRBBsdfBatch &b, cudaStream_t stream, float* kernelMs);

} // namespace vlrb
