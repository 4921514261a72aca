/* libvlr_b200 extension API: entry points with no counterpart in the
 * reference's vlr.h, added for workloads the reference runs only inside its
 * renderer.  All are plain C: pointers, sizes, VLRResult codes.
 */
#ifndef VLRB_VLRB_H
#define VLRB_VLRB_H

#include "vlr.h"

#if defined(__cplusplus)
extern "C" {
#endif

/* Library build identifier, e.g. "vlr_b200 sm_100a". */
const char* vlrbVersion(void);

/* ------------------------------------------------------------------------
 * BSDF shading batch.
 *
 * One query = the reference's BSDF sample, then evaluate and evaluatePDF at
 * the sampled direction, for one of six BSDFs built from immediate values the
 * way the reference's setupBSDF callables build them
 * (libVLR/GPU_kernels/materials.cu:584-1994).  Arrays are AoS float tuples.
 *   material: 0 Matte, 1 SpecularReflection, 2 MicrofacetReflection,
 *             3 MicrofacetScattering, 4 LambertianScattering, 5 UE4.
 *   roughness[2]: per-axis roughness r; alpha = max(0.001, r^2) for the GGX
 *             materials, roughness = max(0.01, r.x) for UE4.
 *   ior: grey index of refraction (interior for the dielectric, eta of the
 *             conductors with k = 0).
 *   albedo[3]: linear Rec.709 reflectance, Meng-upsampled.
 *   u[3] = (uComponent, uDir0, uDir1); wavelengthU[2] = (offset, uSelect).
 * Outputs: value[4], pdf, wi[3], evalValue[4], evalPdf.  Queries whose sample
 * fails (pdf 0) write zeros everywhere.
 * ---------------------------------------------------------------------- */
typedef struct VLRBBsdfBatch {
    int64_t count;
    const float* wo;
    const uint32_t* material;
    const float* roughness;
    const float* ior;
    const float* albedo;
    const float* metallic;
    const float* u;
    const float* wavelengthU;
    float* value;
    float* pdf;
    float* wi;
    float* evalValue;
    float* evalPdf;
} VLRBBsdfBatch;

/* All pointers are device pointers; enqueued on `stream`, asynchronous. */
VLRResult vlrbBsdfBatch(const VLRBBsdfBatch* batch, CUstream stream);

/* All pointers are host pointers; copies in, runs, copies out, returns when
 * done.  kernelMs (may be NULL) receives the kernel's device time. */
VLRResult vlrbBsdfBatchHost(const VLRBBsdfBatch* batch, float* kernelMs);

#if defined(__cplusplus)
}
#endif

#endif /* VLRB_VLRB_H */
