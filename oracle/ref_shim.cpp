// Host build of the reference's own spectral + BSDF code, exposed as a small
// C ABI so tests and the CPU baseline can call it.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  This translation unit is compiled by
// oracle/build_ref.sh against a mirror of the reference tree; the reference
// sources are never copied into this repository.  It supplies the few
// device-only helpers that libVLR/shared/kernel_common.h declares only under
// nvcc (kernel_common.h:674-753), then includes libVLR/GPU_kernels/materials.cu
// verbatim so the BSDF classes (materials.cu:13-1994) are the reference's.
//
// Exports (all extern "C"):
//   vlrref_init                 -> vlr::initializeColorSystem (spectrum_base.cpp:39-49)
//   vlrref_upsample             -> UpsampledSpectrum ctor (spectrum_types.cpp:162-228)
//   vlrref_eval_upsampled       -> UpsampledSpectrum::evaluate (spectrum_types.cpp:273-322)
//   vlrref_wavelengths          -> WavelengthSamples::createWithEqualOffsets (spectrum_types.h:55-65)
//   vlrref_bsdf_batch           -> one sample/eval/pdf triple per query (materials.cu classes)
//   vlrref_tables               -> raw pointers to the Meng tables and CMF bins
//   vlrref_seed_states          -> std::mt19937_64 per-pixel RNG seeds (context.cpp:1176-1190)
#include "shared/kernel_common.h"

#include <omp.h>
#include <cstdarg>

// Host logging hook the reference declares in include/vlr/common.h.
void vlrprintf(const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    std::vfprintf(stderr, fmt, args);
    va_end(args);
}

namespace vlr::shared {
    PipelineLaunchParameters plp;

    // Path-space regularisation is compiled out in the reference
    // (kernel_common.h:744); keep the same constant.
    constexpr bool usePathSpaceRegularization = false;

    inline float computeRegularizationFactor(float* cosEpsilon) {
        *cosEpsilon = 1.0f;
        return 1.0f;
    }

    // Immediate-value node evaluation: the shader-node graph is not used by
    // any workload, so every plug is invalid and the immediate value wins
    // (kernel_common.h:674-676, 717-719 fall through to the default).
    template <typename T>
    inline T calcNode(ShaderNodePlug, const T &defaultValue,
                      const SurfacePoint &, const WavelengthSamples &) {
        return defaultValue;
    }

    inline SampledSpectrum calcNode(ShaderNodePlug, const TripletSpectrum &defaultValue,
                                    const SurfacePoint &, const WavelengthSamples &wls) {
        return defaultValue.evaluate(wls);
    }
}


#include "GPU_kernels/materials.cu"

using namespace vlr;
using namespace vlr::shared;

namespace {
    inline UpsampledSpectrum unpack(const uint32_t p[3]) {
        UpsampledSpectrum s;
        std::memcpy(&s, p, sizeof(UpsampledSpectrum));
        return s;
    }
}

#include "ref_bsdf_batch.inc"

extern "C" {

int vlrref_init(void) {
    initializeColorSystem();
    return static_cast<int>(sizeof(UpsampledSpectrum));
}

void vlrref_upsample(int spType, int colorSpace, float e0, float e1, float e2, uint32_t out[3]) {
    UpsampledSpectrum s(static_cast<SpectrumType>(spType), static_cast<ColorSpace>(colorSpace), e0, e1, e2);
    std::memcpy(out, &s, sizeof(UpsampledSpectrum));
}

void vlrref_eval_upsampled(const uint32_t packed[3], const float lambdas[4], float out[4]) {
    UpsampledSpectrum s = unpack(packed);
    WavelengthSamples wls(lambdas);
    SampledSpectrum v = s.evaluate(wls);
    for (int i = 0; i < 4; ++i) out[i] = v[i];
}

void vlrref_wavelengths(float offset, float uSel, float lambdas[4], uint32_t* selected, float* pdf) {
    WavelengthSamples wls = WavelengthSamples::createWithEqualOffsets(offset, uSel, pdf);
    for (int i = 0; i < 4; ++i) lambdas[i] = wls[i];
    *selected = wls.selectedLambdaIndex();
}

// One query = sample + evaluate + evaluatePDF at the sampled direction of the
// BSDF chosen by mat[i], built the way the reference's setupBSDF callables
// build it from immediate values (materials.cu:653-661, 776-787, 1220-1240,
// 1516-1536, 1674-1684, 1959-1978).  Geometric normal = shading normal.
void vlrref_bsdf_batch(
    int64_t n, int numThreads,
    const float* wo, const uint32_t* mat, const float* rough, const float* ior,
    const float* rgb, const float* metallic, const float* u, const float* wl,
    float* value, float* pdf, float* wi, float* evalValue, float* evalPdf) {
    bsdfBatchQueries(n, numThreads, wo, mat, rough, ior, rgb, metallic, u, wl, value, pdf, wi, evalValue, evalPdf);
}

// n outputs of std::mt19937_64 seeded with `seed`: the reference's per-pixel
// PCG32 seeding (context.cpp:618-626, 1176-1190).
void vlrref_seed_states(uint64_t seed, uint64_t n, uint64_t* out) {
    std::mt19937_64 gen(seed);
    for (uint64_t i = 0; i < n; ++i) out[i] = gen();
}

// Raw table access so the extracted tables can be cross-checked against the
// ones compiled into the reference objects.
void vlrref_tables(const void** grid, const void** points, const float** cmf16, float* integralCMF) {
    *grid = UpsampledSpectrum::spectrum_grid;
    *points = UpsampledSpectrum::spectrum_data_points;
    static float bins[48];
    for (int i = 0; i < 16; ++i) {
        bins[i] = DiscretizedSpectrum::xbar[i];
        bins[16 + i] = DiscretizedSpectrum::ybar[i];
        bins[32 + i] = DiscretizedSpectrum::zbar[i];
    }
    *cmf16 = bins;
    *integralCMF = DiscretizedSpectrum::integralCMF;
}

}

#include "ref_pt.inc"
#include "ref_bpt.inc"
