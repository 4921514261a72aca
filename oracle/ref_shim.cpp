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
    // Material ids of the BSDF batch workload.
    enum : uint32_t {
        kMatte = 0, kSpecularBRDF = 1, kMicrofacetBRDF = 2,
        kMicrofacetBSDF = 3, kLambertianBSDF = 4, kUE4 = 5, kSpecularBSDF = 6,
    };

    struct Packed {
        uint32_t w[3];
    };

    inline UpsampledSpectrum unpack(const uint32_t p[3]) {
        UpsampledSpectrum s;
        std::memcpy(&s, p, sizeof(UpsampledSpectrum));
        return s;
    }

    template <typename BSDFType>
    void runQuery(const BSDFType &bsdf, const BSDFQuery &query, const float u[3],
                  float* value4, float* pdf, float* wi3, float* evalValue4, float* evalPdf) {
        BSDFQueryResult result;
        result.dirPDF = 0.0f;
        result.dirLocal = Vector3D(0.0f, 0.0f, 0.0f);
        const float uDir[2] = { u[1], u[2] };
        SampledSpectrum fs = bsdf.sampleInternal(query, u[0], uDir, &result);
        if (!(result.dirPDF > 0.0f)) {
            for (int i = 0; i < 4; ++i) { value4[i] = 0.0f; evalValue4[i] = 0.0f; }
            *pdf = 0.0f; *evalPdf = 0.0f;
            wi3[0] = wi3[1] = wi3[2] = 0.0f;
            return;
        }
        for (int i = 0; i < 4; ++i) value4[i] = fs[i];
        *pdf = result.dirPDF;
        wi3[0] = result.dirLocal.x; wi3[1] = result.dirLocal.y; wi3[2] = result.dirLocal.z;
        SampledSpectrum ev = bsdf.evaluateInternal(query, result.dirLocal);
        for (int i = 0; i < 4; ++i) evalValue4[i] = ev[i];
        *evalPdf = bsdf.evaluatePDFInternal(query, result.dirLocal);
    }
}

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
    if (numThreads > 0)
        omp_set_num_threads(numThreads);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        float wlPDF;
        WavelengthSamples wls = WavelengthSamples::createWithEqualOffsets(wl[2 * i + 0], wl[2 * i + 1], &wlPDF);
        const Vector3D dirLocal(wo[3 * i + 0], wo[3 * i + 1], wo[3 * i + 2]);
        BSDFQuery query(dirLocal, Normal3D(0.0f, 0.0f, 1.0f), TransportMode::Radiance,
                        DirectionType::All(), wls);
        const float* ui = u + 3 * i;
        float* v4 = value + 4 * i;
        float* p1 = pdf + i;
        float* w3 = wi + 3 * i;
        float* e4 = evalValue + 4 * i;
        float* ep = evalPdf + i;

        UpsampledSpectrum albedoSp(SpectrumType::Reflectance, ColorSpace::Rec709_D65,
                                   rgb[3 * i + 0], rgb[3 * i + 1], rgb[3 * i + 2]);
        UpsampledSpectrum iorSp(SpectrumType::IndexOfRefraction, ColorSpace::Rec709_D65,
                                ior[i], ior[i], ior[i]);
        UpsampledSpectrum oneSp(SpectrumType::IndexOfRefraction, ColorSpace::Rec709_D65, 1.0f, 1.0f, 1.0f);
        UpsampledSpectrum zeroSp(SpectrumType::IndexOfRefraction, ColorSpace::Rec709_D65, 0.0f, 0.0f, 0.0f);
        const float rx = rough[2 * i + 0], ry = rough[2 * i + 1];
        const float alphaX = std::fmax(0.001f, rx * rx);
        const float alphaY = std::fmax(0.001f, ry * ry);

        switch (mat[i]) {
        case kMatte: {
            MatteBRDF b(albedoSp.evaluate(wls), 0.0f);
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        case kSpecularBRDF: {
            SpecularBRDF b(albedoSp.evaluate(wls), iorSp.evaluate(wls), zeroSp.evaluate(wls));
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        case kMicrofacetBRDF: {
            MicrofacetBRDF b(iorSp.evaluate(wls), zeroSp.evaluate(wls), alphaX, alphaY, 0.0f);
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        case kMicrofacetBSDF: {
            MicrofacetBSDF b(albedoSp.evaluate(wls), oneSp.evaluate(wls), iorSp.evaluate(wls),
                             alphaX, alphaY, 0.0f);
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        case kLambertianBSDF: {
            LambertianBSDF b(albedoSp.evaluate(wls), 0.04f);
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        case kSpecularBSDF: {
            // SpecularScatteringSurfaceMaterial_setupBSDF (materials.cu:1046-1058):
            // coefficient, exterior IOR 1, interior IOR, dispersive unless a
            // single wavelength is selected
            SpecularBSDF b(albedoSp.evaluate(wls), oneSp.evaluate(wls), iorSp.evaluate(wls),
                           !wls.singleIsSelected());
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        default: {
            SampledSpectrum baseColor = albedoSp.evaluate(wls);
            const float roughness = std::fmax(0.01f, rx);
            const float m = metallic[i];
            const float specular = 0.5f;
            SampledSpectrum diffuseColor = baseColor * (1 - m);
            SampledSpectrum specularF0Color = lerp(0.08f * specular * SampledSpectrum::One(), baseColor, m);
            DiffuseAndSpecularBRDF b(diffuseColor, specularF0Color, roughness);
            runQuery(b, query, ui, v4, p1, w3, e4, ep);
            break;
        }
        }
    }
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
