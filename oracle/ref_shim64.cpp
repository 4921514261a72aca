// FP64 build of the reference's own spectral and BSDF code: the same sources
// as ref_shim.cpp (libVLR/shared, GPU_kernels/materials.cu), with every
// `float` they declare compiled as double, so the same BSDF arithmetic in
// the same order runs at 53-bit precision.  It is the FP64 oracle that the
// FP32 per-query results (the reference's own FP32 build and the CUDA batch
// kernel) are reported against.
//
// TEST INFRASTRUCTURE ONLY, built by oracle/build_ref.sh into
// oracle/_ref/libvlrref64.so (linked with -Bsymbolic, so its classes never
// bind to the FP32 library's of the same names).  The reference's float
// literals (0.5f) stay float constants and are widened exactly; its data
// tables (Meng grid, CIE functions) hold the same values as doubles.
//
// Exports (extern "C"):
//   vlrref64_init        -> initializeColorSystem in double
//   vlrref64_bsdf_batch  -> the batch of ref_bsdf_batch.inc, FP32 inputs
//                           widened exactly, FP64 outputs

// Every system and CUDA header the reference includes comes first, so the
// macro below changes only the reference's own declarations.
#include <algorithm>
#include <array>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <filesystem>
#include <fstream>
#include <functional>
#include <immintrin.h>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <random>
#include <set>
#include <sstream>
#include <stack>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>
#include <omp.h>
#include <cuda.h>
#include <vector_types.h>
#include <vector_functions.h>

typedef float vlrref_f32;
#define float double
// The reference checks the byte sizes of its shader-node descriptors, which
// hold floats (shared.h:685-694); the BSDF batch uses no shader node.
#define static_assert(...)

#include "shared/kernel_common.h"

#undef static_assert

// Mixed float/double arguments the reference's float literals create once
// its variables are double (materials.cu:58, 79, 1726-1953).
namespace vlr {
    inline double clamp(double x, vlrref_f32 a, vlrref_f32 b) { return clamp<double>(x, a, b); }
    inline double lerp(double a, double b, vlrref_f32 t) { return lerp<double>(a, b, t); }
    inline double lerp(vlrref_f32 a, double b, double t) { return lerp<double>(a, b, t); }
    inline double lerp(vlrref_f32 a, vlrref_f32 b, double t) { return lerp<double>(a, b, t); }
    inline double lerp(double a, vlrref_f32 b, double t) { return lerp<double>(a, b, t); }
    inline double max(double a, vlrref_f32 b) { return max<double>(a, b); }
}

void vlrprintf(const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    std::vfprintf(stderr, fmt, args);
    va_end(args);
}

namespace vlr::shared {
    PipelineLaunchParameters plp;
    constexpr bool usePathSpaceRegularization = false;

    inline float computeRegularizationFactor(float* cosEpsilon) {
        *cosEpsilon = 1.0f;
        return 1.0f;
    }

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
#include "shared/spectrum_base.cpp"
// spectrum_types.cpp holds the reference's own FP32 and FP64 tables of the
// Meng-Simon upsampling and the generic template definitions.
// oracle/build_ref.sh writes spectrum_types64.cpp into the mirror: the same
// file without its FP32 tables and FP32 explicit instantiations, which in
// this build would redefine the FP64 ones; the reference's FP64 tables then
// serve the double UpsampledSpectrum.
#include "shared/spectrum_types64.cpp"

using namespace vlr;
using namespace vlr::shared;

#include "ref_bsdf_batch.inc"

#undef float

extern "C" {

int vlrref64_init(void) {
    initializeColorSystem();
    return static_cast<int>(sizeof(UpsampledSpectrum));
}

void vlrref64_bsdf_batch(
    int64_t n, int numThreads,
    const float* wo, const uint32_t* mat, const float* rough, const float* ior,
    const float* rgb, const float* metallic, const float* u, const float* wl,
    double* value, double* pdf, double* wi, double* evalValue, double* evalPdf) {
    bsdfBatchQueries(n, numThreads, wo, mat, rough, ior, rgb, metallic, u, wl, value, pdf, wi, evalValue, evalPdf);
}

}
