// Host-side spectral utility entry points (include/vlrb.h).
#include "../../include/vlrb.h"
#include "tables.cuh"

#include <cstring>

using namespace vlrb;

extern "C" VLRResult vlrbUpsampleSpectrum(uint32_t spectrumType, uint32_t colorSpace, float e0, float e1, float e2,
                                          uint32_t packed[3]) {
    if (!packed || spectrumType > 3 || colorSpace > 3) return VLRResult_InvalidArgument;
    UpSpec s = mengUpsample(hostMengTables(), hostColorMatrices(), static_cast<SpType>(spectrumType),
                            static_cast<ColorSp>(colorSpace), e0, e1, e2);
    static_assert(sizeof(UpSpec) == 12, "packed spectrum is 12 bytes");
    std::memcpy(packed, &s, 12);
    return VLRResult_NoError;
}

extern "C" VLRResult vlrbEvaluateSpectrum(const uint32_t packed[3], const float lambdas[4], float values[4]) {
    if (!packed || !lambdas || !values) return VLRResult_InvalidArgument;
    UpSpec s;
    std::memcpy(&s, packed, 12);
    const uint32_t b[4] = { s.adj & 0xFF, (s.adj >> 8) & 0xFF, (s.adj >> 16) & 0xFF, (s.adj >> 24) & 0xFF };
    if (b[0] != 0xFF && (b[0] >= 186 || b[1] >= 186 || b[2] >= 186 || (b[3] != 0xFF && b[3] >= 186)))
        return VLRResult_InvalidArgument;
    WLS w;
    for (int i = 0; i < 4; ++i) w.lambda[i] = lambdas[i];
    w.selected = 0;
    w.single = 0;
    S4 v = mengEvaluate(hostMengTables(), s, w);
    for (int i = 0; i < 4; ++i) values[i] = v[i];
    return VLRResult_NoError;
}

extern "C" VLRResult vlrbEvaluateSpectrumTabulated(const uint32_t packed[3], const float lambdas[4], float values[4]) {
    if (!packed || !lambdas || !values) return VLRResult_InvalidArgument;
    UpSpec s;
    std::memcpy(&s, packed, 12);
    const uint32_t b[4] = { s.adj & 0xFF, (s.adj >> 8) & 0xFF, (s.adj >> 16) & 0xFF, (s.adj >> 24) & 0xFF };
    if (b[0] != 0xFF && (b[0] >= 186 || b[1] >= 186 || b[2] >= 186 || (b[3] != 0xFF && b[3] >= 186)))
        return VLRResult_InvalidArgument;
    float tab[kMengSamples];
    mengBlend(hostMengTables(), s, tab);
    WLS w;
    for (int i = 0; i < 4; ++i) w.lambda[i] = lambdas[i];
    w.selected = 0;
    w.single = 0;
    S4 v = blendedEvaluate(tab, w);
    for (int i = 0; i < 4; ++i) values[i] = v[i];
    return VLRResult_NoError;
}

extern "C" VLRResult vlrbCmfStrata(float xyz[48], float* integralCMF) {
    if (!xyz || !integralCMF) return VLRResult_InvalidArgument;
    const CmfStrata &c = hostCmfStrata();
    for (uint32_t i = 0; i < kNumStrata; ++i) {
        xyz[i] = c.xbar[i];
        xyz[16 + i] = c.ybar[i];
        xyz[32 + i] = c.zbar[i];
    }
    *integralCMF = c.integralCMF;
    return VLRResult_NoError;
}
