// Device and host copies of the spectral data tables (Meng-Simon grid and
// points, CIE 1931 colour-matching functions, Rec.709 matrices) and the
// 16-stratum CMF integrals that the film conversion uses.
#pragma once

#include "core.cuh"

namespace vlrb {

// Host-side views; valid for the lifetime of the process.
MengTables hostMengTables();
const ColorMatrices &hostColorMatrices();

// CMF integrated over the 16 storage strata plus the Y integral
// (DiscretizedSpectrumTemplate::initialize, spectrum_types.cpp:634-680).
struct CmfStrata {
    float xbar[kNumStrata], ybar[kNumStrata], zbar[kNumStrata];
    float integralCMF;
};
const CmfStrata &hostCmfStrata();

// Raw 471-sample CIE 1931 2-degree tables, 360-830 nm at 1 nm.
const float* hostCie1931(int component);

#if defined(__CUDACC__)
// Device copies live in module globals; these return their addresses for the
// current device (resolved once per device).
MengTables deviceMengTables();
const ColorMatrices* deviceColorMatrices();
#endif

} // namespace vlrb
