// Spectral data tables: compiled in from the generated include file and
// mirrored into device globals.
#include "tables.cuh"
#include "generated/spectral_tables.inc"

#include <cuda_runtime.h>
#include <mutex>
#include <stdexcept>
#include <string>

namespace vlrb {

__device__ uint8_t g_mengGrid[168 * 8];
__device__ float g_mengPoints[186 * 99];
__device__ ColorMatrices g_colorMatrices;

namespace {

struct HostTables {
    uint8_t grid[168 * 8];
    float points[186 * 99];
    ColorMatrices mats;
    CmfStrata strata;
};

// Integrate the 1 nm CMF samples over 16 equal strata of [360, 830] with the
// trapezoid rule, splitting the sample interval that straddles a stratum
// boundary (DiscretizedSpectrumTemplate::initialize, spectrum_types.cpp:634-680).
void integrateStrata(CmfStrata* s) {
    const float* cmf[3] = { tables::kCIE1931_xbar, tables::kCIE1931_ybar, tables::kCIE1931_zbar };
    float* out[3] = { s->xbar, s->ybar, s->zbar };
    const uint32_t numSamples = 471;
    uint32_t bin = 0;
    float nextP = static_cast<float>(bin + 1) / kNumStrata;
    float sum[3] = { 0, 0, 0 };
    float prev[3] = { cmf[0][0], cmf[1][0], cmf[2][0] };
    const float interval = 1;
    for (uint32_t i = 1; i < numSamples; ++i) {
        float curP = static_cast<float>(i) / (numSamples - 1);
        float width = interval;
        float cur[3] = { cmf[0][i], cmf[1][i], cmf[2][i] };
        if (curP >= nextP) {
            width = (curP - nextP) * (kWavelengthHigh - kWavelengthLow);
            float t = 1 - width / interval;
            for (int c = 0; c < 3; ++c) {
                float in = prev[c] * (1 - t) + cur[c] * t;
                sum[c] += (prev[c] + in) * (interval - width) * 0.5f;
                out[c][bin] = sum[c];
                sum[c] = 0;
                prev[c] = in;
            }
            ++bin;
            nextP = static_cast<float>(bin + 1) / kNumStrata;
        }
        for (int c = 0; c < 3; ++c) {
            sum[c] += (prev[c] + cur[c]) * width * 0.5f;
            prev[c] = cur[c];
        }
    }
    s->integralCMF = 0.0f;
    for (uint32_t i = 0; i < kNumStrata; ++i)
        s->integralCMF += s->ybar[i];
}

HostTables &hostTables() {
    static HostTables* t = [] {
        auto* h = new HostTables;
        for (int c = 0; c < 168; ++c)
            for (int k = 0; k < 8; ++k)
                h->grid[8 * c + k] = tables::kMengGrid[c][k];
        for (int p = 0; p < 186; ++p)
            for (int k = 0; k < 99; ++k)
                h->points[99 * p + k] = tables::kMengPoints[p][k];
        for (int k = 0; k < 9; ++k) {
            h->mats.rec709D65ToXYZ[k] = tables::k_mat_Rec709_D65_to_XYZ[k];
            h->mats.xyzToRec709D65[k] = tables::k_mat_XYZ_to_Rec709_D65[k];
            h->mats.rec709EToXYZ[k] = tables::k_mat_Rec709_E_to_XYZ[k];
            h->mats.xyzToRec709E[k] = tables::k_mat_XYZ_to_Rec709_E[k];
        }
        integrateStrata(&h->strata);
        return h;
    }();
    return *t;
}

struct DeviceSlot {
    bool ready = false;
    MengTables tables{};
    const ColorMatrices* mats = nullptr;
};

std::mutex g_devMutex;
DeviceSlot g_devSlots[64];

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

} // namespace

MengTables hostMengTables() {
    HostTables &h = hostTables();
    return MengTables{ h.grid, h.points };
}

const ColorMatrices &hostColorMatrices() { return hostTables().mats; }
const CmfStrata &hostCmfStrata() { return hostTables().strata; }

const float* hostCie1931(int component) {
    switch (component) {
    case 0: return tables::kCIE1931_xbar;
    case 1: return tables::kCIE1931_ybar;
    default: return tables::kCIE1931_zbar;
    }
}

// The device globals are filled once per device with synchronous copies.
static DeviceSlot &deviceSlot() {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        throw std::runtime_error("device index out of range");
    std::lock_guard<std::mutex> lock(g_devMutex);
    DeviceSlot &s = g_devSlots[dev];
    if (!s.ready) {
        HostTables &h = hostTables();
        check(cudaMemcpyToSymbol(g_mengGrid, h.grid, sizeof(h.grid)), "upload Meng grid");
        check(cudaMemcpyToSymbol(g_mengPoints, h.points, sizeof(h.points)), "upload Meng points");
        check(cudaMemcpyToSymbol(g_colorMatrices, &h.mats, sizeof(h.mats)), "upload colour matrices");
        void* pg = nullptr;
        void* pp = nullptr;
        void* pm = nullptr;
        check(cudaGetSymbolAddress(&pg, g_mengGrid), "grid address");
        check(cudaGetSymbolAddress(&pp, g_mengPoints), "points address");
        check(cudaGetSymbolAddress(&pm, g_colorMatrices), "matrix address");
        s.tables = MengTables{ static_cast<const uint8_t*>(pg), static_cast<const float*>(pp) };
        s.mats = static_cast<const ColorMatrices*>(pm);
        s.ready = true;
    }
    return s;
}

MengTables deviceMengTables() { return deviceSlot().tables; }
const ColorMatrices* deviceColorMatrices() { return deviceSlot().mats; }

} // namespace vlrb
