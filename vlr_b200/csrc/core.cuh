// Core light-transport math shared by every kernel in libvlr_b200:
// vectors, 4-wavelength spectra, PCG32, sample warps, Meng-Simon RGB->spectrum
// upsampling, Fresnel terms, the anisotropic GGX distribution, the BSDFs and
// the EDFs that the renderers use.
//
// Everything is FP32 and written so that the operation order of each formula
// matches the reference implementation it restates; the BSDF batch kernel is
// compiled without FMA contraction so its results can be compared with the
// reference's host build query by query.  Reference locations are cited per
// function (paths relative to the reference project root).
#pragma once

#include <cstdint>
#include <cmath>
#include <cfloat>
#include <cstring>

#if defined(__CUDACC__)
#  define VLRB_HD __host__ __device__ __forceinline__
#else
#  define VLRB_HD inline
#endif

namespace vlrb {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kWavelengthLow = 360.0f;   // spectrum_base.h:6
constexpr float kWavelengthHigh = 830.0f;  // spectrum_base.h:7
constexpr uint32_t kNumLambdas = 4;        // common_internal.h:26
constexpr uint32_t kNumStrata = 16;        // common_internal.h:27

template <typename T> VLRB_HD T vmin(T a, T b) { return a < b ? a : b; }
template <typename T> VLRB_HD T vmax(T a, T b) { return a > b ? a : b; }
template <typename T> VLRB_HD T vclamp(T v, T lo, T hi) { return vmin(vmax(v, lo), hi); }
VLRB_HD float sq(float x) { return x * x; }
VLRB_HD float cube(float x) { return x * x * x; }
VLRB_HD float quint(float x) { return x * x * x * x * x; }
VLRB_HD float lerpf(float a, float b, float t) { return (1 - t) * a + t * b; }

// Single-precision sine and cosine.  Evaluated in double and rounded once so
// the result is the correctly rounded float on host and device alike, which
// is what the reference's host build gets from the C library's sinf/cosf.
VLRB_HD void fsincos(float a, float* s, float* c) {
    double sd, cd;
#if defined(__CUDA_ARCH__)
    sincos(static_cast<double>(a), &sd, &cd);
#else
    sd = std::sin(static_cast<double>(a));
    cd = std::cos(static_cast<double>(a));
#endif
    *s = static_cast<float>(sd);
    *c = static_cast<float>(cd);
}

// ---------------------------------------------------------------- vectors
struct V3 {
    float x, y, z;
    VLRB_HD V3() {}
    VLRB_HD constexpr V3(float a, float b, float c) : x(a), y(b), z(c) {}
    VLRB_HD explicit constexpr V3(float a) : x(a), y(a), z(a) {}
    VLRB_HD V3 operator-() const { return V3(-x, -y, -z); }
    VLRB_HD V3 operator+(const V3 &o) const { return V3(x + o.x, y + o.y, z + o.z); }
    VLRB_HD V3 operator-(const V3 &o) const { return V3(x - o.x, y - o.y, z - o.z); }
    VLRB_HD V3 operator*(float s) const { return V3(x * s, y * s, z * s); }
    VLRB_HD V3 operator/(float s) const { float r = 1 / s; return V3(x * r, y * r, z * r); }
    VLRB_HD V3 &operator+=(const V3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    VLRB_HD V3 &operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
    VLRB_HD V3 &operator/=(float s) { float r = 1 / s; x *= r; y *= r; z *= r; return *this; }
    VLRB_HD float sqLength() const { return x * x + y * y + z * z; }
    VLRB_HD float length() const { return std::sqrt(x * x + y * y + z * z); }
    VLRB_HD bool allFinite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
};
VLRB_HD V3 operator*(float s, const V3 &v) { return V3(s * v.x, s * v.y, s * v.z); }
VLRB_HD float dot(const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VLRB_HD float absDot(const V3 &a, const V3 &b) { return std::fabs(a.x * b.x + a.y * b.y + a.z * b.z); }
VLRB_HD V3 cross(const V3 &a, const V3 &b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
VLRB_HD V3 normalize(const V3 &v) { float l = v.length(); return v / l; }
// include/vlr/basic_types.h:142
VLRB_HD V3 halfVector(const V3 &a, const V3 &b) { return normalize(a + b); }
VLRB_HD V3 vmin3(const V3 &a, const V3 &b) { return V3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
VLRB_HD V3 vmax3(const V3 &a, const V3 &b) { return V3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

// Duff et al. 2017 orthonormal basis (include/vlr/basic_types.h:58-64).
VLRB_HD void makeBasis(const V3 &n, V3* vx, V3* vy) {
    float sign = n.z >= 0 ? 1.0f : -1.0f;
    const float a = -1 / (sign + n.z);
    const float b = n.x * n.y * a;
    *vx = V3(1 + sign * n.x * n.x * a, sign * b, -sign * n.x);
    *vy = V3(b, sign + n.y * n.y * a, -n.y);
}

// Shading frame (shared/kernel_common.h:136-160).
struct Frame {
    V3 x, y, z;
    VLRB_HD Frame() {}
    VLRB_HD Frame(const V3 &t, const V3 &n) : x(t), y(cross(n, t)), z(n) {}
    VLRB_HD Frame(const V3 &t, const V3 &b, const V3 &n) : x(t), y(b), z(n) {}
    VLRB_HD V3 toLocal(const V3 &v) const { return V3(dot(x, v), dot(y, v), dot(z, v)); }
    VLRB_HD V3 fromLocal(const V3 &v) const {
        return V3(dot(V3(x.x, y.x, z.x), v), dot(V3(x.y, y.y, z.y), v), dot(V3(x.z, y.z, z.z), v));
    }
};

// ---------------------------------------------------------------- spectra
// Four hero-wavelength samples (shared/spectrum_types.h:6-70).
struct WLS {
    float lambda[kNumLambdas];
    uint32_t selected;     // hero index
    uint32_t single;       // 1 once a dispersive event has picked the hero only

    // createWithEqualOffsets (spectrum_types.h:55-65).
    VLRB_HD static WLS equalOffsets(float offset, float uLambda, float* pdf) {
        WLS w;
        for (uint32_t i = 0; i < kNumLambdas; ++i)
            w.lambda[i] = kWavelengthLow + (kWavelengthHigh - kWavelengthLow) * (i + offset) / kNumLambdas;
        float fsel = kNumLambdas * uLambda;
        uint32_t sel = static_cast<uint32_t>(static_cast<uint16_t>(fsel));
        w.selected = sel < kNumLambdas - 1 ? sel : kNumLambdas - 1;
        w.single = 0;
        *pdf = kNumLambdas / (kWavelengthHigh - kWavelengthLow);
        return w;
    }
};

// SampledSpectrumTemplate<float, 4> (spectrum_types.h:72-271).
struct S4 {
    float v[kNumLambdas];
    VLRB_HD S4() {}
    VLRB_HD explicit S4(float a) { for (int i = 0; i < 4; ++i) v[i] = a; }
    VLRB_HD static S4 zero() { return S4(0.0f); }
    VLRB_HD static S4 one() { return S4(1.0f); }
    VLRB_HD float &operator[](uint32_t i) { return v[i]; }
    VLRB_HD float operator[](uint32_t i) const { return v[i]; }
    VLRB_HD S4 operator+(const S4 &o) const { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = v[i] + o.v[i]; return r; }
    VLRB_HD S4 operator-(const S4 &o) const { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = v[i] - o.v[i]; return r; }
    VLRB_HD S4 operator*(const S4 &o) const { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = v[i] * o.v[i]; return r; }
    VLRB_HD S4 operator/(const S4 &o) const { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = v[i] / o.v[i]; return r; }
    VLRB_HD S4 operator*(float s) const { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = v[i] * s; return r; }
    VLRB_HD S4 operator/(float s) const { float q = 1 / s; S4 r; for (int i = 0; i < 4; ++i) r.v[i] = v[i] * q; return r; }
    VLRB_HD S4 &operator+=(const S4 &o) { for (int i = 0; i < 4; ++i) v[i] += o.v[i]; return *this; }
    VLRB_HD S4 &operator*=(const S4 &o) { for (int i = 0; i < 4; ++i) v[i] *= o.v[i]; return *this; }
    VLRB_HD S4 &operator*=(float s) { for (int i = 0; i < 4; ++i) v[i] *= s; return *this; }
    VLRB_HD S4 &operator/=(float s) { float q = 1 / s; for (int i = 0; i < 4; ++i) v[i] *= q; return *this; }
    VLRB_HD bool isZero() const { return v[0] == 0 && v[1] == 0 && v[2] == 0 && v[3] == 0; }
    VLRB_HD bool hasNonZero() const { return !isZero(); }
    VLRB_HD bool allFinite() const {
        for (int i = 0; i < 4; ++i) if (!std::isfinite(v[i])) return false;
        return true;
    }
    // Hero-weighted importance (spectrum_types.h:250-264).
    VLRB_HD float importance(uint32_t sel) const {
        float sum = 0;
        for (int i = 0; i < 4; ++i) sum += v[i];
        const float primary = 0.9f;
        const float marginal = (1 - primary) / (kNumLambdas - 1);
        return sum * marginal + v[sel] * (primary - marginal);
    }
};
VLRB_HD S4 operator*(float s, const S4 &c) { S4 r; for (int i = 0; i < 4; ++i) r.v[i] = c.v[i] * s; return r; }
VLRB_HD S4 lerpS(const S4 &a, const S4 &b, float t) { return (1 - t) * a + t * b; }
VLRB_HD S4 sqS(const S4 &a) { return a * a; }

// ---------------------------------------------------------------- RNG
// PCG32 XSH-RR (shared/random_distributions.h:6-27).
struct PCG32 {
    uint64_t state;
    VLRB_HD uint32_t next() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + 1;
        uint32_t xorshifted = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = static_cast<uint32_t>(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((-static_cast<int32_t>(rot)) & 31));
    }
    VLRB_HD float uniform() {
        uint32_t bits = (next() >> 9) | 0x3f800000u;
        float f;
        memcpy(&f, &bits, 4);
        return f - 1.0f;
    }
};

// ---------------------------------------------------------------- warps
// shared/random_distributions.h:54-76
VLRB_HD void concentricDisk(float u0, float u1, float* dx, float* dy) {
    float r, theta;
    float sx = 2 * u0 - 1;
    float sy = 2 * u1 - 1;
    if (sx == 0 && sy == 0) { *dx = 0; *dy = 0; return; }
    if (sx >= -sy) {
        if (sx > sy) { r = sx; theta = sy / sx; }
        else { r = sy; theta = 2 - sx / sy; }
    }
    else {
        if (sx > sy) { r = -sy; theta = 6 + sx / sy; }
        else { r = -sx; theta = 4 + sy / sx; }
    }
    theta *= kPi / 4;
    // The reference's unqualified cos/sin resolve to the double-precision C
    // functions, so the angle is evaluated in double and rounded once.
    *dx = static_cast<float>(r * cos(static_cast<double>(theta)));
    *dy = static_cast<float>(r * sin(static_cast<double>(theta)));
}

// random_distributions.h:81-88
VLRB_HD V3 cosineHemisphere(float u0, float u1) {
    float x, y;
    concentricDisk(u0, u1, &x, &y);
    return V3(x, y, std::sqrt(fmaxf(0.0f, 1.0f - x * x - y * y)));
}

// Low-distortion square-to-triangle map (random_distributions.h:155-170).
VLRB_HD void uniformTriangle(float u0, float u1, float* b0, float* b1) {
    *b0 = 0.5f * u0;
    *b1 = 0.5f * u1;
    float offset = *b1 - *b0;
    if (offset > 0) *b1 += offset;
    else *b0 -= offset;
}

// random_distributions.h:31-50 (two-entry form used by the UE4-like BRDF).
VLRB_HD uint32_t sampleDiscrete2(const float w[2], float u, float* prob, float* sum, float* remapped) {
    float s = 0;
    s += w[0];
    s += w[1];
    *sum = s;
    float su = u * s;
    float cum = 0, base = 0;
    for (uint32_t i = 0; i < 2; ++i) {
        base = cum;
        cum += w[i];
        if (su < cum) {
            *prob = w[i] / s;
            *remapped = (su - base) / w[i];
            return i;
        }
    }
    *prob = w[0] / s;
    return 0;
}

// ---------------------------------------------------------------- direction flags
// shared/kernel_common.h:263-310
namespace dir {
constexpr uint32_t LowFreq = 1u << 0, HighFreq = 1u << 1, Delta0D = 1u << 2, Delta1D = 1u << 3;
constexpr uint32_t NonDelta = LowFreq | HighFreq, Delta = Delta0D | Delta1D, AllFreq = NonDelta | Delta;
constexpr uint32_t Reflection = 1u << 4, Transmission = 1u << 5, Emission = Reflection, Acquisition = Reflection;
constexpr uint32_t WholeSphere = Reflection | Transmission, All = AllFreq | WholeSphere;
constexpr uint32_t Dispersive = 1u << 6;
VLRB_HD bool matches(uint32_t type, uint32_t filter) {
    uint32_t r = type & filter;
    return (r & WholeSphere) && (r & AllFreq);
}
VLRB_HD bool isDelta(uint32_t t) { return (t & Delta) && !(t & NonDelta); }
VLRB_HD bool isReflection(uint32_t t) { return (t & Reflection) && !(t & Transmission); }
VLRB_HD bool isTransmission(uint32_t t) { return !(t & Reflection) && (t & Transmission); }
VLRB_HD bool isDispersive(uint32_t t) { return (t & Dispersive) != 0; }
}

// ---------------------------------------------------------------- Meng-Simon upsampling
// Tables: 12x14 grid cells of 8 bytes {inside, numPoints, idx[6]} and 186 data
// points of 99 floats {xystar[2], uv[2], spectrum[95]}.
struct ColorMatrices;
struct MengTables {
    const uint8_t* grid;
    const float* points;
    const float* blended;   // optional: per-material spectra on the 95-sample grid (mengBlend)
    // optional: Image2DTexture textures of material spectra (device only)
    const unsigned long long* textures;   // cudaTextureObject_t per texture
    const uint32_t* texSpType;            // per texture: SpType | ColorSp << 8 of its image
    const ColorMatrices* colorMats;
};
constexpr uint32_t kMengGridW = 12, kMengGridH = 14, kMengSamples = 95, kMengPointStride = 99;
constexpr uint32_t kMengNumPoints = 186;
constexpr float kMengEqualEnergy = 0.009355121400914532f; // spectrum_types.h:373-375

enum class SpType : uint32_t { Reflectance = 0, LightSource = 1, IOR = 2, NA = 3 };
enum class ColorSp : uint32_t { sRGB = 0, Rec709 = 1, XYZ = 2, xyY = 3 };

struct ColorMatrices {
    float rec709D65ToXYZ[9], xyzToRec709D65[9], rec709EToXYZ[9], xyzToRec709E[9];
};

// spectrum_base.h:45-51
VLRB_HD float sRGBDegamma(float v) {
    if (v <= 0.04045f) return v / 12.92f;
    return std::pow(static_cast<float>(v + 0.055f) / 1.055f, 2.4f);
}

// Column-major 3x3 transform (spectrum_base.h:131-136).
VLRB_HD void mulColMajor(const float m[9], const float s[3], float d[3]) {
    d[0] = m[0] * s[0] + m[3] * s[1] + m[6] * s[2];
    d[1] = m[1] * s[0] + m[4] * s[1] + m[7] * s[2];
    d[2] = m[2] * s[0] + m[5] * s[1] + m[8] * s[2];
}

// UpsampledSpectrum: 4 packed point indices (0xFF in the top byte marks a
// triangle), quantised weights s,t and a brightness scale (spectrum_types.h:304-314).
struct UpSpec {
    uint32_t adj;
    uint16_t s, t;
    float scale;
};

// computeAdjacents (spectrum_types.cpp:10-91): locate (u, v) in the grid and
// store either bilinear weights of an inner quad or barycentrics in the
// boundary triangle fan.
VLRB_HD void mengAdjacents(const MengTables &T, float u, float v, UpSpec* out) {
    u = vclamp<float>(u, 0.0f, static_cast<float>(kMengGridW));
    v = vclamp<float>(v, 0.0f, static_cast<float>(kMengGridH));
    int32_t ui = static_cast<int32_t>(u);
    int32_t vi = static_cast<int32_t>(v);
    const int32_t cell = ui + static_cast<int32_t>(kMengGridW) * vi;
    const uint8_t* c = T.grid + 8 * cell;
    const uint8_t inside = c[0];
    const uint8_t numPoints = c[1];
    const uint8_t* idx = c + 2;
    out->adj = 0xFFFFFFFFu;
    out->s = 0;
    out->t = 0;
    if (inside) {
        float s = u - ui;
        float t = v - vi;
        out->adj = (static_cast<uint32_t>(idx[3]) << 24) | (static_cast<uint32_t>(idx[2]) << 16) |
                   (static_cast<uint32_t>(idx[1]) << 8) | static_cast<uint32_t>(idx[0]);
        out->s = static_cast<uint16_t>(fmaxf(s * (65535 - 1), 0.0f));
        out->t = static_cast<uint16_t>(fmaxf(t * (65535 - 1), 0.0f));
        return;
    }
    const float* p0 = T.points + kMengPointStride * idx[0];
    const float ex = u - p0[2];
    const float ey = v - p0[3];
    const float* p1 = T.points + kMengPointStride * idx[1];
    float e0x = p1[2] - p0[2];
    float e0y = p1[3] - p0[3];
    float uu = e0x * ey - ex * e0y;
    for (int i = 1; i < numPoints; ++i) {
        uint32_t id = idx[i % (numPoints - 1) + 1];
        const float* pi = T.points + kMengPointStride * id;
        float e1x = pi[2] - p0[2];
        float e1y = pi[3] - p0[3];
        float vv = ex * e1y - e1x * ey;
        const float area = e0x * e1y - e1x * e0y;
        const float b0 = uu / area;
        const float b1 = vv / area;
        float b2 = 1.0f - b0 - b1;
        if (b0 < -1e-6f || b1 < -1e-6f || b2 < -1e-6f) {
            uu = -vv;
            e0x = e1x;
            e0y = e1y;
            continue;
        }
        out->adj = (0xFFu << 24) | (static_cast<uint32_t>(idx[0]) << 16) |
                   (static_cast<uint32_t>(idx[i]) << 8) | id;
        out->s = static_cast<uint16_t>(fmaxf(b0 * (65535 - 1), 0.0f));
        out->t = static_cast<uint16_t>(fmaxf(b1 * (65535 - 1), 0.0f));
        break;
    }
}

// RGB/XYZ/xyY -> UpSpec (spectrum_types.cpp:162-228).
VLRB_HD UpSpec mengUpsample(const MengTables &T, const ColorMatrices &M,
                            SpType spType, ColorSp space, float e0, float e1, float e2) {
    float xy[2];
    float brightness;
    if (space == ColorSp::sRGB) {
        e0 = sRGBDegamma(e0);
        e1 = sRGBDegamma(e1);
        e2 = sRGBDegamma(e2);
    }
    if (space == ColorSp::sRGB || space == ColorSp::Rec709) {
        float rgb[3] = { e0, e1, e2 };
        float xyz[3];
        mulColMajor(spType == SpType::LightSource ? M.rec709D65ToXYZ : M.rec709EToXYZ, rgb, xyz);
        e0 = xyz[0]; e1 = xyz[1]; e2 = xyz[2];
    }
    if (space != ColorSp::xyY) {
        float Y = e1;
        float b = e0 + e1 + e2;
        e0 = e0 / b;
        e1 = e1 / b;
        e2 = Y;
    }
    xy[0] = e0;
    xy[1] = e1;
    brightness = e2 / e1;
    if (e2 == 0) {
        xy[0] = 0.3333f;
        xy[1] = 0.3333f;
        brightness = 0;
    }
    UpSpec sp;
    sp.scale = brightness / kMengEqualEnergy;
    // xy_to_uv (spectrum_types.h:382-391)
    float u = 16.730260708356887f * xy[0] + 7.7801960340706f * xy[1] - 2.170152247475828f;
    float v = -7.530081094743006f * xy[0] + 16.192422314095225f * xy[1] + 1.1125529268825947f;
    mengAdjacents(T, u, v, &sp);
    return sp;
}

// evaluate (spectrum_types.cpp:273-322).
VLRB_HD S4 mengEvaluate(const MengTables &T, const UpSpec &sp, const WLS &wls) {
    uint32_t a[4] = { sp.adj & 0xFF, (sp.adj >> 8) & 0xFF, (sp.adj >> 16) & 0xFF, (sp.adj >> 24) & 0xFF };
    // No containing cell or triangle was found (chromaticity outside the
    // tabulated gamut): the reference leaves the spectrum undefined; here it
    // evaluates to zero instead of indexing past the table.
    if (a[0] == 0xFF) return S4(0.0f);
    float sf = static_cast<float>(sp.s) / (65535 - 1);
    float tf = static_cast<float>(sp.t) / (65535 - 1);
    int n;
    float w[4];
    if (a[3] != 0xFF) {
        w[0] = (1 - sf) * (1 - tf);
        w[1] = sf * (1 - tf);
        w[2] = (1 - sf) * tf;
        w[3] = sf * tf;
        n = 4;
    }
    else {
        w[0] = sf;
        w[1] = tf;
        w[2] = 1.0f - sf - tf;
        w[3] = 0.0f;
        n = 3;
    }
    S4 ret(0.0f);
    for (int i = 0; i < 4; ++i) {
        float p = (wls.lambda[i] - 360.0f) / (830.0f - 360.0f);
        p = vclamp<float>(p, 0.0f, 1.0f);
        float binF = p * (kMengSamples - 1);
        uint32_t bin = vmin<uint32_t>(static_cast<uint32_t>(binF), kMengSamples - 1);
        uint32_t binNext = vmin<uint32_t>(bin + 1, kMengSamples - 1);
        float t = binF - bin;
        for (int j = 0; j < n; ++j) {
            const float* spec = T.points + kMengPointStride * a[j] + 4;
#if defined(__CUDA_ARCH__)
            float s0 = __ldg(spec + bin), s1 = __ldg(spec + binNext);
#else
            float s0 = spec[bin], s1 = spec[binNext];
#endif
            ret.v[i] += w[j] * (s0 * (1 - t) + s1 * t);
        }
    }
    return ret * sp.scale;
}

// The spectrum an UpSpec evaluates to, tabulated on the table's 95-sample
// wavelength grid with the point weights and the scale applied.  For a
// spectrum that is the same at every hit (an immediate material colour) this
// is computed once per scene, and evaluating it at a wavelength is one
// linear interpolation (blendedEvaluate) instead of evaluate's 3-4 table
// points.  Equal to evaluate up to float rounding (the weighted sum is taken
// before the interpolation instead of after).
VLRB_HD void mengBlend(const MengTables &T, const UpSpec &sp, float* out) {
    uint32_t a[4] = { sp.adj & 0xFF, (sp.adj >> 8) & 0xFF, (sp.adj >> 16) & 0xFF, (sp.adj >> 24) & 0xFF };
    for (uint32_t b = 0; b < kMengSamples; ++b) out[b] = 0.0f;
    if (a[0] == 0xFF) return;
    for (int j = 0; j < 4; ++j)
        if (a[j] >= kMengNumPoints && !(j == 3 && a[j] == 0xFF)) return;   // not a table point: no spectrum
    float sf = static_cast<float>(sp.s) / (65535 - 1);
    float tf = static_cast<float>(sp.t) / (65535 - 1);
    int n;
    float w[4];
    if (a[3] != 0xFF) {
        w[0] = (1 - sf) * (1 - tf);
        w[1] = sf * (1 - tf);
        w[2] = (1 - sf) * tf;
        w[3] = sf * tf;
        n = 4;
    }
    else {
        w[0] = sf;
        w[1] = tf;
        w[2] = 1.0f - sf - tf;
        w[3] = 0.0f;
        n = 3;
    }
    for (uint32_t b = 0; b < kMengSamples; ++b) {
        float v = 0.0f;
        for (int j = 0; j < n; ++j) v += w[j] * T.points[kMengPointStride * a[j] + 4 + b];
        out[b] = v * sp.scale;
    }
}

VLRB_HD S4 blendedEvaluate(const float* tab, const WLS &wls) {
    S4 ret(0.0f);
    for (int i = 0; i < 4; ++i) {
        float p = (wls.lambda[i] - 360.0f) / (830.0f - 360.0f);
        p = vclamp<float>(p, 0.0f, 1.0f);
        float binF = p * (kMengSamples - 1);
        uint32_t bin = vmin<uint32_t>(static_cast<uint32_t>(binF), kMengSamples - 1);
        uint32_t binNext = vmin<uint32_t>(bin + 1, kMengSamples - 1);
        float t = binF - bin;
#if defined(__CUDA_ARCH__)
        const float s0 = __ldg(tab + bin), s1 = __ldg(tab + binNext);
#else
        const float s0 = tab[bin], s1 = tab[binNext];
#endif
        ret.v[i] = s0 * (1 - t) + s1 * t;
    }
    return ret;
}

// ---------------------------------------------------------------- Fresnel
// materials.cu:13-43
struct FresnelConductor {
    S4 eta, k;
    VLRB_HD S4 eval(float cosEnter) const {
        cosEnter = std::fabs(cosEnter);
        float c2 = cosEnter * cosEnter;
        S4 twoEtaCos = 2.0f * eta * cosEnter;
        S4 tmpF = eta * eta + k * k;
        S4 tmp = tmpF * c2;
        S4 one(1.0f);
        S4 rParl2 = (tmp - twoEtaCos + one) / (tmp + twoEtaCos + one);
        S4 c2s(c2);
        S4 rPerp2 = (tmpF - twoEtaCos + c2s) / (tmpF + twoEtaCos + c2s);
        return (rParl2 + rPerp2) / 2.0f;
    }
};

// materials.cu:96-103
VLRB_HD float fresnelDielectricF(float etaEnter, float etaExit, float cosEnter, float cosExit) {
    float rParl = ((etaExit * cosEnter) - (etaEnter * cosExit)) / ((etaExit * cosEnter) + (etaEnter * cosExit));
    float rPerp = ((etaEnter * cosEnter) - (etaExit * cosExit)) / ((etaEnter * cosEnter) + (etaExit * cosExit));
    return (rParl * rParl + rPerp * rPerp) / 2.0f;
}

// materials.cu:47-94
struct FresnelDielectric {
    S4 etaExt, etaInt;
    VLRB_HD S4 eval(float cosEnter) const {
        cosEnter = vclamp(cosEnter, -1.0f, 1.0f);
        bool entering = cosEnter > 0.0f;
        const S4 &eEnter = entering ? etaExt : etaInt;
        const S4 &eExit = entering ? etaInt : etaExt;
        S4 sinExit = eEnter / eExit * std::sqrt(fmaxf(0.0f, 1.0f - cosEnter * cosEnter));
        S4 ret(0.0f);
        cosEnter = std::fabs(cosEnter);
        for (int i = 0; i < 4; ++i) {
            if (sinExit[i] >= 1.0f) {
                ret[i] = 1.0f;
            }
            else {
                float cosExit = std::sqrt(fmaxf(0.0f, 1.0f - sinExit[i] * sinExit[i]));
                ret[i] = fresnelDielectricF(eEnter[i], eExit[i], cosEnter, cosExit);
            }
        }
        return ret;
    }
    VLRB_HD float eval1(float cosEnter, uint32_t wl) const {
        cosEnter = vclamp(cosEnter, -1.0f, 1.0f);
        bool entering = cosEnter > 0.0f;
        const float eEnter = entering ? etaExt[wl] : etaInt[wl];
        const float eExit = entering ? etaInt[wl] : etaExt[wl];
        float sinExit = eEnter / eExit * std::sqrt(fmaxf(0.0f, 1.0f - cosEnter * cosEnter));
        cosEnter = std::fabs(cosEnter);
        if (sinExit >= 1.0f) return 1.0f;
        float cosExit = std::sqrt(fmaxf(0.0f, 1.0f - sinExit * sinExit));
        return fresnelDielectricF(eEnter, eExit, cosEnter, cosExit);
    }
};

// materials.cu:107-129
VLRB_HD S4 fresnelSchlick(float F0, float cosEnter) {
    bool entering = cosEnter >= 0;
    float cosEval = cosEnter;
    if (!entering) {
        float sqrtF0 = std::sqrt(F0);
        float etaExit = (1 + sqrtF0) / (1 - sqrtF0);
        float invRelIOR = 1.0f / etaExit;
        float sinExit2 = invRelIOR * invRelIOR * fmaxf(0.0f, 1.0f - cosEnter * cosEnter);
        if (sinExit2 > 1.0f) return S4::one();
        cosEval = std::sqrt(1 - sinExit2);
    }
    return S4(F0 + (1.0f - F0) * quint(1 - cosEval));
}

// ---------------------------------------------------------------- GGX
// Anisotropic GGX with rotation and visible-normal sampling (materials.cu:133-228).
struct GGX {
    float ax, ay, cosR, sinR;
    VLRB_HD GGX(float alphaX, float alphaY, float rotation) : ax(alphaX), ay(alphaY) {
        fsincos(rotation, &sinR, &cosR);
    }
    VLRB_HD V3 rot(const V3 &m) const { return V3(cosR * m.x + sinR * m.y, -sinR * m.x + cosR * m.y, m.z); }
    VLRB_HD float D(const V3 &m) const {
        V3 mr = rot(m);
        if (mr.z <= 0) return 0.0f;
        float temp = sq(mr.x / ax) + sq(mr.y / ay) + sq(mr.z);
        return 1.0f / (kPi * ax * ay * sq(temp));
    }
    VLRB_HD float G1(const V3 &v, const V3 &m) const {
        V3 vr = rot(v);
        float a2t2 = (sq(vr.x * ax) + sq(vr.y * ay)) / sq(vr.z);
        float lambda = (-1 + std::sqrt(1 + a2t2)) / 2;
        float chi = (dot(v, m) / v.z) > 0 ? 1.0f : 0.0f;
        return chi / (1 + lambda);
    }
    VLRB_HD float G2HeightCorrelated(const V3 &v1, const V3 &v2, const V3 &m) const {
        V3 v1r = rot(v1);
        V3 v2r = rot(v2);
        float a1 = (sq(v1r.x * ax) + sq(v1r.y * ay)) / sq(v1r.z);
        float a2 = (sq(v2r.x * ax) + sq(v2r.y * ay)) / sq(v2r.z);
        float l1 = (-1 + std::sqrt(1 + a1)) / 2;
        float l2 = (-1 + std::sqrt(1 + a2)) / 2;
        float chi1 = (dot(v1, m) / v1.z) > 0 ? 1.0f : 0.0f;
        float chi2 = (dot(v2, m) / v2.z) > 0 ? 1.0f : 0.0f;
        return chi1 * chi2 / (1 + l1 + l2);
    }
    VLRB_HD float sample(const V3 &v, float u0, float u1, V3* m, float* normalPDF) const {
        V3 vr = rot(v);
        V3 sv = normalize(V3(ax * vr.x, ay * vr.y, vr.z));
        float distIn2D = std::sqrt(sv.x * sv.x + sv.y * sv.y);
        float recDist = 1.0f / distIn2D;
        V3 T1 = (sv.z < 0.9999f) ? V3(sv.y * recDist, -sv.x * recDist, 0) : V3(1, 0, 0);
        V3 T2 = V3(T1.y * sv.z, -T1.x * sv.z, distIn2D);
        float a = 1.0f / (1.0f + sv.z);
        float r = std::sqrt(u0);
        float phi = kPi * ((u1 < a) ? u1 / a : 1 + (u1 - a) / (1.0f - a));
        float sinPhi, cosPhi;
        fsincos(phi, &sinPhi, &cosPhi);
        float P1 = r * cosPhi;
        float P2 = r * sinPhi * ((u1 < a) ? 1.0f : sv.z);
        V3 mr = P1 * T1 + P2 * T2 + std::sqrt(1.0f - P1 * P1 - P2 * P2) * sv;
        mr = normalize(V3(ax * mr.x, ay * mr.y, mr.z));
        float d = D(mr);
        *normalPDF = G1(vr, mr) * absDot(vr, mr) * d / std::fabs(vr.z);
        *m = V3(cosR * mr.x - sinR * mr.y, sinR * mr.x + cosR * mr.y, mr.z);
        return d;
    }
    VLRB_HD float pdf(const V3 &v, const V3 &m) const {
        return G1(v, m) * absDot(v, m) * D(m) / std::fabs(v.z);
    }
};

// ---------------------------------------------------------------- BSDFs
// Material kinds; also the material-sorted queue keys of the renderers.
enum BsdfKind : uint32_t {
    kMatte = 0, kSpecularBRDF = 1, kMicrofacetBRDF = 2, kMicrofacetBSDF = 3,
    kLambertianBSDF = 4, kUE4 = 5, kSpecularBSDF = 6, kNullBSDF = 7, kNumBsdfKinds = 8
};

struct BsdfQuery {
    V3 dirLocal;        // outgoing direction in the shading frame
    uint32_t wlHint;    // hero wavelength index
    uint32_t filter;    // DirectionType filter
    uint32_t importanceMode;  // 0: radiance transport, 1: importance transport
};

struct BsdfSample {
    V3 dirLocal;
    float dirPDF;
    uint32_t sampledType;
};

struct BsdfRev {
    S4 value;
    float dirPDF;
};

// Bsdf::flags of a MicrofacetBSDF: evaluate the pdf of transmission out of
// the medium consistently with the value (see mfBsdfPDF).
constexpr uint32_t kBsdfConsistentPdf = 1u;

// All BSDF parameters in one flat record (largest member: MicrofacetBSDF).
struct Bsdf {
    uint32_t kind;
    S4 a, b, c;         // per-kind spectra
    float f0, f1, f2;   // per-kind scalars
    uint32_t flags;     // SpecularBSDF: dispersive; MicrofacetBSDF: kBsdfConsistentPdf
};

// MatteBRDF (materials.cu:584-651)
VLRB_HD S4 matteSample(const Bsdf &B, const BsdfQuery &q, float uc, float u0, float u1, BsdfSample* r, BsdfRev* rev) {
    (void)uc;
    r->dirLocal = cosineHemisphere(u0, u1);
    r->dirPDF = r->dirLocal.z / kPi;
    r->sampledType = dir::Reflection | dir::LowFreq;
    r->dirLocal.z *= q.dirLocal.z >= 0 ? 1 : -1;
    S4 fs = B.a / kPi;
    if (rev) { rev->value = fs; rev->dirPDF = std::fabs(q.dirLocal.z) / kPi; }
    return fs;
}
VLRB_HD S4 matteEval(const Bsdf &B, const BsdfQuery &q, const V3 &d, S4* revValue) {
    if (q.dirLocal.z * d.z <= 0.0f) { if (revValue) *revValue = S4::zero(); return S4::zero(); }
    S4 fs = B.a / kPi;
    if (revValue) *revValue = fs;
    return fs;
}
VLRB_HD float mattePDF(const Bsdf &, const BsdfQuery &q, const V3 &d, float* revPDF) {
    if (q.dirLocal.z * d.z <= 0.0f) { if (revPDF) *revPDF = 0.0f; return 0.0f; }
    if (revPDF) *revPDF = std::fabs(q.dirLocal.z) / kPi;
    return std::fabs(d.z) / kPi;
}

// SpecularBRDF, delta reflection off a conductor (materials.cu:667-774).
// B.a = coeffR, B.b = eta, B.c = k.
VLRB_HD S4 specBrdfSample(const Bsdf &B, const BsdfQuery &q, float, float, float, BsdfSample* r, BsdfRev* rev) {
    FresnelConductor fr{ B.b, B.c };
    r->dirLocal = V3(-q.dirLocal.x, -q.dirLocal.y, q.dirLocal.z);
    r->dirPDF = 1.0f;
    r->sampledType = dir::Reflection | dir::Delta0D;
    S4 ret = B.a * fr.eval(q.dirLocal.z) * (1.0f / std::fabs(q.dirLocal.z));
    if (rev) { rev->value = ret; rev->dirPDF = 1.0f; }
    return ret;
}

// SpecularBSDF, delta dielectric with hero-wavelength refraction
// (materials.cu:793-1044).  B.a = coeff, B.b = etaExt, B.c = etaInt.
VLRB_HD S4 specBsdfSample(const Bsdf &B, const BsdfQuery &q, float uc, float, float, BsdfSample* r, BsdfRev* rev) {
    if (rev) rev->dirPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    const S4 &eEnter = entering ? B.b : B.c;
    const S4 &eExit = entering ? B.c : B.b;
    FresnelDielectric fr{ eEnter, eExit };
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    S4 F = fr.eval(dirV.z);
    float reflectProb = F.importance(q.wlHint);
    if (dir::isReflection(q.filter)) reflectProb = 1.0f;
    if (dir::isTransmission(q.filter)) reflectProb = 0.0f;
    if (uc < reflectProb) {
        if (dirV.z == 0.0f) { r->dirPDF = 0.0f; return S4::zero(); }
        V3 dirL = V3(-dirV.x, -dirV.y, dirV.z);
        r->dirLocal = entering ? dirL : -dirL;
        r->dirPDF = reflectProb * 1.0f;
        r->sampledType = dir::Reflection | dir::Delta0D;
        S4 ret = B.a * F * (1.0f / std::fabs(dirV.z));
        if (rev) { rev->value = ret; rev->dirPDF = r->dirPDF; }
        return ret;
    }
    float sinEnter2 = 1.0f - dirV.z * dirV.z;
    float recRelIOR = eEnter[q.wlHint] / eExit[q.wlHint];
    float sinExit2 = recRelIOR * recRelIOR * sinEnter2;
    if (sinExit2 >= 1.0f) { r->dirPDF = 0.0f; return S4::zero(); }
    float cosExit = std::sqrt(fmaxf(0.0f, 1.0f - sinExit2));
    V3 dirL = V3(recRelIOR * -dirV.x, recRelIOR * -dirV.y, -cosExit);
    r->dirLocal = entering ? dirL : -dirL;
    r->dirPDF = (1.0f - reflectProb) * 1.0f;
    r->sampledType = dir::Transmission | dir::Delta0D | (B.flags ? dir::Dispersive : 0u);
    S4 ret = S4::zero();
    ret[q.wlHint] = B.a[q.wlHint] * (1.0f - F[q.wlHint]) * 1.0f;
    if (rev) {
        float revSqueeze = 1.0f;
        if (q.importanceMode) revSqueeze = sq(eExit[q.wlHint] / eEnter[q.wlHint]);
        S4 revRet = ret;
        revRet[q.wlHint] *= revSqueeze / std::fabs(q.dirLocal.z);
        rev->value = revRet;
        rev->dirPDF = revSqueeze * r->dirPDF;
    }
    float squeeze = 1.0f;
    if (!q.importanceMode) squeeze *= sq(eEnter[q.wlHint] / eExit[q.wlHint]);
    ret[q.wlHint] *= squeeze / std::fabs(cosExit);
    r->dirPDF *= squeeze;
    return ret;
}

// MicrofacetBRDF, anisotropic GGX conductor (materials.cu:1064-1218).
// B.b = eta, B.c = k, f0/f1/f2 = alphaX/alphaY/rotation.
VLRB_HD S4 mfBrdfSample(const Bsdf &B, const BsdfQuery &q, float, float u0, float u1, BsdfSample* r, BsdfRev* rev) {
    if (rev) rev->dirPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    FresnelConductor fr{ B.b, B.c };
    GGX ggx(B.f0, B.f1, B.f2);
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 m;
    float mPDF;
    float D = ggx.sample(dirV, u0, u1, &m, &mPDF);
    float dotHV = dot(dirV, m);
    if (dotHV <= 0) { r->dirPDF = 0.0f; return S4::zero(); }
    V3 dirL = 2 * dotHV * m - dirV;
    r->dirLocal = entering ? dirL : -dirL;
    if (dirL.z * dirV.z <= 0) { r->dirPDF = 0.0f; return S4::zero(); }
    float common = 1.0f / (4 * dotHV);
    r->dirPDF = common * mPDF;
    r->sampledType = dir::Reflection | dir::HighFreq;
    S4 F = fr.eval(dotHV);
    float G = ggx.G1(dirV, m) * ggx.G1(dirL, m);
    S4 fs = F * D * G / (4 * dirV.z * dirL.z);
    if (rev) { rev->value = fs; rev->dirPDF = common * ggx.pdf(dirL, m); }
    return fs;
}
VLRB_HD S4 mfBrdfEval(const Bsdf &B, const BsdfQuery &q, const V3 &d, S4* revValue) {
    bool entering = q.dirLocal.z >= 0.0f;
    FresnelConductor fr{ B.b, B.c };
    GGX ggx(B.f0, B.f1, B.f2);
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    float nvnl = dirL.z * dirV.z;
    if (nvnl <= 0) return S4::zero();
    V3 m = halfVector(dirV, dirL);
    float dotHV = dot(dirV, m);
    float D = ggx.D(m);
    S4 F = fr.eval(dotHV);
    float G = ggx.G1(dirV, m) * ggx.G1(dirL, m);
    S4 fs = F * D * G / (4 * nvnl);
    if (revValue) *revValue = fs;
    return fs;
}
VLRB_HD float mfBrdfPDF(const Bsdf &B, const BsdfQuery &q, const V3 &d, float* revPDF) {
    if (revPDF) *revPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    GGX ggx(B.f0, B.f1, B.f2);
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    float nvnl = dirL.z * dirV.z;
    if (nvnl <= 0.0f) return 0.0f;
    V3 m = halfVector(dirV, dirL);
    float dotHV = dot(dirV, m);
    if (dotHV <= 0) return 0.0f;
    float mPDF = ggx.pdf(dirV, m);
    float common = 1.0f / (4 * dotHV);
    if (revPDF) *revPDF = common * ggx.pdf(dirL, m);
    return common * mPDF;
}

// Per-wavelength transmission term of the GGX dielectric (materials.cu:1355-1370).
VLRB_HD S4 mfBsdfTransmission(const GGX &ggx, const FresnelDielectric &fr, const S4 &eEnter, const S4 &eExit,
                              const V3 &dirV, const V3 &dirL, bool entering) {
    S4 ret = S4::zero();
    for (int w = 0; w < 4; ++w) {
        V3 mw = normalize(-(eEnter[w] * dirV + eExit[w] * dirL) * (entering ? 1.0f : -1.0f));
        float dhv = dot(dirV, mw);
        float dhl = dot(dirL, mw);
        float Fw = fr.eval1(dhv, w);
        float Gw = ggx.G1(dirV, mw) * ggx.G1(dirL, mw);
        float Dw = ggx.D(mw);
        ret[w] = std::fabs(dhv * dhl) * (1 - Fw) * Gw * Dw / sq(eEnter[w] * dhv + eExit[w] * dhl);
    }
    return ret;
}

// MicrofacetBSDF, GGX dielectric (materials.cu:1246-1514).
// B.a = coeff, B.b = etaExt, B.c = etaInt, f0/f1/f2 = alphaX/alphaY/rotation.
VLRB_HD S4 mfBsdfSample(const Bsdf &B, const BsdfQuery &q, float uc, float u0, float u1, BsdfSample* r, BsdfRev* rev) {
    if (rev) rev->dirPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    const S4 &eEnter = entering ? B.b : B.c;
    const S4 &eExit = entering ? B.c : B.b;
    FresnelDielectric fr{ eEnter, eExit };
    GGX ggx(B.f0, B.f1, B.f2);
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 m;
    float mPDF;
    float D = ggx.sample(dirV, u0, u1, &m, &mPDF);
    float dotHV = dot(dirV, m);
    if (dotHV <= 0 || std::isnan(D)) { r->dirPDF = 0.0f; return S4::zero(); }
    S4 F = fr.eval(dotHV);
    float reflectProb = F.importance(q.wlHint);
    if (dir::isReflection(q.filter)) reflectProb = 1.0f;
    if (dir::isTransmission(q.filter)) reflectProb = 0.0f;
    if (uc < reflectProb) {
        V3 dirL = 2 * dotHV * m - dirV;
        r->dirLocal = entering ? dirL : -dirL;
        if (dirL.z * dirV.z <= 0) { r->dirPDF = 0.0f; return S4::zero(); }
        float common = reflectProb / (4 * dotHV);
        r->dirPDF = common * mPDF;
        r->sampledType = dir::Reflection | dir::HighFreq;
        float G = ggx.G1(dirV, m) * ggx.G1(dirL, m);
        S4 ret = B.a * F * D * G / (4 * dirV.z * dirL.z);
        if (rev) { rev->value = ret; rev->dirPDF = common * ggx.pdf(dirL, m); }
        return ret;
    }
    float recRelIOR = eEnter[q.wlHint] / eExit[q.wlHint];
    float innerRoot = 1 + recRelIOR * recRelIOR * (dotHV * dotHV - 1);
    if (innerRoot < 0) { r->dirPDF = 0.0f; return S4::zero(); }
    V3 dirL = (recRelIOR * dotHV - std::sqrt(innerRoot)) * m - recRelIOR * dirV;
    r->dirLocal = entering ? dirL : -dirL;
    if (dirL.z * dirV.z >= 0) { r->dirPDF = 0.0f; return S4::zero(); }
    float dotHL = dot(dirL, m);
    float common = (1 - reflectProb) / sq(eEnter[q.wlHint] * dotHV + eExit[q.wlHint] * dotHL);
    r->dirPDF = common * mPDF * sq(eExit[q.wlHint]) * std::fabs(dotHL);
    r->sampledType = dir::Transmission | dir::HighFreq;
    S4 ret = mfBsdfTransmission(ggx, fr, eEnter, eExit, dirV, dirL, entering);
    ret /= std::fabs(dirV.z * dirL.z);
    ret *= B.a;
    ret *= !q.importanceMode ? sqS(eEnter) : sqS(eExit);
    if (rev) {
        rev->value = ret;
        rev->dirPDF = common * ggx.pdf(dirL, m) * sq(eEnter[q.wlHint]) * std::fabs(dotHV);
    }
    return ret;
}
VLRB_HD S4 mfBsdfEval(const Bsdf &B, const BsdfQuery &q, const V3 &d, S4* revValue) {
    bool entering = q.dirLocal.z >= 0.0f;
    const S4 &eEnter = entering ? B.b : B.c;
    const S4 &eExit = entering ? B.c : B.b;
    FresnelDielectric fr{ eEnter, eExit };
    GGX ggx(B.f0, B.f1, B.f2);
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    float nvnl = dirL.z * dirV.z;
    if (nvnl > 0 && dir::matches(q.filter, dir::Reflection | dir::AllFreq)) {
        V3 m = halfVector(dirV, dirL);
        float dotHV = dot(dirV, m);
        float D = ggx.D(m);
        S4 F = fr.eval(dotHV);
        float G = ggx.G1(dirV, m) * ggx.G1(dirL, m);
        S4 ret = B.a * F * D * G / (4 * nvnl);
        if (revValue) *revValue = ret;
        return ret;
    }
    if (nvnl < 0 && dir::matches(q.filter, dir::Transmission | dir::AllFreq)) {
        S4 ret = mfBsdfTransmission(ggx, fr, eEnter, eExit, dirV, dirL, entering);
        ret /= std::fabs(nvnl);
        ret *= B.a;
        ret *= !q.importanceMode ? sqS(eEnter) : sqS(eExit);
        if (revValue) *revValue = ret;
        return ret;
    }
    return S4::zero();
}
// The reference's pdf builds the transmission half vector without the
// orientation flip its value function applies to paths leaving the medium
// (evaluatePDFInternal, materials.cu:1448-1513, vs evaluateInternal,
// :1385-1446), so every transmission out of the
// dielectric gets pdf 0: MIS then gives NEE full weight through the exit
// although BSDF sampling also reaches those paths (double counting), and the
// unsuppressed NEE values near the GGX peak are fireflies.  Kept by default
// for parity; Bsdf::flags & kBsdfConsistentPdf applies the same flip as the
// value function.
VLRB_HD float mfBsdfPDF(const Bsdf &B, const BsdfQuery &q, const V3 &d, float* revPDF) {
    if (revPDF) *revPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    const S4 &eEnter = entering ? B.b : B.c;
    const S4 &eExit = entering ? B.c : B.b;
    FresnelDielectric fr{ eEnter, eExit };
    GGX ggx(B.f0, B.f1, B.f2);
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    float nvnl = dirL.z * dirV.z;
    if (nvnl == 0) return 0.0f;
    V3 m;
    if (nvnl > 0) m = halfVector(dirV, dirL);
    else {
        m = normalize(-(eEnter[q.wlHint] * dirV + eExit[q.wlHint] * dirL));
        if ((B.flags & kBsdfConsistentPdf) && !entering) m = -m;
    }
    float dotHV = dot(dirV, m);
    if (dotHV <= 0) return 0.0f;
    float mPDF = ggx.pdf(dirV, m);
    S4 F = fr.eval(dotHV);
    float reflectProb = F.importance(q.wlHint);
    if (dir::isReflection(q.filter)) reflectProb = 1.0f;
    if (dir::isTransmission(q.filter)) reflectProb = 0.0f;
    if (nvnl > 0) {
        float common = reflectProb / (4 * dotHV);
        if (revPDF) *revPDF = common * ggx.pdf(dirL, m);
        return common * mPDF;
    }
    float dotHL = dot(dirL, m);
    float common = (1 - reflectProb) / sq(eEnter[q.wlHint] * dotHV + eExit[q.wlHint] * dotHL);
    if (revPDF) *revPDF = common * ggx.pdf(dirL, m) * sq(eEnter[q.wlHint]) * std::fabs(dotHV);
    return common * mPDF * sq(eExit[q.wlHint]) * std::fabs(dotHL);
}

// LambertianBSDF, Schlick-blended reflect/transmit cosine lobes
// (materials.cu:1542-1672).  B.a = coeff, f0 = F0.
VLRB_HD S4 lambSample(const Bsdf &B, const BsdfQuery &q, float uc, float u0, float u1, BsdfSample* r, BsdfRev* rev) {
    if (rev) rev->dirPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = cosineHemisphere(u0, u1);
    r->dirPDF = dirL.z / kPi;
    S4 F = fresnelSchlick(B.f0, q.dirLocal.z);
    float reflectProb = F.importance(q.wlHint);
    if (dir::isReflection(q.filter)) reflectProb = 1.0f;
    if (dir::isTransmission(q.filter)) reflectProb = 0.0f;
    if (uc < reflectProb) {
        r->dirLocal = entering ? dirL : -dirL;
        r->sampledType = dir::Reflection | dir::LowFreq;
        S4 ret = F * B.a / kPi;
        r->dirPDF *= reflectProb;
        if (rev) { rev->value = ret; rev->dirPDF = reflectProb * dirV.z / kPi; }
        return ret;
    }
    r->dirLocal = entering ? -dirL : dirL;
    r->sampledType = dir::Transmission | dir::LowFreq;
    S4 ret = (S4::one() - F) * B.a / kPi;
    r->dirPDF *= (1 - reflectProb);
    if (rev) { rev->value = ret; rev->dirPDF = (1 - reflectProb) * dirV.z / kPi; }
    return ret;
}
VLRB_HD S4 lambEval(const Bsdf &B, const BsdfQuery &q, const V3 &d, S4* revValue) {
    bool entering = q.dirLocal.z >= 0.0f;
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    S4 F = fresnelSchlick(B.f0, q.dirLocal.z);
    S4 ret = (dirV.z * dirL.z > 0.0f) ? F * B.a / kPi : (S4::one() - F) * B.a / kPi;
    if (revValue) *revValue = ret;
    return ret;
}
VLRB_HD float lambPDF(const Bsdf &B, const BsdfQuery &q, const V3 &d, float* revPDF) {
    if (revPDF) *revPDF = 0.0f;
    bool entering = q.dirLocal.z >= 0.0f;
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    S4 F = fresnelSchlick(B.f0, q.dirLocal.z);
    float reflectProb = F.importance(q.wlHint);
    if (dir::isReflection(q.filter)) reflectProb = 1.0f;
    if (dir::isTransmission(q.filter)) reflectProb = 0.0f;
    if (dirV.z * dirL.z > 0.0f) {
        if (revPDF) *revPDF = reflectProb * dirV.z / kPi;
        return reflectProb * dirL.z / kPi;
    }
    if (revPDF) *revPDF = (1 - reflectProb) * dirV.z / kPi;
    return (1 - reflectProb) * std::fabs(dirL.z) / kPi;
}

// UE4-like diffuse + GGX specular BRDF with one-sample MIS between the two
// lobes (materials.cu:1692-1957).  B.a = diffuseColor, B.b = specularF0Color,
// f0 = roughness.
struct UE4Weights { float diffuse, specular; };
VLRB_HD UE4Weights ue4Weights(const Bsdf &B, float cosV, float qz, uint32_t wl, bool squareViaPow2) {
    float rough = B.f0;
    // The reference squares with pow2() in sample/reverse paths and by two
    // left-to-right products in evaluatePDF (materials.cu:1724 vs :1898).
    float expF_D90 = squareViaPow2 ? 0.5f * rough + 2 * rough * sq(qz)
                                   : 0.5f * rough + 2 * rough * qz * qz;
    float oneMinusDotVN5 = quint(1 - cosV);
    float expDiffuseFresnel = lerpf(1.0f, expF_D90, oneMinusDotVN5);
    float iBase = squareViaPow2
        ? B.a.importance(wl) * sq(expDiffuseFresnel) * lerpf(1.0f, 1.0f / 1.51f, rough)
        : B.a.importance(wl) * expDiffuseFresnel * expDiffuseFresnel * lerpf(1.0f, 1.0f / 1.51f, rough);
    float expOneMinusDotVH5 = quint(1 - cosV);
    float iSpecF0 = B.b.importance(wl);
    return UE4Weights{ iBase, lerpf(iSpecF0, 1.0f, expOneMinusDotVH5) };
}
VLRB_HD S4 ue4Value(const Bsdf &B, const GGX &ggx, const V3 &dirL, const V3 &dirV, const V3 &m, float dotLH,
                    float D, float oneMinusDotVN5, bool dotLHSquaredByPow2) {
    float rough = B.f0;
    float oneMinusDotLH5 = quint(1 - dotLH);
    float G = ggx.G2HeightCorrelated(dirL, dirV, m);
    S4 F = lerpS(B.b, S4::one(), oneMinusDotLH5);
    float denom = 4 * dirL.z * dirV.z;
    S4 specular = F * ((D * G) / denom);
    float F_D90 = dotLHSquaredByPow2 ? 0.5f * rough + 2 * rough * sq(dotLH)
                                     : 0.5f * rough + 2 * rough * dotLH * dotLH;
    float oneMinusDotLN5 = quint(1 - dirL.z);
    float dfOut = lerpf(1.0f, F_D90, oneMinusDotVN5);
    float dfIn = lerpf(1.0f, F_D90, oneMinusDotLN5);
    S4 diffuse = B.a * (dfOut * dfIn * lerpf(1.0f, 1.0f / 1.51f, rough) / kPi);
    return diffuse + specular;
}
VLRB_HD float ue4RevPDF(const Bsdf &B, const GGX &ggx, const V3 &dirL, const V3 &dirV, const V3 &m, float dotLH, uint32_t wl) {
    float revDiffusePDF = dirV.z / kPi;
    float common = 1.0f / (4 * dotLH);
    float revSpecPDF = common * ggx.pdf(dirL, m);
    UE4Weights w = ue4Weights(B, dirL.z, dirL.z, wl, true);
    return (revDiffusePDF * w.diffuse + revSpecPDF * w.specular) / (w.diffuse + w.specular);
}
VLRB_HD S4 ue4Sample(const Bsdf &B, const BsdfQuery &q, float uc, float u0, float u1, BsdfSample* r, BsdfRev* rev) {
    if (rev) rev->dirPDF = 0.0f;
    float alpha = sq(B.f0);
    GGX ggx(alpha, alpha, 0.0f);
    bool entering = q.dirLocal.z >= 0.0f;
    V3 dirL;
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    float oneMinusDotVN5 = quint(1 - dirV.z);
    UE4Weights w = ue4Weights(B, dirV.z, q.dirLocal.z, q.wlHint, true);
    float weights[2] = { w.diffuse, w.specular };
    float probSel, sumW = 0.0f, ucr;
    uint32_t comp = sampleDiscrete2(weights, uc, &probSel, &sumW, &ucr);
    float diffusePDF = 0.0f, specPDF = 0.0f;
    V3 m;
    float dotLH = 0.0f;
    float D = 0.0f;
    if (comp == 0) {
        r->sampledType = dir::Reflection | dir::LowFreq;
        dirL = cosineHemisphere(u0, u1);
        diffusePDF = dirL.z / kPi;
        m = halfVector(dirL, dirV);
        dotLH = dot(dirL, m);
        float common = 1.0f / (4 * dotLH);
        specPDF = common * ggx.pdf(dirV, m);
        D = ggx.D(m);
    }
    else {
        r->sampledType = dir::Reflection | dir::HighFreq;
        float mPDF;
        D = ggx.sample(dirV, u0, u1, &m, &mPDF);
        float dotVH = dot(dirV, m);
        dotLH = dotVH;
        dirL = 2 * dotVH * m - dirV;
        if (dirL.z * dirV.z <= 0) { r->dirPDF = 0.0f; return S4::zero(); }
        float common = 1.0f / (4 * dotLH);
        specPDF = common * mPDF;
        diffusePDF = dirL.z / kPi;
    }
    S4 ret = ue4Value(B, ggx, dirL, dirV, m, dotLH, D, oneMinusDotVN5, false);
    r->dirLocal = entering ? dirL : -dirL;
    r->dirPDF = (diffusePDF * w.diffuse + specPDF * w.specular) / sumW;
    if (rev) {
        rev->value = ret;
        rev->dirPDF = ue4RevPDF(B, ggx, dirL, dirV, m, dotLH, q.wlHint);
    }
    return ret;
}
VLRB_HD S4 ue4Eval(const Bsdf &B, const BsdfQuery &q, const V3 &d, S4* revValue) {
    float alpha = sq(B.f0);
    GGX ggx(alpha, alpha, 0.0f);
    if (d.z * q.dirLocal.z <= 0) return S4::zero();
    bool entering = q.dirLocal.z >= 0.0f;
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    V3 m = halfVector(dirL, dirV);
    float dotLH = dot(dirL, m);
    float D = ggx.D(m);
    float oneMinusDotVN5 = quint(1 - dirV.z);
    S4 ret = ue4Value(B, ggx, dirL, dirV, m, dotLH, D, oneMinusDotVN5, true);
    if (revValue) *revValue = ret;
    return ret;
}
VLRB_HD float ue4PDF(const Bsdf &B, const BsdfQuery &q, const V3 &d, float* revPDF) {
    if (revPDF) *revPDF = 0.0f;
    float alpha = sq(B.f0);
    GGX ggx(alpha, alpha, 0.0f);
    bool entering = q.dirLocal.z >= 0.0f;
    V3 dirV = entering ? q.dirLocal : -q.dirLocal;
    V3 dirL = entering ? d : -d;
    V3 m = halfVector(dirL, dirV);
    float dotLH = dot(dirL, m);
    float common = 1.0f / (4 * dotLH);
    UE4Weights w = ue4Weights(B, dirV.z, q.dirLocal.z, q.wlHint, false);
    float sumW = w.diffuse + w.specular;
    float diffusePDF = vmax(dirL.z / kPi, 0.0f);
    float specPDF = common * ggx.pdf(dirV, m);
    float ret = (diffusePDF * w.diffuse + specPDF * w.specular) / sumW;
    if (revPDF) *revPDF = ue4RevPDF(B, ggx, dirL, dirV, m, dotLH, q.wlHint);
    return ret;
}

// Type flags each BSDF "matches" against (the matches() members in materials.cu).
VLRB_HD uint32_t bsdfTypeFlags(uint32_t kind) {
    switch (kind) {
    case kMatte: return dir::Reflection | dir::LowFreq;
    case kSpecularBRDF: return dir::Reflection | dir::Delta0D;
    case kMicrofacetBRDF: return dir::Reflection | dir::HighFreq;
    case kMicrofacetBSDF: return dir::WholeSphere | dir::HighFreq;
    case kLambertianBSDF: return dir::WholeSphere | dir::LowFreq;
    case kUE4: return dir::Reflection | dir::LowFreq | dir::HighFreq;
    case kSpecularBSDF: return dir::WholeSphere | dir::Delta0D;
    default: return 0u;
    }
}

// Unwrapped ("Internal") entry points, static dispatch on the kind.
VLRB_HD S4 bsdfSampleInternal(const Bsdf &B, const BsdfQuery &q, float uc, float u0, float u1,
                              BsdfSample* r, BsdfRev* rev) {
    switch (B.kind) {
    case kMatte: return matteSample(B, q, uc, u0, u1, r, rev);
    case kSpecularBRDF: return specBrdfSample(B, q, uc, u0, u1, r, rev);
    case kMicrofacetBRDF: return mfBrdfSample(B, q, uc, u0, u1, r, rev);
    case kMicrofacetBSDF: return mfBsdfSample(B, q, uc, u0, u1, r, rev);
    case kLambertianBSDF: return lambSample(B, q, uc, u0, u1, r, rev);
    case kUE4: return ue4Sample(B, q, uc, u0, u1, r, rev);
    case kSpecularBSDF: return specBsdfSample(B, q, uc, u0, u1, r, rev);
    default:
        r->dirPDF = 0.0f;
        if (rev) rev->dirPDF = 0.0f;
        return S4::zero();
    }
}
VLRB_HD S4 bsdfEvalInternal(const Bsdf &B, const BsdfQuery &q, const V3 &d, S4* revValue) {
    switch (B.kind) {
    case kMatte: return matteEval(B, q, d, revValue);
    case kMicrofacetBRDF: return mfBrdfEval(B, q, d, revValue);
    case kMicrofacetBSDF: return mfBsdfEval(B, q, d, revValue);
    case kLambertianBSDF: return lambEval(B, q, d, revValue);
    case kUE4: return ue4Eval(B, q, d, revValue);
    default:
        if (revValue) *revValue = S4::zero();
        return S4::zero();
    }
}
VLRB_HD float bsdfPDFInternal(const Bsdf &B, const BsdfQuery &q, const V3 &d, float* revPDF) {
    switch (B.kind) {
    case kMatte: return mattePDF(B, q, d, revPDF);
    case kMicrofacetBRDF: return mfBrdfPDF(B, q, d, revPDF);
    case kMicrofacetBSDF: return mfBsdfPDF(B, q, d, revPDF);
    case kLambertianBSDF: return lambPDF(B, q, d, revPDF);
    case kUE4: return ue4PDF(B, q, d, revPDF);
    default:
        if (revPDF) *revPDF = 0.0f;
        return 0.0f;
    }
}

// BSDF wrapper with the shading-normal correction (shared/renderer_common.h:96-163
// unidirectional, :230-311 bidirectional).  ngLocal = geometric normal in the
// shading frame.
VLRB_HD bool bsdfHasNonDelta(const Bsdf &B) {
    return dir::matches(bsdfTypeFlags(B.kind), dir::WholeSphere | dir::NonDelta);
}
VLRB_HD S4 bsdfSample(const Bsdf &B, const BsdfQuery &q, const V3 &ngLocal, float uc, float u0, float u1,
                      BsdfSample* r, BsdfRev* rev) {
    r->dirPDF = 0.0f;
    r->sampledType = 0;
    if (rev) rev->dirPDF = 0.0f;
    if (!dir::matches(bsdfTypeFlags(B.kind), q.filter)) return S4::zero();
    S4 fs = bsdfSampleInternal(B, q, uc, u0, u1, r, rev);
    float sn = !q.importanceMode ? std::fabs(r->dirLocal.z / dot(r->dirLocal, ngLocal))
                                 : std::fabs(q.dirLocal.z / dot(q.dirLocal, ngLocal));
    if (!std::isfinite(sn)) return S4::zero();
    if (rev) rev->value *= sn;
    return fs * sn;
}
VLRB_HD S4 bsdfEval(const Bsdf &B, const BsdfQuery &q, const V3 &ngLocal, const V3 &d, S4* revValue) {
    float sn = !q.importanceMode ? std::fabs(d.z / dot(d, ngLocal))
                                 : std::fabs(q.dirLocal.z / dot(q.dirLocal, ngLocal));
    if (!std::isfinite(sn)) { if (revValue) *revValue = S4::zero(); return S4::zero(); }
    S4 fs = bsdfEvalInternal(B, q, d, revValue);
    if (revValue) *revValue *= sn;
    return fs * sn;
}
VLRB_HD float bsdfPDF(const Bsdf &B, const BsdfQuery &q, const V3 &d, float* revPDF) {
    if (!dir::matches(bsdfTypeFlags(B.kind), q.filter)) { if (revPDF) *revPDF = 0.0f; return 0.0f; }
    return bsdfPDFInternal(B, q, d, revPDF);
}

// ---------------------------------------------------------------- EDFs
// DiffuseEDF (materials.cu:2040-2093): Le = M / pi on the front hemisphere.
VLRB_HD float diffuseEdfEval(const V3 &dirLocal) { return dirLocal.z > 0.0f ? 1.0f / kPi : 0.0f; }

// uniformSampleSphere (random_distributions.h:141-145): theta = acos(1 - 2 u0),
// phi = 2 pi u1, z up.
VLRB_HD V3 uniformSphere(float u0, float u1) {
    const float phi = 2 * kPi * u1, theta = acosf(1 - 2 * u0);
    float sinPhi, cosPhi, sinTheta, cosTheta;
    fsincos(phi, &sinPhi, &cosPhi);
    fsincos(theta, &sinTheta, &cosTheta);
    return V3(cosPhi * sinTheta, sinPhi * sinTheta, cosTheta);
}

// Emitter kinds (MatDesc::emitter) and their EDFs' directional factors
// (materials.cu:2040-2250, 2830-2893): diffuse and environment 1/pi on the
// front side, a point 1/(4 pi) everywhere, a directional emitter 0 (its
// emission is a delta direction: only light subpaths carry it).
enum : uint32_t { kEmitNone = 0, kEmitDiffuse = 1, kEmitEnvironment = 2, kEmitPoint = 3, kEmitDirectional = 4 };
VLRB_HD float edfEval(uint32_t emitter, const V3 &dirLocal) {
    if (emitter == kEmitPoint) return 1.0f / (4 * kPi);
    if (emitter == kEmitDirectional) return 0.0f;
    return diffuseEdfEval(dirLocal);
}
VLRB_HD float diffuseEdfPDF(const V3 &dirLocal) { return dirLocal.z <= 0.0f ? 0.0f : dirLocal.z / kPi; }

} // namespace vlrb
