// Device-side scene: flattened world-space triangles, materials, the light
// selection structures and the camera, plus the per-hit surface decoding and
// light sampling the integrators share.
//
// The light-selection scheme and the probabilities it reports are the
// reference's: a discrete distribution over emitting instances (the
// environment first), then over the emitting material groups of the instance,
// then over the group's triangles by area
// (shared/light_transport_common.h:179-192, GPU_kernels/triangle.cu:113-177).
#pragma once

#include "core.cuh"
#include "lbvh.cuh"

namespace vlrb {

// Material descriptor: everything the hit shader needs, spectra kept as
// Meng-upsampled triplets and evaluated at the path's wavelengths.
struct MatDesc {
    uint32_t bsdfKind;      // BsdfKind; kNullBSDF for pure emitters
    uint32_t emitter;       // 0 none, 1 diffuse area emitter, 2 environment
    UpSpec sp[3];           // per-kind spectra (see buildBsdf)
    float f[4];             // per-kind scalars
    UpSpec emit;            // emittance
    float emitScale;
    uint32_t bsdfFlags;     // Bsdf::flags bits chosen at scene build (kBsdfConsistentPdf)
    int32_t table[4] = { -1, -1, -1, -1 };   // sp[0..2], emit: index of the blended spectrum
                                             // in MengTables::blended (-1: evaluate the UpSpec)
    int32_t tex[3] = { -1, -1, -1 };         // sp[0..2]: Image2DTexture index (-1: none)
};

// Spectrum slot 0-2 (sp) or 3 (emit) of material m at the path's wavelengths
// and texture coordinates (tu, tv): a texture's filtered RGB upsampled at the
// hit (Image2DTextureShaderNode_Spectrum, shader_nodes.cu:410-445), else the
// scene's blended table, else the UpSpec.
VLRB_HD S4 matSpectrum(const MengTables &T, const MatDesc &m, int slot, const WLS &wls, float tu = 0.0f,
                       float tv = 0.0f) {
#if defined(__CUDA_ARCH__)
    if (slot < 3 && m.tex[slot] >= 0 && T.textures) {
        const float4 c = tex2DLod<float4>(T.textures[m.tex[slot]], tu, tv, 0.0f);
        const uint32_t info = T.texSpType[m.tex[slot]];
        const UpSpec up = mengUpsample(T, *T.colorMats, static_cast<SpType>(info & 0xFFu),
                                       static_cast<ColorSp>(info >> 8), c.x, c.y, c.z);
        return mengEvaluate(T, up, wls);
    }
#else
    (void)tu; (void)tv;
#endif
    if (T.blended && m.table[slot] >= 0) return blendedEvaluate(T.blended + m.table[slot] * kMengSamples, wls);
    return mengEvaluate(T, slot < 3 ? m.sp[slot] : m.emit, wls);
}

// A discrete distribution in the reference's layout (shared/shared.h:182-231):
// PMF[n], CDF[n + 1] with CDF[n] = 1, integral = sum of the raw weights.
struct Dist1D {
    const float* pmf;
    const float* cdf;
    float integral;
    uint32_t n;

    VLRB_HD uint32_t sample(float u, float* prob, float* remapped) const {
        int idx = 0;
        uint32_t np2 = 1;
        while (np2 < n) np2 <<= 1;
        for (int d = static_cast<int>(np2 >> 1); d >= 1; d >>= 1) {
            if (idx + d >= static_cast<int>(n)) continue;
            if (cdf[idx + d] <= u) idx += d;
        }
        *prob = pmf[idx];
        if (remapped) *remapped = (u - cdf[idx]) / (cdf[idx + 1] - cdf[idx]);
        return static_cast<uint32_t>(idx);
    }
};

// Piecewise-constant 2D distribution over [0,1)^2 with an FP64 CDF: one
// conditional CDF per row plus the marginal over rows.  Replaces the
// reference's FP32 RegularConstantContinuousDistribution2D
// (shared/shared.h:235-302, host builder context.cpp:1844-1919).
struct EnvDist {
    const double* rowCdf;     // [h][w + 1]
    const double* margCdf;    // [h + 1]
    const float* rowPdf;      // [h][w] conditional density (normalised to mean 1)
    const float* margPdf;     // [h]
    uint32_t w, h;
};

struct EmitGroup {
    uint32_t firstTri;        // offset into lightTris
    uint32_t numTris;
    uint32_t material;
    uint32_t points;          // 1: the group is points (lightTris holds point ids), 0: triangles
    Dist1D prims;             // area distribution over the group's triangles (uniform over points)
};

enum : uint32_t { kCameraPerspective = 0, kCameraEquirectangular = 1 };

struct Camera {
    V3 position;
    V3 right, up, forward;    // orientation matrix columns
    float sensitivity;
    float lensRadius;         // 0 for the equirectangular camera (a point)
    float imgPlaneDistance, objPlaneDistance;
    float opWidth, opHeight, imgPlaneArea;
    uint32_t kind;            // kCamera*
    float phiAngle, thetaAngle;   // equirectangular: horizontal and vertical extent (radians)
};

// The camera's IDF sample for screen position (u0, u1) in [0, 1)^2 from the
// lens point (xOnLens, yOnLens): the direction in the lens frame (z =
// forward) and its density per solid angle over the whole image
// (PerspectiveCameraIDF::sampleInternal, cameras.cu:144-157;
// EquirectangularCameraIDF::sampleInternal, :272-288).
VLRB_HD V3 cameraSampleDir(const Camera &C, float xOnLens, float yOnLens, float u0, float u1, float* dirPDF) {
    if (C.kind == kCameraEquirectangular) {
        const float phi = kPi + C.phiAngle * (u0 - 0.5f);
        const float theta = 0.5f * kPi + C.thetaAngle * (u1 - 0.5f);
        float sinPhi, cosPhi, sinTheta, cosTheta;
        fsincos(phi, &sinPhi, &cosPhi);
        fsincos(theta, &sinTheta, &cosTheta);
        *dirPDF = 1.0f / (C.phiAngle * C.thetaAngle * sinTheta);
        return V3(sinPhi * sinTheta, cosTheta, -cosPhi * sinTheta);
    }
    V3 pFocus(C.opWidth * (0.5f - u0), C.opHeight * (0.5f - u1), C.objPlaneDistance);
    V3 dirLocal = normalize(pFocus - V3(xOnLens, yOnLens, 0.0f));
    *dirPDF = sq(C.imgPlaneDistance) / (cube(dirLocal.z) * C.imgPlaneArea);
    return dirLocal;
}

// Inverse of cameraSampleDir: the screen position a lens-frame direction
// projects to and its density, false off the frame (evaluatePDFInternal and
// backProjectDirection, cameras.cu:175-211, :301-341).
VLRB_HD bool cameraProject(const Camera &C, float xOnLens, float yOnLens, const V3 &dirLocal, float* u0, float* u1,
                           float* pdf) {
    if (C.kind == kCameraEquirectangular) {
        const float theta = acosf(vclamp(dirLocal.y, -1.0f, 1.0f));
        const float phi = fmodf(atan2f(dirLocal.x, -dirLocal.z) + 2 * kPi, 2 * kPi);
        *u0 = (phi - kPi) / C.phiAngle + 0.5f;
        *u1 = (theta - 0.5f * kPi) / C.thetaAngle + 0.5f;
        if (*u0 < 0.0f || *u0 >= 1.0f || *u1 < 0.0f || *u1 >= 1.0f) return false;
        const float sinTheta = sqrtf(1.0f - sq(dirLocal.y));
        *pdf = 1.0f / (C.phiAngle * C.thetaAngle * sinTheta);
        return true;
    }
    if (dirLocal.z <= 0.0f) return false;
    V3 org(xOnLens, yOnLens, 0.0f);
    float objZ = C.objPlaneDistance / dirLocal.z;
    V3 pFocus = dirLocal * objZ + org;
    *u0 = -pFocus.x / C.opWidth + 0.5f;
    *u1 = -pFocus.y / C.opHeight + 0.5f;
    if (*u0 < 0.0f || *u0 >= 1.0f || *u1 < 0.0f || *u1 >= 1.0f) return false;
    *pdf = sq(C.imgPlaneDistance) / (cube(dirLocal.z) * C.imgPlaneArea);
    return true;
}

// SurfacePoint::calcCosTerm at the lens (shared/kernel_common.h:202-204):
// the equirectangular camera is a point (cosine 1).
VLRB_HD float lensCos(const Camera &C, const V3 &dirWorld, const V3 &lensNormal) {
    return C.kind == kCameraEquirectangular ? 1.0f : absDot(dirWorld, lensNormal);
}

struct SceneBounds {
    V3 lo, hi, center;
    float worldRadius, worldDiscArea;
};

struct SceneGPU {
    Bvh bvh;
    uint32_t numTris;
    const float4* pos;        // [numVerts] world position
    const float4* nrm;        // [numVerts] world shading normal
    const float4* tan;        // [numVerts] world tc0Direction
    const float2* uv;         // [numVerts] texture coordinates (null when no material is textured)
    const uint4* tri;         // [numTris] i0, i1, i2, geomInst
    const uint32_t* triMaterial;
    const MatDesc* mats;
    // lights
    Dist1D lightInsts;              // over light instances (env first if present)
    const uint32_t* instFirstGroup; // per light instance
    const Dist1D* instGroups;       // per light instance: distribution over its groups
    const EmitGroup* groups;        // emitting material groups
    const float* geomLightPdfArea;  // per geomInst: instProb * groupProb / groupArea (0: not emitting)
    const uint32_t* geomInstGroup;  // per geomInst: emitting group index or ~0
    const uint32_t* lightTris;      // triangle ids of all emitting groups (point ids for point groups)
    const float4* ptPos;            // emitting points (PointSurfaceNode), world space
    const float4* ptNrm;
    const float4* ptTan;
    uint32_t hasDeltaEmitters;      // point or directional emitters present
    int32_t envInst;                // light-instance index of the environment, -1 if none
    uint32_t envMaterial;
    float envRotation;
    float envLightProb;             // instProb * geomInstProb of the environment
    EnvDist env;
    const UpSpec* envTexels;        // [h][w] upsampled radiance per texel
    SceneBounds bounds;
    Camera cam;
    MengTables meng;
};

struct SurfPt {
    V3 position;
    V3 gn;            // geometric normal
    Frame frame;      // shading frame
    uint32_t prim;
    uint32_t geomInst;
    float u, v;
    bool atInfinity;
    float tu = 0.0f, tv = 0.0f;   // texture coordinates (scenes with textures)
};

// Instantiate the BSDF of material m at the given wavelengths (the setupBSDF
// callables of materials.cu with immediate values).
// K >= 0: the material is known to be of that kind (the shade kernels
// specialised per material queue), which lets every BSDF dispatch fold.
template <int K = -1>
VLRB_HD Bsdf buildBsdf(const MengTables &T, const MatDesc &m, const WLS &wls, float tu = 0.0f, float tv = 0.0f) {
    Bsdf B;
    const uint32_t kind = K >= 0 ? static_cast<uint32_t>(K) : m.bsdfKind;
    B.kind = kind;
    B.flags = 0;
    B.f0 = m.f[0]; B.f1 = m.f[1]; B.f2 = m.f[2];
    switch (kind) {
    case kMatte:
    case kLambertianBSDF:
        B.a = matSpectrum(T, m, 0, wls, tu, tv);
        break;
    case kSpecularBRDF:
    case kSpecularBSDF:
    case kMicrofacetBSDF:
        B.a = matSpectrum(T, m, 0, wls, tu, tv);
        B.b = matSpectrum(T, m, 1, wls, tu, tv);
        B.c = matSpectrum(T, m, 2, wls, tu, tv);
        if (kind == kSpecularBSDF) B.flags = wls.single ? 0u : 1u;
        if (kind == kMicrofacetBSDF) B.flags = m.bsdfFlags & kBsdfConsistentPdf;
        break;
    case kMicrofacetBRDF:
        B.b = matSpectrum(T, m, 1, wls, tu, tv);
        B.c = matSpectrum(T, m, 2, wls, tu, tv);
        break;
    case kUE4: {
        // UE4SurfaceMaterial_setupBSDF (materials.cu:1959-1978); f[1] = metallic.
        S4 base = matSpectrum(T, m, 0, wls, tu, tv);
        const float metallic = m.f[1];
        const float specular = 0.5f;
        B.a = base * (1 - metallic);
        B.b = lerpS(0.08f * specular * S4::one(), base, metallic);
        B.f0 = m.f[0];
        break;
    }
    default:
        break;
    }
    return B;
}

VLRB_HD S4 emittance(const MengTables &T, const MatDesc &m, const WLS &wls) {
    if (m.emitter == kEmitNone) return S4::zero();
    return matSpectrum(T, m, 3, wls) * m.emitScale;
}

#if defined(__CUDACC__)

__device__ __forceinline__ V3 ld3(const float4* p, uint32_t i) {
    float4 v = __ldg(p + i);
    return V3(v.x, v.y, v.z);
}

// decodeLocalHitPointForTriangle + calcSurfacePoint (triangle.cu:6-53,
// renderer_common.h:609-626) on world-space vertices.
__device__ __forceinline__ void decodeHit(const SceneGPU &S, uint32_t prim, float b1, float b2, SurfPt* sp,
                                          float* hypAreaPDF) {
    uint4 t = __ldg(S.tri + prim);
    V3 p0 = ld3(S.pos, t.x), p1 = ld3(S.pos, t.y), p2 = ld3(S.pos, t.z);
    V3 e1 = p1 - p0, e2 = p2 - p0;
    V3 gn = cross(e1, e2);
    float area = gn.length() / 2;
    gn /= 2 * area;
    uint32_t g = t.w;
    sp->geomInst = g;
    uint32_t grp = __ldg(S.geomInstGroup + g);
    if (hypAreaPDF) {
        float integral = grp != 0xFFFFFFFFu ? S.groups[grp].prims.integral : 1.0f;
        float probLightPrim = area / integral;
        *hypAreaPDF = probLightPrim / area;
    }
    float b0 = 1 - b1 - b2;
    V3 position = b0 * p0 + b1 * p1 + b2 * p2;
    V3 n0 = ld3(S.nrm, t.x), n1 = ld3(S.nrm, t.y), n2 = ld3(S.nrm, t.z);
    V3 sn = normalize(b0 * n0 + b1 * n1 + b2 * n2);
    V3 t0 = ld3(S.tan, t.x), t1 = ld3(S.tan, t.y), t2 = ld3(S.tan, t.z);
    V3 tc0 = b0 * t0 + b1 * t1 + b2 * t2;
    if (!sn.allFinite() || !tc0.allFinite()) {
        V3 bt;
        sn = gn;
        makeBasis(sn, &tc0, &bt);
    }
    float dotNT = dot(sn, tc0);
    tc0 = tc0 - dotNT * sn;
    sp->position = position;
    sp->frame = Frame(normalize(tc0), normalize(sn));
    sp->gn = normalize(gn);
    sp->prim = prim;
    if (S.uv) {
        // texCoord = b0 t0 + b1 t1 + b2 t2 (triangle.cu:35)
        const float2 a = __ldg(S.uv + t.x), b = __ldg(S.uv + t.y), c = __ldg(S.uv + t.z);
        sp->tu = b0 * a.x + b1 * b.x + b2 * c.x;
        sp->tv = b0 * a.y + b1 * b.y + b2 * c.y;
    }
    else {
        sp->tu = 0.0f;
        sp->tv = 0.0f;
    }
    sp->u = b0;
    sp->v = b1;
    sp->atInfinity = false;
}

// Ray Tracing Gems ch. 6 origin offset (renderer_common.h:502-528).
__device__ __forceinline__ V3 offsetRayOrigin(const V3 &p, const V3 &n) {
    const float kOrigin = 1.0f / 32.0f;
    const float kFloatScale = 1.0f / 65536.0f;
    const float kIntScale = 256.0f;
    int ox = static_cast<int>(kIntScale * n.x), oy = static_cast<int>(kIntScale * n.y), oz = static_cast<int>(kIntScale * n.z);
    V3 p1(__int_as_float(__float_as_int(p.x) + (p.x < 0 ? -1 : 1) * ox),
          __int_as_float(__float_as_int(p.y) + (p.y < 0 ? -1 : 1) * oy),
          __int_as_float(__float_as_int(p.z) + (p.z < 0 ? -1 : 1) * oz));
    V3 p2 = p + kFloatScale * n;
    return V3(fabsf(p.x) < kOrigin ? p2.x : p1.x, fabsf(p.y) < kOrigin ? p2.y : p1.y,
              fabsf(p.z) < kOrigin ? p2.z : p1.z);
}

struct LightSample {
    SurfPt sp;
    float areaPDF;
    uint32_t material;
    bool delta;
    bool isPoint;            // calcCosTerm is 1 at a point (kernel_common.h:202-204)
};

// Sample a point on an emitting triangle group (triangle.cu:113-177).
__device__ __forceinline__ void sampleTriangleGroup(const SceneGPU &S, uint32_t grp, float uElem, float u0, float u1,
                                                    LightSample* ls) {
    const EmitGroup &G = S.groups[grp];
    float primProb;
    uint32_t local = G.prims.sample(uElem, &primProb, nullptr);
    ls->isPoint = false;
    if (G.points) {
        // samplePoint (point.cu:40-80): a delta position with the
        // hypothetical area of a unit sphere
        const uint32_t pt = __ldg(S.lightTris + G.firstTri + local);
        ls->areaPDF = primProb / (4 * kPi);
        ls->material = G.material;
        ls->delta = true;
        ls->isPoint = true;
        const V3 n = normalize(ld3(S.ptNrm, pt)), t = normalize(ld3(S.ptTan, pt));
        ls->sp.position = ld3(S.ptPos, pt);
        ls->sp.frame = Frame(t, n);
        ls->sp.gn = n;
        ls->sp.prim = pt;
        ls->sp.geomInst = 0;
        ls->sp.u = 0.0f;
        ls->sp.v = 0.0f;
        ls->sp.atInfinity = false;
        return;
    }
    uint32_t prim = __ldg(S.lightTris + G.firstTri + local);
    uint4 t = __ldg(S.tri + prim);
    V3 p0 = ld3(S.pos, t.x), p1 = ld3(S.pos, t.y), p2 = ld3(S.pos, t.z);
    V3 e1 = p1 - p0, e2 = p2 - p0;
    V3 gn = cross(e1, e2);
    float area = gn.length() / 2;
    gn /= 2 * area;
    ls->areaPDF = primProb / area;
    ls->material = G.material;
    ls->delta = false;
    float b0, b1;
    uniformTriangle(u0, u1, &b0, &b1);
    float b2 = 1.0f - b0 - b1;
    V3 position = b0 * p0 + b1 * p1 + b2 * p2;
    V3 n0 = ld3(S.nrm, t.x), n1 = ld3(S.nrm, t.y), n2 = ld3(S.nrm, t.z);
    V3 sn = normalize(b0 * n0 + b1 * n1 + b2 * n2);
    V3 t0 = ld3(S.tan, t.x), t1 = ld3(S.tan, t.y), t2 = ld3(S.tan, t.z);
    V3 tc0 = b0 * t0 + b1 * t1 + b2 * t2;
    float dotNT = dot(sn, tc0);
    tc0 = normalize(tc0 - dotNT * sn);
    ls->sp.position = position;
    ls->sp.frame = Frame(tc0, sn);
    ls->sp.gn = gn;
    ls->sp.prim = prim;
    ls->sp.geomInst = t.w;
    ls->sp.u = b0;
    ls->sp.v = b1;
    ls->sp.atInfinity = false;
}

// Equirectangular environment: direction <-> (phi, theta) with Y up
// (include/vlr/basic_types.h:72-88).
__device__ __forceinline__ V3 dirFromPolarYUp(float phi, float theta) {
    float sp, cp, st, ct;
    fsincos(phi, &sp, &cp);
    fsincos(theta, &st, &ct);
    return V3(-sp * st, ct, cp * st);
}
__device__ __forceinline__ void toPolarYUp(const V3 &d, float* theta, float* phi) {
    *theta = acosf(vclamp(d.y, -1.0f, 1.0f));
    *phi = fmodf(atan2f(-d.x, d.z) + 2 * kPi, 2 * kPi);
}

// Sample the FP64 CDF of the environment importance map.
__device__ __forceinline__ uint32_t searchCdf64(const double* cdf, uint32_t n, double u) {
    uint32_t lo = 0, hi = n;  // cdf has n + 1 entries, find last i with cdf[i] <= u
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (cdf[mid] <= u) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void envSampleUV(const EnvDist &E, float u0, float u1, float* uu, float* vv, float* pdf) {
    uint32_t row = searchCdf64(E.margCdf, E.h, static_cast<double>(u1));
    double c0 = E.margCdf[row], c1 = E.margCdf[row + 1];
    double tv = c1 > c0 ? (static_cast<double>(u1) - c0) / (c1 - c0) : 0.5;
    const double* rc = E.rowCdf + static_cast<size_t>(row) * (E.w + 1);
    uint32_t col = searchCdf64(rc, E.w, static_cast<double>(u0));
    double r0 = rc[col], r1 = rc[col + 1];
    double tu = r1 > r0 ? (static_cast<double>(u0) - r0) / (r1 - r0) : 0.5;
    *uu = static_cast<float>((col + tu) / E.w);
    *vv = static_cast<float>((row + tv) / E.h);
    *pdf = E.margPdf[row] * E.rowPdf[static_cast<size_t>(row) * E.w + col];
}

__device__ __forceinline__ float envPdfUV(const EnvDist &E, float u, float v) {
    uint32_t row = min(static_cast<uint32_t>(v * E.h), E.h - 1);
    uint32_t col = min(static_cast<uint32_t>(u * E.w), E.w - 1);
    return E.margPdf[row] * E.rowPdf[static_cast<size_t>(row) * E.w + col];
}

// Radiance of the environment at texture coordinate (u, v), nearest texel.
__device__ __forceinline__ S4 envRadiance(const SceneGPU &S, float u, float v, const WLS &wls) {
    uint32_t row = min(static_cast<uint32_t>(v * S.env.h), S.env.h - 1);
    uint32_t col = min(static_cast<uint32_t>(u * S.env.w), S.env.w - 1);
    UpSpec t = S.envTexels[static_cast<size_t>(row) * S.env.w + col];
    return mengEvaluate(S.meng, t, wls);
}

#endif

} // namespace vlrb
