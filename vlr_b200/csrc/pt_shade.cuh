// Shading steps of the path tracer shared by the wavefront kernels (pt.cu)
// and the persistent batch kernel (pt_persistent.cu).  Each follows
// path_tracing.cu's arithmetic in its order, so both integrators produce
// the same values from the same random numbers.
#pragma once

#include "pt.cuh"
#include "wavefront.cuh"

namespace vlrb {

#if defined(__CUDACC__)

// A camera path's start (path_tracing.cu:30-77): pixel jitter, the hero
// wavelengths, the lens sample and the camera's IDF sample
// (PerspectiveCamera_sample, cameras.cu:42-74; the IDF, cameras.cu:142-155
// perspective and :272-288 equirectangular), the density per pixel.
struct CameraRay {
    WLS wls;
    S4 alpha;
    float initImportance, dirPDF;
    V3 org, dir;
};

__device__ __forceinline__ CameraRay cameraSample(const SceneGPU &S, uint32_t px, uint32_t py, uint32_t W,
                                                  uint32_t H, PCG32 &rng) {
    CameraRay r;
    const float jx = rng.uniform(), jy = rng.uniform();
    const float fx = px + jx, fy = py + jy;
    float selectWLPDF;
    const float wo = rng.uniform(), ws = rng.uniform();
    r.wls = WLS::equalOffsets(wo, ws, &selectWLPDF);
    const Camera &C = S.cam;
    float lx, ly;
    const float l0 = rng.uniform(), l1 = rng.uniform();
    concentricDisk(l0, l1, &lx, &ly);
    const V3 orgLocal(C.lensRadius * lx, C.lensRadius * ly, 0.0f);
    const V3 gn = normalize(C.forward);
    Frame camFrame;
    camFrame.z = gn;
    camFrame.x = normalize(C.right);
    camFrame.y = cross(camFrame.z, camFrame.x);
    r.org = C.right * orgLocal.x + C.up * orgLocal.y + C.forward * orgLocal.z + C.position;
    const float areaPDF = C.lensRadius > 0.0f ? 1.0f / (kPi * C.lensRadius * C.lensRadius) : 1.0f;
    const float u0 = fx / W, u1 = fy / H;
    float dirPDF;
    const V3 dirLocal = cameraSampleDir(C, C.lensRadius * lx, C.lensRadius * ly, u0, u1, &dirPDF);
    dirPDF *= static_cast<float>(W * H);
    r.dir = camFrame.fromLocal(dirLocal);
    const S4 We0(C.sensitivity);
    r.alpha = (We0 * S4::one()) * (lensCos(C, r.dir, gn) / (areaPDF * dirPDF * selectWLPDF));
    r.initImportance = r.alpha.importance(r.wls.selected);
    r.dirPDF = dirPDF;
    return r;
}

// The previous vertex's sampling record of a path (its direction type and
// density), read only where a MIS weight needs it: from the wavefront's
// path buffers, or from registers in the persistent kernel.
struct PrevFromBuffers {
    const PathBuffers* pb;
    uint32_t p;
    __device__ __forceinline__ uint32_t type() const { return pb->prevType[p]; }
    __device__ __forceinline__ float dirPDF() const { return pb->prevDirPDF[p]; }
};
struct PrevInRegisters {
    uint32_t t;
    float pdf;
    __device__ __forceinline__ uint32_t type() const { return t; }
    __device__ __forceinline__ float dirPDF() const { return pdf; }
};

// Environment light reaching a path that left the scene, MIS-weighted
// against the environment's light sampling (path_tracing.cu:266-337), added
// to contrib as alpha * Le * MIS.  Nothing without an environment.
// EnvironmentEDF: emittance pi*E, directional factor 1/pi for the direction
// facing the scene (materials.cu:2830-2893).
template <class Prev>
__device__ __forceinline__ void envMissContribution(const SceneGPU &S, const V3 &direction, const WLS &wls,
                                                    const S4 &alpha, const Prev &prev, uint32_t pathLength,
                                                    S4 &contrib) {
    if (S.envInst < 0) return;
    float phi, theta;
    toPolarYUp(direction, &theta, &phi);
    phi += S.envRotation;
    phi = phi - floorf(phi / (2 * kPi)) * 2 * kPi;
    const float tu = phi / (2 * kPi), tv = theta / kPi;
    const float uvPDF = envPdfUV(S.env, tu, tv);
    const float hypAreaPDF = uvPDF / (2 * kPi * kPi * sinf(theta));
    const MatDesc &m = S.mats[S.envMaterial];
    const S4 E = envRadiance(S, tu, tv, wls) * m.emitScale;
    const S4 spEmittance = kPi * E;
    if (!spEmittance.hasNonZero()) return;
    const S4 Le = spEmittance * (1.0f / kPi);
    float MIS = 1.0f;
    if (!dir::isDelta(prev.type()) && pathLength > 1) {
        const float bsdfPDF = prev.dirPDF();
        const float lightPDF = S.envLightProb * hypAreaPDF * 1.0f / 1.0f;
        MIS = (bsdfPDF * bsdfPDF) / (lightPDF * lightPDF + bsdfPDF * bsdfPDF);
    }
    contrib += alpha * Le * MIS;
}

// Emission of the surface a path hit, MIS-weighted against light sampling
// (path_tracing.cu:146-176), added to contrib as alpha * Le * MIS.
template <class Prev>
__device__ __forceinline__ void implicitEmission(const SceneGPU &S, const MatDesc &mat, const WLS &wls,
                                                 const SurfPt &sp, const V3 &dirOutLocal, const V3 &rayOrg,
                                                 float hypAreaPDF, const Prev &prev, uint32_t pathLength,
                                                 const S4 &alpha, S4 &contrib) {
    const S4 spEmittance = emittance(S.meng, mat, wls);
    if (!spEmittance.hasNonZero()) return;
    const S4 Le = spEmittance * edfEval(mat.emitter, dirOutLocal);
    float MIS = 1.0f;
    if (!dir::isDelta(prev.type()) && pathLength > 1) {
        const float bsdfPDF = prev.dirPDF();
        const float dist2 = (sp.position - rayOrg).sqLength();
        const float lightPDF = __ldg(S.geomLightPdfArea + sp.geomInst) * hypAreaPDF * dist2 / fabsf(dirOutLocal.z);
        MIS = (bsdfPDF * bsdfPDF) / (lightPDF * lightPDF + bsdfPDF * bsdfPDF);
    }
    contrib += alpha * Le * MIS;
}

// A next-event-estimation shadow ray and the contribution it carries when
// unoccluded.
struct NeeRay {
    V3 org, dir;
    float tmax;
    S4 contrib;
};

// Next-event estimation at a surface point (path_tracing.cu:177-233,
// light_transport_common.h:147-177): two-level light selection, the
// environment's infinite sphere (infinite_sphere.cu:60-114) or an emitting
// triangle group, the BSDF value and MIS weight.  Draws uLight, ue0, ue1 when
// the BSDF has a non-delta component and the scene has lights.  Returns
// false when no shadow ray is needed (no light, zero emission or zero
// contribution).  With guided, the BSDF density in the MIS weight is the
// one-sample mixture 0.5 BSDF + 0.5 network.
template <bool kGuide>
__device__ __forceinline__ bool neeSample(const SceneGPU &S, const SurfPt &sp, const Bsdf &bsdf, const BsdfQuery &q,
                                          const V3 &gnLocal, const WLS &wls, const S4 &alpha, PCG32 &rng,
                                          bool guided, const guide::Mixture &mix, NeeRay* out) {
    if (!(bsdfHasNonDelta(bsdf) && S.lightInsts.n > 0)) return false;
    const float uLight = rng.uniform();
    float instProb, uInst;
    const uint32_t li = S.lightInsts.sample(uLight, &instProb, &uInst);
    const float ue0 = rng.uniform(), ue1 = rng.uniform();
    LightSample ls;
    float lightProb;
    S4 M;
    bool ok = true;
    if (static_cast<int32_t>(li) == S.envInst) {
        // sampleInfiniteSphere (infinite_sphere.cu:60-114)
        float groupProb, uPrim;
        S.instGroups[li].sample(uInst, &groupProb, &uPrim);
        lightProb = instProb * groupProb;
        float uu, vv, uvPDF;
        envSampleUV(S.env, ue0, ue1, &uu, &vv, &uvPDF);
        const float phi = 2 * kPi * uu, theta = kPi * vv;
        float posPhi = phi - S.envRotation;
        posPhi = posPhi - floorf(posPhi / (2 * kPi)) * 2 * kPi;
        const V3 dirE = dirFromPolarYUp(posPhi, theta);
        ls.sp.position = dirE;
        ls.sp.gn = -dirE;
        ls.sp.frame.z = -dirE;
        ls.sp.atInfinity = true;
        ls.areaPDF = uvPDF / (2 * kPi * kPi * sinf(theta));
        ls.delta = false;
        ls.isPoint = false;
        ls.material = S.envMaterial;
        M = kPi * envRadiance(S, uu, vv, wls) * S.mats[S.envMaterial].emitScale;
        ok = uvPDF > 0.0f;
    }
    else {
        float groupProb, uPrim;
        const uint32_t g = S.instGroups[li].sample(uInst, &groupProb, &uPrim);
        lightProb = instProb * groupProb;
        const uint32_t grp = __ldg(S.instFirstGroup + li) + g;
        sampleTriangleGroup(S, grp, uPrim, ue0, ue1, &ls);
        M = emittance(S.meng, S.mats[ls.material], wls);
    }
    if (!(ok && M.hasNonZero())) return false;
    // testVisibility (light_transport_common.h:147-177)
    V3 shadowDir;
    float dist2;
    if (ls.sp.atInfinity) { shadowDir = normalize(ls.sp.position); dist2 = 1.0f; }
    else {
        const V3 dv = ls.sp.position - sp.position;
        dist2 = dv.sqLength();
        shadowDir = dv / sqrtf(dist2);
    }
    const bool front = dot(sp.gn, shadowDir) > 0;
    const V3 sOrg = offsetRayOrigin(sp.position, front ? sp.gn : -sp.gn);
    float tmax = FLT_MAX;
    if (!ls.sp.atInfinity) {
        const bool lfront = -dot(ls.sp.gn, shadowDir) > 0;
        const V3 lPt = offsetRayOrigin(ls.sp.position, lfront ? ls.sp.gn : -ls.sp.gn);
        tmax = (lPt - sOrg).length() * 0.9999f;
    }
    const float recSqDist = 1.0f / dist2;
    const V3 dirL = ls.sp.atInfinity ? V3(0.0f, 0.0f, 1.0f) : ls.sp.frame.toLocal(-shadowDir);
    const V3 dirSn = sp.frame.toLocal(shadowDir);
    const S4 Le = M * edfEval(S.mats[ls.material].emitter, dirL);
    const float lightPDF = lightProb * ls.areaPDF;
    const S4 fs = bsdfEval(bsdf, q, gnLocal, dirSn, nullptr);
    const float cosLight = ls.isPoint ? 1.0f : absDot(-shadowDir, ls.sp.gn);
    float dirPdfV = bsdfPDF(bsdf, q, dirSn, nullptr);
    if constexpr (kGuide) {
        if (guided) dirPdfV = 0.5f * dirPdfV + 0.5f * guide::mixturePdf(mix, shadowDir);
    }
    const float bsdfPdfV = dirPdfV * cosLight * recSqDist;
    float MIS = 1.0f;
    if (!ls.delta && !isinf(lightPDF))
        MIS = (lightPDF * lightPDF) / (lightPDF * lightPDF + bsdfPdfV * bsdfPdfV);
    const float G = absDot(dirSn, gnLocal) * cosLight * recSqDist;
    const float scalar = G * MIS / lightPDF;
    const S4 c = alpha * Le * fs * scalar;
    if (!c.hasNonZero()) return false;
    out->org = sOrg;
    out->dir = shadowDir;
    out->tmax = tmax;
    out->contrib = c;
    return true;
}

#endif

} // namespace vlrb
