// Light-vertex-cache bidirectional path tracing (Davidovic et al. 2014, as the
// reference implements it in GPU_kernels/lvc_bpt.cu), as wavefronts:
//
//   lightStartKernel   pick a light, store vertex y0, sample the emission
//                      direction (lvc_bpt.cu:144-243)
//   per bounce:        sorted trace, then lightShadeKernel: MIS partial-sum
//                      recursion, store the vertex in the cache with a bounded
//                      append, sample the BSDF in importance mode, Russian
//                      roulette folded into the densities (lvc_bpt.cu:246-334)
//   eyeStartKernel     lens sample, the t=1 connection (lens to a random cached
//                      vertex, splatted to the pixel it projects to), camera
//                      ray (lvc_bpt.cu:338-506)
//   per bounce:        sorted trace, then eyeShadeKernel: implicit emission
//                      (s=0) with its MIS weight, one connection to a random
//                      cached vertex, BSDF sample (lvc_bpt.cu:561-836), misses
//                      against the environment (lvc_bpt.cu:841-971);
//                      connectKernel traces the connection rays and adds the
//                      visible ones
//   eyeFilmKernel      adds each eye path's accumulated contribution.
//
// Unlike the reference, the cache append is bounded: a full cache drops the
// vertex and counts it (the reference's atomicAdd has no capacity check,
// lvc_bpt.cu:113-114).
#include "bpt.cuh"
#include "wavefront.cuh"

#include <stdexcept>
#include <string>

namespace vlrb {

namespace {

constexpr uint32_t kFlagSingle = 1u, kFlagOriginPoint = 2u, kFlagOriginInf = 4u, kFlagPrevDelta = 8u,
                   kFlagSecondPrevDelta = 16u;
constexpr uint32_t kSplatBit = 0x80000000u;

struct BptArgs {
    SceneGPU S;
    PathBuffers pb;        // light or eye paths, as the kernel needs
    BptExtra ex;
    BptBuffers bb;
    Film film;
    WLS wls;               // the frame's common wavelength samples
    float wlPdf;
    uint32_t numLightPaths;
    uint32_t numPaths;
    uint32_t width, height;   // the image being rendered
    uint32_t stride;          // film row length in pixels
    uint32_t maxPathLength;
    uint32_t bounce;
    struct LtConnection* conn;   // light tracing: lens connections of the current stage
};

__device__ __forceinline__ uint32_t pathLengthOf(uint32_t f) { return (f >> 8) & 0xFFFFu; }
__device__ __forceinline__ uint32_t withPathLength(uint32_t f, uint32_t l) { return (f & 0xFFu) | (l << 8); }

// computeRRProbability (lvc_bpt.cu:135-139)
__device__ __forceinline__ float rrProb(const S4 &fs, const V3 &dirLocal, float dirDensity, const V3 &gnLocal,
                                        uint32_t sel) {
    S4 lt = fs * absDot(dirLocal, gnLocal) / dirDensity;
    return fminf(lt.importance(sel), 1.0f);
}

__device__ __forceinline__ WLS frameWls(const BptArgs &a, uint32_t flags) {
    WLS w = a.wls;
    w.single = (flags & kFlagSingle) ? 1u : 0u;
    return w;
}

// Environment "surface point" for a direction (infinite_sphere.cu:17-56).
__device__ __forceinline__ void envSurfPt(const V3 &direction, float posPhi, SurfPt* sp) {
    float sinPhi, cosPhi;
    fsincos(posPhi, &sinPhi, &cosPhi);
    V3 t0 = normalize(V3(-cosPhi, 0.0f, -sinPhi));
    sp->frame.x = t0;
    sp->frame.z = -direction;
    sp->frame.y = cross(sp->frame.z, sp->frame.x);
    sp->position = direction;
    sp->gn = -direction;
    sp->atInfinity = true;
    sp->prim = 0;
    sp->geomInst = 0;
}

__device__ __forceinline__ void storeVertex(const BptArgs &a, const SurfPt &sp, uint32_t material, const S4 &flux,
                                            const V3 &dirInLocal, float backConv, float probDensity,
                                            float prevProbDensity, float secondPrevPartial, float secondPrevRatio,
                                            bool deltaSampled, bool prevDeltaSampled, bool wlSelected,
                                            uint32_t pathLength, bool isPoint = false) {
    uint32_t slot = appendSlot(a.bb.counters, 0u);
    if (slot >= a.bb.capacity) {
        atomicAdd(a.bb.counters + 1, 1u);
        return;
    }
    uint32_t flags = (wlSelected ? 1u : 0u) | (deltaSampled ? 2u : 0u) | (prevDeltaSampled ? 4u : 0u) |
                     (sp.atInfinity ? 8u : 0u) | (isPoint ? 16u : 0u) | (pathLength << 8);
    LightVertex v;
    v.posMat = make_float4(sp.position.x, sp.position.y, sp.position.z, __uint_as_float(material));
    v.nrmFlags = make_float4(sp.frame.z.x, sp.frame.z.y, sp.frame.z.z, __uint_as_float(flags));
    v.tanGeom = make_float4(sp.frame.x.x, sp.frame.x.y, sp.frame.x.z, __uint_as_float(sp.geomInst));
    v.gnConv = make_float4(sp.gn.x, sp.gn.y, sp.gn.z, backConv);
    v.flux = toF4(flux);
    v.dirInPdf = make_float4(dirInLocal.x, dirInLocal.y, dirInLocal.z, probDensity);
    v.misPdfs = make_float4(prevProbDensity, secondPrevPartial, secondPrevRatio, 0.0f);
    v.texCoord = make_float4(sp.tu, sp.tv, 0.0f, 0.0f);
    a.bb.cache[slot] = v;
}

struct CachedVertex {
    SurfPt sp;
    uint32_t material;
    uint32_t flags;
    float backConv;
    S4 flux;
    V3 dirInLocal;
    float probDensity, prevProbDensity, secondPrevPartial, secondPrevRatio;
    bool isPoint;      // a point light's position (calcCosTerm 1)
};

__device__ __forceinline__ void loadVertex(const BptArgs &a, uint32_t i, CachedVertex* c) {
    const float4* p = reinterpret_cast<const float4*>(a.bb.cache + i);
    float4 f0 = p[0], f1 = p[1], f2 = p[2], f3 = p[3], f4 = p[4], f5 = p[5], f6 = p[6], f7 = p[7];
    c->sp.position = V3(f0.x, f0.y, f0.z);
    c->material = __float_as_uint(f0.w);
    V3 n(f1.x, f1.y, f1.z), t(f2.x, f2.y, f2.z);
    c->sp.frame = Frame(t, n);
    c->flags = __float_as_uint(f1.w);
    c->sp.geomInst = __float_as_uint(f2.w);
    c->sp.gn = V3(f3.x, f3.y, f3.z);
    c->backConv = f3.w;
    c->flux = toS4(f4);
    c->dirInLocal = V3(f5.x, f5.y, f5.z);
    c->probDensity = f5.w;
    c->prevProbDensity = f6.x;
    c->secondPrevPartial = f6.y;
    c->secondPrevRatio = f6.z;
    c->sp.atInfinity = (c->flags & 8u) != 0;
    c->sp.prim = 0;
    c->sp.tu = f7.x;
    c->sp.tv = f7.y;
    c->isPoint = (c->flags & 16u) != 0;
}

// The light vertex's scattering function: its BSDF in importance transport,
// or for y0 the EDF acting as a BSDF (materials.cu:416-470).
struct VertexBsdf {
    Bsdf bsdf;
    bool fromEdf;
    bool envEdf;
    float envDiscArea;
    uint32_t emitter;   // fromEdf: the emitter kind (kEmit*)
};

__device__ __forceinline__ bool vbHasNonDelta(const VertexBsdf &v) {
    // Diffuse, environment and point EDFs are Emission | LowFreq; a
    // directional EDF is a delta direction (materials.cu:2097-2160)
    if (v.fromEdf) return v.emitter != kEmitDirectional;
    return bsdfHasNonDelta(v.bsdf);
}

// Bidirectional BSDF wrapper evaluate / evaluatePDF (renderer_common.h:230-311).
__device__ __forceinline__ S4 vbEval(const VertexBsdf &v, const BsdfQuery &q, const V3 &ngLocal, const V3 &d,
                                     S4* rev) {
    if (!v.fromEdf) return bsdfEval(v.bsdf, q, ngLocal, d, rev);
    float sn = fabsf(q.dirLocal.z / dot(q.dirLocal, ngLocal));
    if (!isfinite(sn)) { *rev = S4::zero(); return S4::zero(); }
    *rev = S4::zero();
    return S4(edfEval(v.emitter, d)) * sn;
}
__device__ __forceinline__ float vbPdf(const VertexBsdf &v, const BsdfQuery &q, const V3 &d, float* rev) {
    if (!v.fromEdf) return bsdfPDF(v.bsdf, q, d, rev);
    *rev = 0.0f;
    if (v.emitter == kEmitPoint) return 1.0f / (4 * kPi);
    if (v.emitter == kEmitDirectional) return 0.0f;
    if (d.z <= 0.0f) return 0.0f;
    return v.envEdf ? 1.0f / v.envDiscArea : d.z / kPi;
}

// testVisibility's ray (light_transport_common.h:147-177).
__device__ __forceinline__ void visibilityRay(const SurfPt &from, const SurfPt &to, V3* dir, float* dist2, V3* org,
                                              float* tmax) {
    if (to.atInfinity) {
        *dist2 = 1.0f;
        *dir = normalize(to.position);
    }
    else {
        V3 d = to.position - from.position;
        *dist2 = d.sqLength();
        *dir = d / sqrtf(*dist2);
    }
    bool front = dot(from.gn, *dir) > 0;
    *org = offsetRayOrigin(from.position, front ? from.gn : -from.gn);
    *tmax = FLT_MAX;
    if (!to.atInfinity) {
        bool lfront = -dot(to.gn, *dir) > 0;
        V3 lp = offsetRayOrigin(to.position, lfront ? to.gn : -to.gn);
        *tmax = (lp - *org).length() * 0.9999f;
    }
}

__device__ __forceinline__ uint32_t numCached(const BptArgs &a) {
    uint32_t n = *reinterpret_cast<volatile uint32_t*>(a.bb.counters);
    return n < a.bb.capacity ? n : a.bb.capacity;
}

__device__ __forceinline__ void emitConnection(const BptArgs &a, uint32_t bounce, const V3 &org, const V3 &dir,
                                               float tmax, const S4 &c, uint32_t target) {
    uint32_t slot = appendSlot(bounceCounters(a.pb, bounce) + kCntShadow, 0u);
    ShadowRay sr;
    sr.org = make_float4(org.x, org.y, org.z, tmax);
    sr.dir = make_float4(dir.x, dir.y, dir.z, __uint_as_float(target));
    sr.contrib = toF4(c);
    a.pb.shadow[slot] = sr;
}

// ----------------------------------------------------------------- light subpaths
__global__ void __launch_bounds__(256) lightStartKernel(BptArgs a) {
    const SceneGPU &S = a.S;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.numPaths; p += gridDim.x * blockDim.x) {
        PCG32 rng{ a.pb.rng[p] };
        float uLight = rng.uniform();
        float instProb, uInst;
        uint32_t li = S.lightInsts.sample(uLight, &instProb, &uInst);
        float groupProb, uPrim;
        uint32_t g = S.instGroups[li].sample(uInst, &groupProb, &uPrim);
        const float lightProb = instProb * groupProb;
        float ue0 = rng.uniform(), ue1 = rng.uniform();
        LightSample ls;
        S4 Le0;
        bool env = static_cast<int32_t>(li) == S.envInst;
        float envDisc = S.bounds.worldDiscArea;
        if (env) {
            float uu, vv, uvPDF;
            envSampleUV(S.env, ue0, ue1, &uu, &vv, &uvPDF);
            float phi = 2 * kPi * uu, theta = kPi * vv;
            float posPhi = phi - S.envRotation;
            posPhi = posPhi - floorf(posPhi / (2 * kPi)) * 2 * kPi;
            envSurfPt(dirFromPolarYUp(posPhi, theta), posPhi, &ls.sp);
            ls.areaPDF = uvPDF / (2 * kPi * kPi * sinf(theta));
            ls.material = S.envMaterial;
            ls.delta = false;
            ls.isPoint = false;
            Le0 = kPi * envRadiance(S, uu, vv, a.wls) * S.mats[S.envMaterial].emitScale;
        }
        else {
            uint32_t grp = __ldg(S.instFirstGroup + li) + g;
            sampleTriangleGroup(S, grp, uPrim, ue0, ue1, &ls);
            Le0 = emittance(S.meng, S.mats[ls.material], a.wls);
        }
        float probDensity0 = a.numLightPaths * lightProb * ls.areaPDF;
        S4 alpha = Le0 / probDensity0;
        storeVertex(a, ls.sp, ls.material, alpha, V3(0.0f, 0.0f, 1.0f), 0.0f, probDensity0, 1.0f, 0.0f, 1.0f,
                    ls.delta, false, false, 0, ls.isPoint);
        // EDF direction sample: cosine lobe (DiffuseEDF, materials.cu:2057-2066), a
        // point on the disc that covers the scene (EnvironmentEDF, :2844-2857),
        // the whole sphere (PointEDF, :2190-2196) or the normal (DirectionalEDF,
        // :2110-2125, a delta direction)
        const uint32_t emitter = env ? kEmitEnvironment : S.mats[ls.material].emitter;
        float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
        (void)uc;
        V3 dirLocal;
        float dirPDF;
        S4 Le1(1.0f / kPi);
        uint32_t emitType = dir::Emission | dir::LowFreq;
        if (env) {
            float dx, dy;
            concentricDisk(ud0, ud1, &dx, &dy);
            dirLocal = V3(S.bounds.worldRadius * dx, S.bounds.worldRadius * dy, 1.0f);
            dirPDF = 1.0f / envDisc;
        }
        else if (emitter == kEmitPoint) {
            dirLocal = uniformSphere(ud0, ud1);
            dirPDF = 1.0f / (4 * kPi);
            Le1 = S4(1.0f / (4 * kPi));
        }
        else if (emitter == kEmitDirectional) {
            dirLocal = V3(0.0f, 0.0f, 1.0f);
            dirPDF = 1.0f;
            Le1 = S4(1.0f);
            emitType = dir::Emission | dir::Delta0D;
        }
        else {
            dirLocal = cosineHemisphere(ud0, ud1);
            dirPDF = dirLocal.z / kPi;
        }
        V3 rayOrg = offsetRayOrigin(ls.sp.position, ls.sp.gn);
        if (ls.sp.atInfinity) {
            rayOrg = S.bounds.center + 1.1f * S.bounds.worldRadius * ls.sp.position + ls.sp.frame.x * dirLocal.x +
                     ls.sp.frame.y * dirLocal.y;
            dirLocal.x = 0;
            dirLocal.y = 0;
        }
        V3 rayDir = ls.sp.frame.fromLocal(dirLocal);
        float cosTerm = ls.isPoint ? 1.0f : absDot(rayDir, ls.sp.gn);
        alpha *= Le1 * (cosTerm / dirPDF);
        a.pb.rng[p] = rng.state;
        a.pb.alpha[p] = toF4(alpha);
        a.pb.prevDirPDF[p] = dirPDF;
        a.ex.cosTerm[p] = cosTerm;
        a.ex.prevRevAreaPDF[p] = 1.0f;
        a.ex.probDensity[p] = probDensity0;
        a.ex.prevProbDensity[p] = 1.0f;
        a.ex.secondPrevPartial[p] = 0.0f;
        a.ex.secondPrevRatio[p] = 1.0f;
        a.pb.flags[p] = (ls.sp.atInfinity ? kFlagOriginInf : 0u) | (ls.delta ? kFlagPrevDelta : 0u) |
                        (ls.isPoint ? kFlagOriginPoint : 0u);
        a.pb.prevType[p] = emitType;
        a.pb.rayOrg[p] = make_float4(rayOrg.x, rayOrg.y, rayOrg.z, FLT_MAX);
        a.pb.rayDir[p] = make_float4(rayDir.x, rayDir.y, rayDir.z, 0.0f);
        a.pb.active[0][p] = p;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) bounceCounters(a.pb, 0)[kCntActive] = a.numPaths;
}

__global__ void __launch_bounds__(256) lightShadeKernel(BptArgs a) {
    const SceneGPU &S = a.S;
    uint32_t* ctr = bounceCounters(a.pb, a.bounce);
    uint32_t* next = bounceCounters(a.pb, a.bounce + 1);
    __shared__ uint32_t sOff[kNumShadeBuckets + 1];
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < kNumShadeBuckets; ++k) { sOff[k] = run; run += ctr[kCntBucket0 + k]; }
        sOff[kNumShadeBuckets] = run;
    }
    __syncthreads();
    const uint32_t total = sOff[kNumBsdfKinds];   // misses end light subpaths
    uint32_t* nextQueue = a.pb.active[(a.bounce + 1) & 1];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        uint32_t k = 0;
        while (j >= sOff[k + 1]) ++k;
        const uint32_t p = a.pb.buckets[k * a.numPaths + (j - sOff[k])];
        uint32_t flags = a.pb.flags[p];
        const uint32_t pathLength = pathLengthOf(flags) + 1;
        flags = withPathLength(flags, pathLength);
        WLS wls = frameWls(a, flags);
        float4 h = a.pb.hit[p];
        SurfPt sp;
        decodeHit(S, __float_as_uint(h.w), h.y, h.z, &sp, nullptr);
        float bsdfScale = 1.0f;
        uint32_t mat = __ldg(S.triMaterial + __float_as_uint(h.w));
        if (S.mats[mat].bsdfKind == kMultiBSDF)
            mat = bsdfMaterial(S, mat, a.pb.rng[p], __float_as_uint(h.w), &bsdfScale);
        Bsdf bsdf = buildBsdf(S.meng, S.mats[mat], wls, sp.tu, sp.tv);
        float4 o4 = a.pb.rayOrg[p], d4 = a.pb.rayDir[p];
        V3 dirInLocal = sp.frame.toLocal(-V3(d4.x, d4.y, d4.z));
        V3 gnLocal = sp.frame.toLocal(sp.gn);
        BsdfQuery q;
        q.dirLocal = dirInLocal;
        q.wlHint = wls.selected;
        q.filter = dir::All;
        q.importanceMode = 1;
        // partial MIS weight of the segment two back (lvc_bpt.cu:268-285)
        const bool prevDelta = (flags & kFlagPrevDelta) != 0;
        const bool secondPrevDelta = (flags & kFlagSecondPrevDelta) != 0;
        bool validSecondLast = (!prevDelta && !secondPrevDelta) && pathLength > 2;
        float probRatio = a.ex.prevRevAreaPDF[p] / a.ex.prevProbDensity[p];
        float secondPrevPartial = sq(probRatio) * (a.ex.secondPrevPartial[p] + (validSecondLast ? 1 : 0));
        float secondPrevRatio = a.ex.secondPrevRatio[p] * probRatio;
        float prevProbDensity = a.ex.probDensity[p];
        float lastDist2 = (V3(o4.x, o4.y, o4.z) - sp.position).sqLength();
        if (flags & kFlagOriginInf) lastDist2 = 1;
        float probDensity = a.pb.prevDirPDF[p] * absDot(dirInLocal, gnLocal) / lastDist2;
        S4 alpha = toS4(a.pb.alpha[p]) * bsdfScale;   // a Multi material's component choice
        const uint32_t sampledType = a.pb.prevType[p];
        const float cosTermIn = a.ex.cosTerm[p];
        storeVertex(a, sp, mat, alpha, dirInLocal, cosTermIn / lastDist2, probDensity, prevProbDensity,
                    secondPrevPartial, secondPrevRatio, dir::isDelta(sampledType), prevDelta,
                    (flags & kFlagSingle) != 0, pathLength);
        a.pb.flags[p] = flags;
        if (pathLength >= a.maxPathLength) continue;
        PCG32 rng{ a.pb.rng[p] };
        float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
        BsdfSample bs;
        BsdfRev rev;
        S4 fs = bsdfSample(bsdf, q, gnLocal, uc, ud0, ud1, &bs, &rev);
        if (fs.isZero() || bs.dirPDF == 0.0f) { a.pb.rng[p] = rng.state; continue; }
        if (dir::isDispersive(bs.sampledType) && !(flags & kFlagSingle)) flags |= kFlagSingle;
        float cosTerm = dot(bs.dirLocal, gnLocal);
        S4 local = fs * (fabsf(cosTerm) / bs.dirPDF);
        alpha *= local;
        float continueProb = fminf(local.importance(wls.selected), 1.0f);
        if (rng.uniform() >= continueProb) { a.pb.rng[p] = rng.state; continue; }
        a.pb.rng[p] = rng.state;
        alpha /= continueProb;
        V3 dirOut = sp.frame.fromLocal(bs.dirLocal);
        V3 org = offsetRayOrigin(sp.position, cosTerm > 0.0f ? sp.gn : -sp.gn);
        float revAreaPDF = rev.dirPDF * cosTermIn / lastDist2;
        revAreaPDF *= rrProb(rev.value, q.dirLocal, rev.dirPDF, gnLocal, wls.selected);
        if (flags & kFlagOriginPoint) revAreaPDF = 0;
        // shift the per-segment state (lvc_bpt.cu:233-240)
        uint32_t nf = flags & ~(kFlagOriginPoint | kFlagOriginInf | kFlagPrevDelta | kFlagSecondPrevDelta);
        if (prevDelta) nf |= kFlagSecondPrevDelta;
        if (dir::isDelta(sampledType)) nf |= kFlagPrevDelta;
        a.pb.flags[p] = nf;
        a.pb.alpha[p] = toF4(alpha);
        a.pb.prevDirPDF[p] = bs.dirPDF * continueProb;
        a.pb.prevType[p] = bs.sampledType;
        a.ex.cosTerm[p] = fabsf(cosTerm);
        a.ex.prevRevAreaPDF[p] = revAreaPDF;
        a.ex.probDensity[p] = probDensity;
        a.ex.prevProbDensity[p] = prevProbDensity;
        a.ex.secondPrevPartial[p] = secondPrevPartial;
        a.ex.secondPrevRatio[p] = secondPrevRatio;
        a.pb.rayOrg[p] = make_float4(org.x, org.y, org.z, FLT_MAX);
        a.pb.rayDir[p] = make_float4(dirOut.x, dirOut.y, dirOut.z, 0.0f);
        uint32_t slot = appendSlot(next + kCntActive, 0u);
        nextQueue[slot] = p;
    }
}

// ----------------------------------------------------------------- eye subpaths
// Perspective camera importance function (cameras.cu:124-224).
struct Lens {
    V3 position;
    Frame frame;
    float xOnLens, yOnLens;
};

__device__ __forceinline__ bool idfProject(const Camera &C, const Lens &L, const V3 &dirLocal, float* u0, float* u1,
                                           float* pdf) {
    return cameraProject(C, L.xOnLens, L.yOnLens, dirLocal, u0, u1, pdf);
}

// PerspectiveCamera_sample (cameras.cu:40-74): a point on the lens, its frame
// and area density.
__device__ __forceinline__ Lens sampleLens(const Camera &C, float ul0, float ul1, float* areaPDF) {
    float lx, ly;
    concentricDisk(ul0, ul1, &lx, &ly);
    Lens L;
    const V3 orgLocal(C.lensRadius * lx, C.lensRadius * ly, 0.0f);
    L.frame.z = normalize(C.forward);
    L.frame.x = normalize(C.right);
    L.frame.y = cross(L.frame.z, L.frame.x);
    L.position = C.right * orgLocal.x + C.up * orgLocal.y + C.forward * orgLocal.z + C.position;
    L.xOnLens = C.lensRadius * lx;
    L.yOnLens = C.lensRadius * ly;
    *areaPDF = C.lensRadius > 0.0f ? 1.0f / (kPi * C.lensRadius * C.lensRadius) : 1.0f;
    return L;
}

__global__ void __launch_bounds__(256) eyeStartKernel(BptArgs a) {
    const SceneGPU &S = a.S;
    const Camera &C = S.cam;
    const uint32_t nCached = numCached(a);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.numPaths; p += gridDim.x * blockDim.x) {
        const uint32_t pixel = pixelOfPath(p, a.width, a.height);
        const uint32_t px = pixel % a.width, py = pixel / a.width;
        PCG32 rng{ a.pb.rng[p] };
        float fx = px + rng.uniform(), fy = py + rng.uniform();
        const WLS wls = a.wls;
        float lx, ly;
        float l0 = rng.uniform(), l1 = rng.uniform();
        concentricDisk(l0, l1, &lx, &ly);
        Lens L;
        V3 orgLocal(C.lensRadius * lx, C.lensRadius * ly, 0.0f);
        V3 gn = normalize(C.forward);
        L.frame.z = gn;
        L.frame.x = normalize(C.right);
        L.frame.y = cross(L.frame.z, L.frame.x);
        L.position = C.right * orgLocal.x + C.up * orgLocal.y + C.forward * orgLocal.z + C.position;
        L.xOnLens = C.lensRadius * lx;
        L.yOnLens = C.lensRadius * ly;
        const bool lensDelta = !(C.lensRadius > 0.0f);
        const float areaPDF = C.lensRadius > 0.0f ? 1.0f / (kPi * C.lensRadius * C.lensRadius) : 1.0f;
        S4 We0(C.sensitivity);
        S4 alpha = We0 / (areaPDF * a.wlPdf * a.width * a.height);
        SurfPt spE;
        spE.position = L.position;
        spE.gn = gn;
        spE.frame = L.frame;
        spE.atInfinity = false;
        // t = 1: connect the lens vertex with a random cached light vertex
        if (nCached > 0) {
            uint32_t vi = vmin<uint32_t>(static_cast<uint32_t>(nCached * rng.uniform()), nCached - 1);
            float vertexProb = 1.0f / nCached;
            CachedVertex v;
            loadVertex(a, vi, &v);
            const uint32_t vPathLength = (v.flags >> 8) & 0xFFFFu;
            VertexBsdf vb;
            vb.fromEdf = vPathLength == 0;
            vb.envEdf = v.sp.atInfinity;
            vb.envDiscArea = S.bounds.worldDiscArea;
            vb.emitter = S.mats[v.material].emitter;
            if (!vb.fromEdf) vb.bsdf = buildBsdf(S.meng, S.mats[v.material], wls, v.sp.tu, v.sp.tv);
            V3 conDir, sOrg;
            float dist2, tmax;
            visibilityRay(spE, v.sp, &conDir, &dist2, &sOrg, &tmax);
            if (vbHasNonDelta(vb)) {
                float recSq = 1.0f / dist2;
                V3 gnLocalL = v.sp.frame.toLocal(v.sp.gn);
                BsdfQuery qL;
                qL.dirLocal = v.dirInLocal;
                qL.wlHint = wls.selected;
                qL.filter = dir::All;
                qL.importanceMode = 1;
                V3 conLocalL = v.sp.frame.toLocal(-conDir);
                V3 conLocalE = L.frame.toLocal(conDir);
                float cosL = v.isPoint ? 1.0f : absDot(conDir, v.sp.gn);
                float cosE = lensCos(C, conDir, gn);
                float G = cosL * cosE * recSq;
                float scalarConTerm = G / vertexProb;
                if (v.flags & 1u) scalarConTerm *= kNumLambdas;
                S4 backFsL;
                S4 fwdFsL = vbEval(vb, qL, gnLocalL, conLocalL, &backFsL);
                float backDirDensL;
                vbPdf(vb, qL, conLocalL, &backDirDensL);
                backDirDensL *= rrProb(backFsL, qL.dirLocal, backDirDensL, gnLocalL, wls.selected);
                float backAreaDensL = backDirDensL * v.backConv;
                if (v.flags & 4u) backAreaDensL = 0;
                float u0, u1, fwdDirDensE;
                bool onScreen = idfProject(C, L, conLocalE, &u0, &u1, &fwdDirDensE);
                if (onScreen) {
                    float fwdAreaDensE = fwdDirDensE * cosL * recSq;
                    if (v.isPoint) fwdAreaDensE = 0;   // a delta position cannot be hit (lvc_bpt.cu:430-431)
                    bool lastValid = (!(v.flags & 2u) && !(v.flags & 4u)) && vPathLength > 1;
                    float lastToSecondLast = backAreaDensL / v.prevProbDensity;
                    float partialL = sq(lastToSecondLast) * (v.secondPrevPartial + (lastValid ? 1 : 0));
                    float ratioToFirst = v.secondPrevRatio;
                    if (vPathLength > 0) ratioToFirst *= lastToSecondLast;
                    bool curValid = !(v.flags & 2u) && vPathLength > 0;
                    float curToLast = fwdAreaDensE / v.probDensity;
                    partialL = sq(curToLast) * (partialL + (curValid ? 1 : 0));
                    ratioToFirst *= curToLast;
                    partialL += sq(ratioToFirst / vertexProb);
                    S4 conTerm = fwdFsL * scalarConTerm * S4::one();
                    S4 unweighted = v.flux * conTerm * alpha;
                    float mis = 1.0f / (1.0f + partialL);
                    S4 c = mis * unweighted;
                    uint32_t ipx = static_cast<uint32_t>(u0 * a.width), ipy = static_cast<uint32_t>(u1 * a.height);
                    if (c.allFinite() && c.hasNonZero() && ipx < a.width && ipy < a.height)
                        emitConnection(a, 0, sOrg, conDir, tmax, c, kSplatBit | (ipy * a.stride + ipx));
                }
            }
        }
        // camera ray (lvc_bpt.cu:481-503)
        float u0 = fx / a.width, u1 = fy / a.height;
        float dirPDF;
        V3 dirLocal = cameraSampleDir(C, orgLocal.x, orgLocal.y, u0, u1, &dirPDF);
        V3 rayDir = L.frame.fromLocal(dirLocal);
        float cosTerm = lensCos(C, rayDir, gn);
        alpha *= S4::one() * (cosTerm / dirPDF);
        a.pb.rng[p] = rng.state;
        a.pb.alpha[p] = toF4(alpha);
        a.pb.contrib[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        a.pb.prevDirPDF[p] = dirPDF;
        a.pb.prevType[p] = dir::Acquisition | dir::LowFreq;
        a.pb.flags[p] = lensDelta ? kFlagPrevDelta : 0u;
        a.ex.cosTerm[p] = cosTerm;
        a.ex.prevRevAreaPDF[p] = 1.0f;
        a.ex.probDensity[p] = areaPDF;
        a.ex.prevProbDensity[p] = 1.0f;
        a.ex.secondPrevPartial[p] = 0.0f;
        a.pb.rayOrg[p] = make_float4(L.position.x, L.position.y, L.position.z, FLT_MAX);
        a.pb.rayDir[p] = make_float4(rayDir.x, rayDir.y, rayDir.z, 0.0f);
        a.pb.active[0][p] = p;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) bounceCounters(a.pb, 0)[kCntActive] = a.numPaths;
}

// MIS denominator terms on the eye side for a vertex that ends the eye
// subpath by hitting an emitter (lvc_bpt.cu:636-659, 935-958).
__device__ __forceinline__ float eyeImplicitPartial(float backAreaDensE, float prevProbDensity, float secondPrevPartial,
                                                    float probDensity, float fwdAreaDensL, bool lastValid,
                                                    bool curValid, float vertexProb) {
    float lastToSecondLast = backAreaDensE / prevProbDensity;
    float pe = sq(lastToSecondLast) * (secondPrevPartial + (lastValid ? 1 : 0));
    float curToLast = fwdAreaDensL / probDensity;
    pe = sq(curToLast) * (pe + (curValid ? 1 : 0));
    return pe * sq(vertexProb);
}

__global__ void __launch_bounds__(256) eyeShadeKernel(BptArgs a) {
    const SceneGPU &S = a.S;
    uint32_t* ctr = bounceCounters(a.pb, a.bounce);
    uint32_t* next = bounceCounters(a.pb, a.bounce + 1);
    __shared__ uint32_t sOff[kNumShadeBuckets + 1];
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < kNumShadeBuckets; ++k) { sOff[k] = run; run += ctr[kCntBucket0 + k]; }
        sOff[kNumShadeBuckets] = run;
    }
    __syncthreads();
    const uint32_t total = sOff[kNumShadeBuckets];
    const uint32_t nCached = numCached(a);
    const float vertexProb = nCached > 0 ? 1.0f / nCached : 0.0f;
    uint32_t* nextQueue = a.pb.active[(a.bounce + 1) & 1];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        uint32_t k = 0;
        while (j >= sOff[k + 1]) ++k;
        const uint32_t p = a.pb.buckets[k * a.numPaths + (j - sOff[k])];
        uint32_t flags = a.pb.flags[p];
        const uint32_t pathLength = pathLengthOf(flags) + 1;
        flags = withPathLength(flags, pathLength);
        a.pb.flags[p] = flags;
        WLS wls = frameWls(a, flags);
        const bool prevDelta = (flags & kFlagPrevDelta) != 0;
        const bool secondPrevDelta = (flags & kFlagSecondPrevDelta) != 0;
        const uint32_t sampledType = a.pb.prevType[p];
        const float cosTermIn = a.ex.cosTerm[p];
        bool validSecondLast = (!prevDelta && !secondPrevDelta) && pathLength > 2;
        float secondPrevPartial = sq(a.ex.prevRevAreaPDF[p] / a.ex.prevProbDensity[p]) *
                                  (a.ex.secondPrevPartial[p] + (validSecondLast ? 1 : 0));
        float prevProbDensity = a.ex.probDensity[p];
        S4 alpha = toS4(a.pb.alpha[p]);
        S4 contrib = toS4(a.pb.contrib[p]);
        float4 o4 = a.pb.rayOrg[p], d4 = a.pb.rayDir[p];
        V3 rayDir(d4.x, d4.y, d4.z);
        if (k == kNumBsdfKinds) {
            // environment (lvc_bpt.cu:841-971)
            if (S.envInst >= 0) {
                float probDensity = a.pb.prevDirPDF[p] / 1.0f;
                float theta, posPhi;
                toPolarYUp(rayDir, &theta, &posPhi);
                float phi = posPhi + S.envRotation;
                phi = phi - floorf(phi / (2 * kPi)) * 2 * kPi;
                float tu = phi / (2 * kPi), tv = theta / kPi;
                float uvPDF = envPdfUV(S.env, tu, tv);
                float hypAreaPDF = uvPDF / (2 * kPi * kPi * sinf(theta));
                S4 spEm = kPi * envRadiance(S, tu, tv, wls) * S.mats[S.envMaterial].emitScale;
                if (spEm.hasNonZero()) {
                    S4 Le = spEm * (1.0f / kPi);
                    S4 unweighted = alpha * Le;
                    if (flags & kFlagSingle) unweighted *= static_cast<float>(kNumLambdas);
                    float fwdAreaDensL = a.numLightPaths * S.envLightProb * hypAreaPDF;
                    float backAreaDensE = (1.0f / S.bounds.worldDiscArea) * cosTermIn / 1.0f;
                    float pe = eyeImplicitPartial(backAreaDensE, prevProbDensity, secondPrevPartial, probDensity,
                                                  fwdAreaDensL, !dir::isDelta(sampledType) && !prevDelta && pathLength > 1,
                                                  !dir::isDelta(sampledType), vertexProb);
                    S4 c = (1.0f / (1.0f + pe)) * unweighted;
                    if (c.allFinite()) contrib += c;
                }
            }
            a.pb.contrib[p] = toF4(contrib);
            continue;
        }
        float4 h = a.pb.hit[p];
        SurfPt sp;
        float hypAreaPDF;
        decodeHit(S, __float_as_uint(h.w), h.y, h.z, &sp, &hypAreaPDF);
        const uint32_t matIndex = __ldg(S.triMaterial + __float_as_uint(h.w));
        const MatDesc &mat = S.mats[matIndex];
        float bsdfScale = 1.0f;
        const uint32_t bsdfIndex = mat.bsdfKind == kMultiBSDF
                                       ? bsdfMaterial(S, matIndex, a.pb.rng[p], __float_as_uint(h.w), &bsdfScale)
                                       : matIndex;
        Bsdf bsdfE = buildBsdf(S.meng, S.mats[bsdfIndex], wls, sp.tu, sp.tv);
        V3 dirOutLocal = sp.frame.toLocal(-rayDir);
        V3 gnLocal = sp.frame.toLocal(sp.gn);
        BsdfQuery qE;
        qE.dirLocal = dirOutLocal;
        qE.wlHint = wls.selected;
        qE.filter = dir::All;
        qE.importanceMode = 0;
        float lastDist2 = (V3(o4.x, o4.y, o4.z) - sp.position).sqLength();
        float probDensity = a.pb.prevDirPDF[p] * absDot(dirOutLocal, gnLocal) / lastDist2;
        // s = 0: implicit light sampling (lvc_bpt.cu:611-670)
        S4 spEm = emittance(S.meng, mat, wls);
        if (spEm.hasNonZero()) {
            S4 Le = spEm * edfEval(mat.emitter, dirOutLocal);
            S4 unweighted = alpha * Le;
            if (flags & kFlagSingle) unweighted *= static_cast<float>(kNumLambdas);
            float fwdAreaDensL = a.numLightPaths * __ldg(S.geomLightPdfArea + sp.geomInst) * hypAreaPDF;
            float backAreaDensE = diffuseEdfPDF(dirOutLocal) * cosTermIn / lastDist2;
            float pe = eyeImplicitPartial(backAreaDensE, prevProbDensity, secondPrevPartial, probDensity, fwdAreaDensL,
                                          !dir::isDelta(sampledType) && !prevDelta && pathLength > 1,
                                          !dir::isDelta(sampledType), vertexProb);
            S4 c = (1.0f / (1.0f + pe)) * unweighted;
            if (c.allFinite()) contrib += c;
        }
        a.pb.contrib[p] = toF4(contrib);
        alpha *= bsdfScale;   // a Multi material's component choice (after the emission)
        PCG32 rng{ a.pb.rng[p] };
        // connection to one random cached light vertex (lvc_bpt.cu:672-803)
        if (bsdfHasNonDelta(bsdfE) && nCached > 0) {
            uint32_t vi = vmin<uint32_t>(static_cast<uint32_t>(nCached * rng.uniform()), nCached - 1);
            CachedVertex v;
            loadVertex(a, vi, &v);
            const uint32_t vPathLength = (v.flags >> 8) & 0xFFFFu;
            VertexBsdf vb;
            vb.fromEdf = vPathLength == 0;
            vb.envEdf = v.sp.atInfinity;
            vb.envDiscArea = S.bounds.worldDiscArea;
            vb.emitter = S.mats[v.material].emitter;
            if (!vb.fromEdf) vb.bsdf = buildBsdf(S.meng, S.mats[v.material], wls, v.sp.tu, v.sp.tv);
            V3 conDir, sOrg;
            float dist2, tmax;
            visibilityRay(sp, v.sp, &conDir, &dist2, &sOrg, &tmax);
            if (vbHasNonDelta(vb)) {
                float recSq = 1.0f / dist2;
                V3 gnLocalL = v.sp.frame.toLocal(v.sp.gn);
                BsdfQuery qL;
                qL.dirLocal = v.dirInLocal;
                qL.wlHint = wls.selected;
                qL.filter = dir::All;
                qL.importanceMode = 1;
                V3 conLocalL = v.sp.frame.toLocal(-conDir);
                V3 conLocalE = sp.frame.toLocal(conDir);
                float cosL = v.isPoint ? 1.0f : absDot(conDir, v.sp.gn);
                float cosE = absDot(conDir, sp.gn);
                float G = cosL * cosE * recSq;
                float scalarConTerm = G / vertexProb;
                if ((v.flags & 1u) || (flags & kFlagSingle)) scalarConTerm *= kNumLambdas;
                S4 backFsL;
                S4 fwdFsL = vbEval(vb, qL, gnLocalL, conLocalL, &backFsL);
                float backDirDensL;
                float fwdDirDensL = vbPdf(vb, qL, conLocalL, &backDirDensL);
                if (vPathLength > 0) fwdDirDensL *= rrProb(fwdFsL, conLocalL, fwdDirDensL, gnLocalL, wls.selected);
                backDirDensL *= rrProb(backFsL, qL.dirLocal, backDirDensL, gnLocalL, wls.selected);
                float fwdAreaDensL = fwdDirDensL * cosE * recSq;
                float backAreaDensL = backDirDensL * v.backConv;
                if (v.flags & 4u) backAreaDensL = 0;
                S4 backFsE;
                S4 fwdFsE = bsdfEval(bsdfE, qE, gnLocal, conLocalE, &backFsE);
                float backDirDensE;
                float fwdDirDensE = bsdfPDF(bsdfE, qE, conLocalE, &backDirDensE);
                fwdDirDensE *= rrProb(fwdFsE, conLocalE, fwdDirDensE, gnLocal, wls.selected);
                backDirDensE *= rrProb(backFsE, qE.dirLocal, backDirDensE, gnLocal, wls.selected);
                float fwdAreaDensE = fwdDirDensE * cosL * recSq;
                if (v.isPoint) fwdAreaDensE = 0;       // a delta position cannot be hit (lvc_bpt.cu:738-739)
                float backAreaDensE = backDirDensE * cosTermIn / lastDist2;
                float partialL;
                {
                    bool lastValid = (!(v.flags & 2u) && !(v.flags & 4u)) && vPathLength > 1;
                    float lastToSecondLast = backAreaDensL / v.prevProbDensity;
                    partialL = sq(lastToSecondLast) * (v.secondPrevPartial + (lastValid ? 1 : 0));
                    float ratioToFirst = v.secondPrevRatio;
                    if (vPathLength > 0) ratioToFirst *= lastToSecondLast;
                    bool curValid = !(v.flags & 2u) && vPathLength > 0;
                    float curToLast = fwdAreaDensE / v.probDensity;
                    partialL = sq(curToLast) * (partialL + (curValid ? 1 : 0));
                    ratioToFirst *= curToLast;
                    partialL += sq(ratioToFirst / vertexProb);
                }
                float partialE;
                {
                    bool lastValid = !dir::isDelta(sampledType) && !prevDelta;
                    float lastToSecondLast = backAreaDensE / prevProbDensity;
                    partialE = sq(lastToSecondLast) * (secondPrevPartial + (lastValid ? 1 : 0));
                    bool curValid = !dir::isDelta(sampledType);
                    float curToLast = fwdAreaDensL / probDensity;
                    partialE = sq(curToLast) * (partialE + (curValid ? 1 : 0));
                }
                S4 conTerm = fwdFsL * scalarConTerm * fwdFsE;
                S4 unweighted = v.flux * conTerm * alpha;
                float mis = 1.0f / (1.0f + partialL + partialE);
                S4 c = mis * unweighted;
                if (c.allFinite() && c.hasNonZero()) emitConnection(a, a.bounce + 1, sOrg, conDir, tmax, c, p);
            }
        }
        if (pathLength >= a.maxPathLength) { a.pb.rng[p] = rng.state; continue; }
        float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
        BsdfSample bs;
        BsdfRev rev;
        S4 fs = bsdfSample(bsdfE, qE, gnLocal, uc, ud0, ud1, &bs, &rev);
        if (fs.isZero() || bs.dirPDF == 0.0f) { a.pb.rng[p] = rng.state; continue; }
        if (dir::isDispersive(bs.sampledType) && !(flags & kFlagSingle)) flags |= kFlagSingle;
        float cosTerm = dot(bs.dirLocal, gnLocal);
        S4 local = fs * (fabsf(cosTerm) / bs.dirPDF);
        alpha *= local;
        float continueProb = fminf(local.importance(wls.selected), 1.0f);
        if (rng.uniform() >= continueProb) { a.pb.rng[p] = rng.state; continue; }
        a.pb.rng[p] = rng.state;
        alpha /= continueProb;
        V3 dirIn = sp.frame.fromLocal(bs.dirLocal);
        V3 org = offsetRayOrigin(sp.position, cosTerm > 0.0f ? sp.gn : -sp.gn);
        float revAreaPDF = rev.dirPDF * cosTermIn / lastDist2;
        revAreaPDF *= rrProb(rev.value, qE.dirLocal, rev.dirPDF, gnLocal, wls.selected);
        uint32_t nf = flags & ~(kFlagPrevDelta | kFlagSecondPrevDelta);
        if (prevDelta) nf |= kFlagSecondPrevDelta;
        if (dir::isDelta(sampledType)) nf |= kFlagPrevDelta;
        a.pb.flags[p] = nf;
        a.pb.alpha[p] = toF4(alpha);
        a.pb.prevDirPDF[p] = bs.dirPDF * continueProb;
        a.pb.prevType[p] = bs.sampledType;
        a.ex.cosTerm[p] = fabsf(cosTerm);
        a.ex.prevRevAreaPDF[p] = revAreaPDF;
        a.ex.probDensity[p] = probDensity;
        a.ex.prevProbDensity[p] = prevProbDensity;
        a.ex.secondPrevPartial[p] = secondPrevPartial;
        a.pb.rayOrg[p] = make_float4(org.x, org.y, org.z, FLT_MAX);
        a.pb.rayDir[p] = make_float4(dirIn.x, dirIn.y, dirIn.z, 0.0f);
        uint32_t slot = appendSlot(next + kCntActive, 0u);
        nextQueue[slot] = p;
    }
}

// Connection rays: visible ones add to their eye path, or splat to the pixel
// they project to (t = 1).
__global__ void __launch_bounds__(256) connectKernel(BptArgs a) {
    const uint32_t n = bounceCounters(a.pb, a.bounce)[kCntShadow];
    const float lam[4] = { a.wls.lambda[0], a.wls.lambda[1], a.wls.lambda[2], a.wls.lambda[3] };
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        ShadowRay sr = a.pb.shadow[i];
        const float vis = shadowVisibility(a.S, V3(sr.org.x, sr.org.y, sr.org.z), V3(sr.dir.x, sr.dir.y, sr.dir.z),
                                           sr.org.w);
        if (vis == 0.0f) continue;
        uint32_t target = __float_as_uint(sr.dir.w);
        if (target & kSplatBit) {
            uint32_t pixel = target & ~kSplatBit;
            filmAdd(a.film.strata + static_cast<size_t>(pixel) * kNumStrata, lam, vis * toS4(sr.contrib));
        }
        else {
            float4 c = a.pb.contrib[target];
            c.x += vis * sr.contrib.x; c.y += vis * sr.contrib.y; c.z += vis * sr.contrib.z; c.w += vis * sr.contrib.w;
            a.pb.contrib[target] = c;
        }
    }
}

__global__ void __launch_bounds__(256) eyeFilmKernel(BptArgs a) {
    const float lam[4] = { a.wls.lambda[0], a.wls.lambda[1], a.wls.lambda[2], a.wls.lambda[3] };
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.numPaths; p += gridDim.x * blockDim.x) {
        S4 c = toS4(a.pb.contrib[p]);
        if (!c.allFinite()) continue;
        const uint32_t pixel = pixelOfPath(p, a.width, a.height);
        const uint32_t fi = (pixel / a.width) * a.stride + pixel % a.width;
        filmAdd(a.film.strata + static_cast<size_t>(fi) * kNumStrata, lam, c);
    }
}

// ----------------------------------------------------------------- light tracing
// One light subpath per slot with wavelength samples of its own; the light
// point and every scattering vertex connect to a lens sample and splat what
// they send there to the pixel it projects to (light_tracing.cu:49-263).
// Connections of one stage are traced and splatted before the next stage.
struct LtConnection {
    float4 org;       // xyz, tmax
    float4 dir;       // xyz, pixel (bits)
    float4 contrib;
    float4 lambda;    // the path's wavelengths
};

// Connection from lens sample L to vertex sp (testVisibility from the lens,
// light_transport_common.h:147-177): false when the direction misses the
// frame; else the ray, the pixel, the vertex-side direction in its shading
// frame and G / lensPDF with G = cos(vertex, geometric) cos(lens) / d^2.
__device__ __forceinline__ bool lensConnection(const Camera &C, const Lens &L, float lensAreaPDF, const SurfPt &sp,
                                               bool vertexIsPoint, uint32_t W, uint32_t H, uint32_t stride, V3* dir,
                                               V3* org, float* tmax, uint32_t* pixel, V3* dirAtVertex,
                                               float* scalar) {
    SurfPt spE;
    spE.position = L.position;
    spE.gn = L.frame.z;
    spE.frame = L.frame;
    spE.atInfinity = false;
    float dist2;
    visibilityRay(spE, sp, dir, &dist2, org, tmax);
    const V3 dLens = L.frame.toLocal(*dir);
    float u0, u1, pdf;
    if (!idfProject(C, L, dLens, &u0, &u1, &pdf)) return false;
    const uint32_t ipx = static_cast<uint32_t>(u0 * W), ipy = static_cast<uint32_t>(u1 * H);
    if (ipx >= W || ipy >= H) return false;
    *pixel = ipy * stride + ipx;
    *dirAtVertex = sp.frame.toLocal(-*dir);
    *scalar = (vertexIsPoint ? 1.0f : absDot(*dir, sp.gn)) * lensCos(C, *dir, L.frame.z) / dist2 / lensAreaPDF;
    return true;
}

__device__ __forceinline__ void emitLensConnection(const BptArgs &a, uint32_t stage, const V3 &org, const V3 &dir,
                                                   float tmax, uint32_t pixel, const S4 &c, const WLS &wls) {
    const uint32_t slot = appendSlot(bounceCounters(a.pb, stage) + kCntShadow, 0u);
    if (slot >= a.numPaths) return;
    LtConnection k;
    k.org = make_float4(org.x, org.y, org.z, tmax);
    k.dir = make_float4(dir.x, dir.y, dir.z, __uint_as_float(pixel));
    k.contrib = toF4(c);
    k.lambda = make_float4(wls.lambda[0], wls.lambda[1], wls.lambda[2], wls.lambda[3]);
    a.conn[slot] = k;
}

__global__ void __launch_bounds__(256) ltStartKernel(BptArgs a) {
    const SceneGPU &S = a.S;
    const Camera &C = S.cam;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.numPaths; p += gridDim.x * blockDim.x) {
        PCG32 rng{ a.pb.rng[p] };
        float selectWLPDF;
        const float wo = rng.uniform(), ws = rng.uniform();
        const WLS wls = WLS::equalOffsets(wo, ws, &selectWLPDF);
        float uLight = rng.uniform();
        float instProb, uInst;
        uint32_t li = S.lightInsts.sample(uLight, &instProb, &uInst);
        float groupProb, uPrim;
        uint32_t g = S.instGroups[li].sample(uInst, &groupProb, &uPrim);
        const float lightProb = instProb * groupProb;
        float ue0 = rng.uniform(), ue1 = rng.uniform();
        LightSample ls;
        S4 Le0;
        const bool env = static_cast<int32_t>(li) == S.envInst;
        if (env) {
            float uu, vv, uvPDF;
            envSampleUV(S.env, ue0, ue1, &uu, &vv, &uvPDF);
            float phi = 2 * kPi * uu, theta = kPi * vv;
            float posPhi = phi - S.envRotation;
            posPhi = posPhi - floorf(posPhi / (2 * kPi)) * 2 * kPi;
            envSurfPt(dirFromPolarYUp(posPhi, theta), posPhi, &ls.sp);
            ls.areaPDF = uvPDF / (2 * kPi * kPi * sinf(theta));
            ls.material = S.envMaterial;
            ls.delta = false;
            ls.isPoint = false;
            Le0 = kPi * envRadiance(S, uu, vv, wls) * S.mats[S.envMaterial].emitScale;
        }
        else {
            uint32_t grp = __ldg(S.instFirstGroup + li) + g;
            sampleTriangleGroup(S, grp, uPrim, ue0, ue1, &ls);
            Le0 = emittance(S.meng, S.mats[ls.material], wls);
        }
        const uint32_t emitter = S.mats[ls.material].emitter;
        S4 alpha = Le0 / (a.numLightPaths * lightProb * ls.areaPDF * selectWLPDF);
        // explicit lens sampling from the light point (light_tracing.cu:70-106)
        {
            float lensPDF;
            const Lens L = sampleLens(C, rng.uniform(), rng.uniform(), &lensPDF);
            V3 dir, org, dv;
            float tmax, scalar;
            uint32_t pixel;
            if (lensConnection(C, L, lensPDF, ls.sp, ls.isPoint, a.width, a.height, a.stride, &dir, &org, &tmax,
                               &pixel, &dv, &scalar)) {
                const S4 Le1(edfEval(emitter, dv));
                const S4 c = alpha * S4(C.sensitivity) * Le1 * scalar;
                if (c.allFinite() && c.hasNonZero()) emitLensConnection(a, 0, org, dir, tmax, pixel, c, wls);
            }
        }
        // emission direction: the EDF's sample (materials.cu:2057-2066 diffuse,
        // :2110-2125 directional, :2190-2196 point, :2844-2857 environment)
        float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
        (void)uc;
        V3 dirLocal;
        float dirPDF;
        float feValue = 1.0f / kPi;
        if (env) {
            float dx, dy;
            concentricDisk(ud0, ud1, &dx, &dy);
            dirLocal = V3(S.bounds.worldRadius * dx, S.bounds.worldRadius * dy, 1.0f);
            dirPDF = 1.0f / S.bounds.worldDiscArea;
        }
        else if (emitter == kEmitPoint) {
            dirLocal = uniformSphere(ud0, ud1);
            dirPDF = 1.0f / (4 * kPi);
            feValue = 1.0f / (4 * kPi);
        }
        else if (emitter == kEmitDirectional) {
            dirLocal = V3(0.0f, 0.0f, 1.0f);
            dirPDF = 1.0f;
            feValue = 1.0f;
        }
        else {
            dirLocal = cosineHemisphere(ud0, ud1);
            dirPDF = dirLocal.z / kPi;
        }
        V3 rayOrg = offsetRayOrigin(ls.sp.position, ls.sp.gn);
        if (ls.sp.atInfinity) {
            rayOrg = S.bounds.center + 1.1f * S.bounds.worldRadius * ls.sp.position + ls.sp.frame.x * dirLocal.x +
                     ls.sp.frame.y * dirLocal.y;
            dirLocal.x = 0;
            dirLocal.y = 0;
        }
        const V3 rayDir = ls.sp.frame.fromLocal(dirLocal);
        alpha *= S4(feValue) * ((ls.isPoint ? 1.0f : absDot(rayDir, ls.sp.gn)) / dirPDF);
        a.pb.rng[p] = rng.state;
        a.pb.alpha[p] = toF4(alpha);
        a.pb.lambda[p] = make_float4(wls.lambda[0], wls.lambda[1], wls.lambda[2], wls.lambda[3]);
        a.pb.flags[p] = wls.selected;
        a.pb.initImportance[p] = alpha.importance(wls.selected);
        a.pb.rayOrg[p] = make_float4(rayOrg.x, rayOrg.y, rayOrg.z, FLT_MAX);
        a.pb.rayDir[p] = make_float4(rayDir.x, rayDir.y, rayDir.z, 0.0f);
        a.pb.active[0][p] = p;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) bounceCounters(a.pb, 0)[kCntActive] = a.numPaths;
}

// One scattering vertex of every live light subpath (lightTracingIteration,
// light_tracing.cu:186-263, and the Russian roulette of its caller, :159-163).
__global__ void __launch_bounds__(256) ltShadeKernel(BptArgs a) {
    const SceneGPU &S = a.S;
    const Camera &C = S.cam;
    uint32_t* ctr = bounceCounters(a.pb, a.bounce);
    uint32_t* next = bounceCounters(a.pb, a.bounce + 1);
    __shared__ uint32_t sOff[kNumShadeBuckets + 1];
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < kNumShadeBuckets; ++k) { sOff[k] = run; run += ctr[kCntBucket0 + k]; }
        sOff[kNumShadeBuckets] = run;
    }
    __syncthreads();
    const uint32_t total = sOff[kNumBsdfKinds];   // misses end light subpaths
    uint32_t* nextQueue = a.pb.active[(a.bounce + 1) & 1];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < total; j += gridDim.x * blockDim.x) {
        uint32_t k = 0;
        while (j >= sOff[k + 1]) ++k;
        const uint32_t p = a.pb.buckets[k * a.numPaths + (j - sOff[k])];
        uint32_t flags = a.pb.flags[p];
        const uint32_t traced = ((flags >> 8) & 0xFFFFu) + 1;
        const float4 l4 = a.pb.lambda[p];
        WLS wls;
        wls.lambda[0] = l4.x; wls.lambda[1] = l4.y; wls.lambda[2] = l4.z; wls.lambda[3] = l4.w;
        wls.selected = flags & 0xFu;
        wls.single = (flags >> 4) & 1u;
        const float4 h = a.pb.hit[p];
        SurfPt sp;
        decodeHit(S, __float_as_uint(h.w), h.y, h.z, &sp, nullptr);
        float bsdfScale = 1.0f;
        uint32_t mat = __ldg(S.triMaterial + __float_as_uint(h.w));
        if (S.mats[mat].bsdfKind == kMultiBSDF)
            mat = bsdfMaterial(S, mat, a.pb.rng[p], __float_as_uint(h.w), &bsdfScale);
        const Bsdf bsdf = buildBsdf(S.meng, S.mats[mat], wls, sp.tu, sp.tv);
        const float4 d4 = a.pb.rayDir[p];
        BsdfQuery q;
        q.dirLocal = sp.frame.toLocal(-V3(d4.x, d4.y, d4.z));
        q.wlHint = wls.selected;
        q.filter = dir::All;
        q.importanceMode = 1;
        const V3 gnLocal = sp.frame.toLocal(sp.gn);
        S4 alpha = toS4(a.pb.alpha[p]) * bsdfScale;   // a Multi material's component choice
        PCG32 rng{ a.pb.rng[p] };
        if (bsdfHasNonDelta(bsdf)) {
            float lensPDF;
            const Lens L = sampleLens(C, rng.uniform(), rng.uniform(), &lensPDF);
            V3 dir, org, dv;
            float tmax, scalar;
            uint32_t pixel;
            if (lensConnection(C, L, lensPDF, sp, false, a.width, a.height, a.stride, &dir, &org, &tmax, &pixel,
                               &dv, &scalar)) {
                const S4 fs = bsdfEval(bsdf, q, gnLocal, dv, nullptr);
                const S4 c = alpha * S4(C.sensitivity) * fs * scalar;
                if (c.allFinite() && c.hasNonZero())
                    emitLensConnection(a, a.bounce + 1, org, dir, tmax, pixel, c, wls);
            }
        }
        float uc = rng.uniform(), ud0 = rng.uniform(), ud1 = rng.uniform();
        BsdfSample bs;
        const S4 fs = bsdfSample(bsdf, q, gnLocal, uc, ud0, ud1, &bs, nullptr);
        if (fs.isZero() || !(bs.dirPDF > 0.0f)) { a.pb.rng[p] = rng.state; continue; }
        if (dir::isDispersive(bs.sampledType) && !wls.single) {
            bs.dirPDF /= kNumLambdas;
            flags |= 0x10u;
        }
        const float cosFactor = dot(bs.dirLocal, gnLocal);
        alpha *= fs * (fabsf(cosFactor) / bs.dirPDF);
        const float continueProb = fminf(alpha.importance(wls.selected) / a.pb.initImportance[p], 1.0f);
        const bool survive = rng.uniform() < continueProb;
        a.pb.rng[p] = rng.state;
        if (!survive || traced + 1 >= a.maxPathLength) continue;
        alpha /= continueProb;
        const V3 dirOut = sp.frame.fromLocal(bs.dirLocal);
        const V3 org = offsetRayOrigin(sp.position, cosFactor > 0.0f ? sp.gn : -sp.gn);
        a.pb.flags[p] = (flags & 0xFFu) | (traced << 8);
        a.pb.alpha[p] = toF4(alpha);
        a.pb.rayOrg[p] = make_float4(org.x, org.y, org.z, FLT_MAX);
        a.pb.rayDir[p] = make_float4(dirOut.x, dirOut.y, dirOut.z, 0.0f);
        const uint32_t slot = appendSlot(next + kCntActive, 0u);
        nextQueue[slot] = p;
    }
}

// Traces one stage's lens connections and splats the unoccluded ones.
__global__ void __launch_bounds__(256) ltSplatKernel(BptArgs a, uint32_t stage) {
    const uint32_t n = min(bounceCounters(a.pb, stage)[kCntShadow], a.numPaths);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const LtConnection k = a.conn[i];
        const float vis = shadowVisibility(a.S, V3(k.org.x, k.org.y, k.org.z), V3(k.dir.x, k.dir.y, k.dir.z), k.org.w);
        if (vis == 0.0f) continue;
        const uint32_t pixel = __float_as_uint(k.dir.w);
        if (pixel >= a.stride * a.height) continue;
        const float lam[4] = { k.lambda.x, k.lambda.y, k.lambda.z, k.lambda.w };
        filmAdd(a.film.strata + static_cast<size_t>(pixel) * kNumStrata, lam, vis * toS4(k.contrib));
    }
}

__global__ void bptStatsKernel(PathBuffers pb, uint32_t bounces) {
    unsigned long long seg = 0, sh = 0;
    for (uint32_t b = threadIdx.x; b <= bounces; b += 32) {
        seg += bounceCounters(pb, b)[kCntActive];
        sh += bounceCounters(pb, b)[kCntShadow];
    }
    for (int off = 16; off > 0; off >>= 1) {
        seg += __shfl_xor_sync(0xFFFFFFFFu, seg, off);
        sh += __shfl_xor_sync(0xFFFFFFFFu, sh, off);
    }
    if (threadIdx.x == 0) { pb.totals[0] += seg; pb.totals[1] += sh; }
}

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("bpt ") + what + ": " + cudaGetErrorString(e));
}

inline size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

size_t extraBytes(uint32_t n) { return 6 * a256(size_t(n) * 4); }

void carveExtra(char*& s, uint32_t n, BptExtra* e) {
    float** f[6] = { &e->probDensity, &e->prevProbDensity, &e->secondPrevPartial, &e->secondPrevRatio,
                     &e->cosTerm, &e->prevRevAreaPDF };
    for (auto p : f) { *p = reinterpret_cast<float*>(s); s += a256(size_t(n) * 4); }
}

} // namespace

size_t bptBufferBytes(uint32_t numLightPaths, uint32_t numEyePaths, uint32_t cacheCapacity) {
    return pathBufferBytes(numLightPaths) + a256(size_t(cacheCapacity) * sizeof(LightVertex)) + a256(16) +
           extraBytes(numLightPaths) + extraBytes(numEyePaths);
}

void carveBptBuffers(void* base, uint32_t numLightPaths, uint32_t numEyePaths, uint32_t cacheCapacity,
                     PathBuffers* lightPaths, BptBuffers* bb) {
    char* s = static_cast<char*>(base);
    carvePathBuffers(s, numLightPaths, lightPaths);
    s += pathBufferBytes(numLightPaths);
    bb->cache = reinterpret_cast<LightVertex*>(s);
    s += a256(size_t(cacheCapacity) * sizeof(LightVertex));
    bb->counters = reinterpret_cast<uint32_t*>(s);
    s += a256(16);
    bb->capacity = cacheCapacity;
    carveExtra(s, numLightPaths, &bb->light);
    carveExtra(s, numEyePaths, &bb->eye);
}

void bptRenderLaunch(const SceneGPU &scene, const PathBuffers &eyePaths, const PathBuffers &lightPaths,
                     const BptBuffers &bb, const Film &film, const FrameParams &fp, uint32_t numLightPaths,
                     const WLS &commonWls, float wlPdf, int numSMs, cudaStream_t stream, StageTimer* timer) {
    if (fp.maxPathLength == 0 || fp.maxPathLength >= kMaxBounces)
        throw std::runtime_error("maxPathLength out of range");
    if (scene.lightInsts.n == 0)
        throw std::runtime_error("LVC-BPT needs at least one light");

    StageTimer dummy;
    StageTimer &T = timer ? *timer : dummy;
    const int grid = numSMs * static_cast<int>(fp.blocksPerSM ? fp.blocksPerSM : 8);
    const size_t pBytes = sizeof(BptArgs);
    BptArgs a{};
    a.S = scene;
    a.bb = bb;
    a.film = film;
    a.wls = commonWls;
    a.wlPdf = wlPdf;
    a.numLightPaths = numLightPaths;
    a.width = fp.width;
    a.height = fp.height;
    a.stride = fp.stride;
    a.maxPathLength = fp.maxPathLength;
    // light subpaths
    ck(cudaMemsetAsync(bb.counters, 0, 8, stream), "cache counters");
    ck(cudaMemsetAsync(lightPaths.counters, 0, size_t(kMaxBounces + 1) * kCountersPerBounce * 4, stream), "counters");
    a.pb = lightPaths;
    a.ex = bb.light;
    a.numPaths = numLightPaths;
    T.begin(kStageCamera, stream, pBytes);
    lightStartKernel<<<grid, 256, 0, stream>>>(a);
    T.end(stream);
    FrameParams lf = fp;
    lf.numPaths = numLightPaths;
    for (uint32_t b = 0; b < fp.maxPathLength; ++b) {
        lf.bounce = b;
        a.bounce = b;
        T.begin(kStageTrace, stream, sizeof(SceneGPU) + sizeof(PathBuffers) + sizeof(FrameParams));
        launchTraceSorted(scene, lightPaths, lf, grid, stream);
        T.end(stream);
        T.begin(kStageShade, stream, pBytes);
        lightShadeKernel<<<grid, 256, 0, stream>>>(a);
        T.end(stream);
    }
    T.begin(kStageFilm, stream, sizeof(PathBuffers) + 4);
    bptStatsKernel<<<1, 32, 0, stream>>>(lightPaths, fp.maxPathLength);
    T.end(stream);
    // eye subpaths
    ck(cudaMemsetAsync(eyePaths.counters, 0, size_t(kMaxBounces + 1) * kCountersPerBounce * 4, stream), "counters");
    a.pb = eyePaths;
    a.ex = bb.eye;
    a.numPaths = fp.numPaths;
    a.bounce = 0;
    T.begin(kStageCamera, stream, pBytes);
    eyeStartKernel<<<grid, 256, 0, stream>>>(a);
    T.end(stream);
    T.begin(kStageShadow, stream, pBytes);
    connectKernel<<<grid, 256, 0, stream>>>(a);
    T.end(stream);
    FrameParams ef = fp;
    for (uint32_t b = 0; b < fp.maxPathLength; ++b) {
        ef.bounce = b;
        a.bounce = b;
        T.begin(kStageTrace, stream, sizeof(SceneGPU) + sizeof(PathBuffers) + sizeof(FrameParams));
        launchTraceSorted(scene, eyePaths, ef, grid, stream);
        T.end(stream);
        T.begin(kStageShade, stream, pBytes);
        eyeShadeKernel<<<grid, 256, 0, stream>>>(a);
        T.end(stream);
        a.bounce = b + 1;
        T.begin(kStageShadow, stream, pBytes);
        connectKernel<<<grid, 256, 0, stream>>>(a);
        T.end(stream);
    }
    a.bounce = 0;
    T.begin(kStageFilm, stream, pBytes);
    eyeFilmKernel<<<grid, 256, 0, stream>>>(a);
    T.end(stream);
    T.begin(kStageFilm, stream, sizeof(PathBuffers) + 4);
    bptStatsKernel<<<1, 32, 0, stream>>>(eyePaths, fp.maxPathLength);
    T.end(stream);
    ck(cudaGetLastError(), "launch");
    T.collect();
}

size_t ltConnectionBytes(uint32_t numPaths) { return a256(size_t(numPaths) * sizeof(LtConnection)); }

void ltRenderLaunch(const SceneGPU &scene, const PathBuffers &lightPaths, void* connections, const Film &film,
                    const FrameParams &fp, uint32_t numLightPaths, uint32_t frames, int numSMs, cudaStream_t stream,
                    StageTimer* timer) {
    if (fp.maxPathLength == 0 || fp.maxPathLength >= kMaxBounces)
        throw std::runtime_error("maxPathLength out of range");
    if (scene.lightInsts.n == 0)
        throw std::runtime_error("light tracing needs at least one light");
    StageTimer dummy;
    StageTimer &T = timer ? *timer : dummy;
    const int grid = numSMs * static_cast<int>(fp.blocksPerSM ? fp.blocksPerSM : 8);
    const size_t pBytes = sizeof(BptArgs);
    BptArgs a{};
    a.S = scene;
    a.pb = lightPaths;
    a.film = film;
    a.numLightPaths = numLightPaths;            // per frame: the alpha normalisation
    a.numPaths = numLightPaths * frames;        // slots: `frames` frames in one launch
    a.width = fp.width;
    a.height = fp.height;
    a.stride = fp.stride;
    a.maxPathLength = fp.maxPathLength;
    a.conn = static_cast<LtConnection*>(connections);
    ck(cudaMemsetAsync(lightPaths.counters, 0, size_t(kMaxBounces + 1) * kCountersPerBounce * 4, stream), "counters");
    T.begin(kStageCamera, stream, pBytes);
    ltStartKernel<<<grid, 256, 0, stream>>>(a);
    T.end(stream);
    T.begin(kStageShadow, stream, pBytes + 4);
    ltSplatKernel<<<grid, 256, 0, stream>>>(a, 0u);
    T.end(stream);
    FrameParams lf = fp;
    lf.numPaths = a.numPaths;
    // at most maxPathLength - 1 traced segments before the lens connection
    // (the loop of light_tracing.cu:145-171 with MaxPathLength)
    for (uint32_t b = 0; b + 1 < fp.maxPathLength; ++b) {
        lf.bounce = b;
        a.bounce = b;
        T.begin(kStageTrace, stream, sizeof(SceneGPU) + sizeof(PathBuffers) + sizeof(FrameParams));
        launchTraceSorted(scene, lightPaths, lf, grid, stream);
        T.end(stream);
        T.begin(kStageShade, stream, pBytes);
        ltShadeKernel<<<grid, 256, 0, stream>>>(a);
        T.end(stream);
        T.begin(kStageShadow, stream, pBytes + 4);
        ltSplatKernel<<<grid, 256, 0, stream>>>(a, b + 1);
        T.end(stream);
    }
    T.begin(kStageFilm, stream, sizeof(PathBuffers) + 4);
    bptStatsKernel<<<1, 32, 0, stream>>>(lightPaths, fp.maxPathLength);
    T.end(stream);
    ck(cudaGetLastError(), "launch");
    T.collect();
}

} // namespace vlrb
