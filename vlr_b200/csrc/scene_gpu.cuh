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
    int32_t sub[4] = { -1, -1, -1, -1 };     // Multi: the non-emitting sub-materials' indices
    uint32_t numSub = 0;
    int32_t texF = -1;      // float3 plug texture: roughness/anisotropy/rotation (microfacet) or
                            // occlusion/roughness/metallic (UE4); -1: the immediate f[]
    uint32_t texFOpt = 0;   // plug option: 0 the texel's xyz, 1 its yzw; LambertianScattering's
                            // "f0" (a float1 plug): the channel << 8
};

// MatDesc::bsdfKind of a Multi material: outside the BSDF kinds, so nothing
// shades it directly; hits resolve it to one of its sub-materials first.
constexpr uint32_t kMultiBSDF = 0x100u;

// Bump types of Image2DTexture (shared/shared.h:147-151).
enum BumpKind : uint32_t { kBumpNormalDirectX = 0, kBumpNormalOpenGL = 1, kBumpHeight = 2 };

// Normal and alpha maps of one geometry instance: the material group's
// nodeNormal and nodeAlpha plugs when they are Image2DTexture nodes
// (kernel_common.h:70-72).  Texture indices address MengTables::textures;
// height maps read a point-sampled texture of their image.
struct GeomMaps {
    int32_t normalTex = -1;     // -1: no normal map
    uint32_t normalInfo = 0;    // BumpKind | plug option << 8
    float bumpCoeff = 1.0f;     // decoded 5-bit coefficient
    float texW = 0.0f, texH = 0.0f;   // size of the normal map's image
    int32_t alphaTex = -1;      // -1: opaque
    uint32_t alphaOption = 0;   // channel read as alpha
    uint32_t pad = 0;
};

// Spectrum slot 0-2 (sp) or 3 (emit) of material m at the path's wavelengths
// and texture coordinates (tu, tv): a texture's filtered RGB upsampled at the
// hit (Image2DTextureShaderNode_Spectrum, shader_nodes.cu:410-445), else the
// scene's blended table, else the UpSpec.
VLRB_HD S4 matSpectrum(const MengTables &T, const MatDesc &m, int slot, const WLS &wls, float tu = 0.0f,
                       float tv = 0.0f) {
#if defined(__CUDA_ARCH__)
    if (T.textures && slot < 3 && m.tex[slot] >= 0) {
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
    const GeomMaps* geomMaps;       // [numGeomInsts], null when no group has a normal or alpha map
    uint32_t hasAlphaMaps;          // some group has an alpha map: traversal runs the alpha test
    uint32_t hasScalarTextures;     // some material has a float3 texture plug (MatDesc::texF)
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
    const UpSpec* envTexels;        // [1] the immediate emittance of an untextured environment
    unsigned long long envTex;      // cudaTextureObject_t of the environment image (0: untextured):
                                    // per texel Meng (u, v, s) + alpha in half precision, bilinear,
                                    // repeat in u and v, normalised coordinates
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
// kScalarTextures false: the caller knows no material has a float3 texture
// plug (a hit shader compiled without that read keeps its registers).
template <int K = -1, bool kScalarTextures = true>
VLRB_HD Bsdf buildBsdf(const MengTables &T, const MatDesc &m, const WLS &wls, float tu = 0.0f, float tv = 0.0f) {
    Bsdf B;
    const uint32_t kind = K >= 0 ? static_cast<uint32_t>(K) : m.bsdfKind;
    B.kind = kind;
    B.flags = 0;
    B.f0 = m.f[0]; B.f1 = m.f[1]; B.f2 = m.f[2];
    float metallic = m.f[1];
#if defined(__CUDA_ARCH__)
    if (kScalarTextures && T.textures && m.texF >= 0) {
        // the float3 plug's texel (Image2DTextureShaderNode_float3,
        // shader_nodes.cu:320-334), turned into the BSDF's scalars as the
        // setupBSDF programs do (materials.cu:1521-1533, 1964-1969)
        const float4 c = tex2DLod<float4>(T.textures[m.texF], tu, tv, 0.0f);
        const float x = m.texFOpt == 0 ? c.x : c.y, y = m.texFOpt == 0 ? c.y : c.z, z = m.texFOpt == 0 ? c.z : c.w;
        if (kind == kLambertianBSDF) {
            // "f0", a float1 plug: the option's channel (shader_nodes.cu:284-301)
            const uint32_t o = m.texFOpt >> 8;
            B.f0 = o == 0 ? c.x : o == 1 ? c.y : o == 2 ? c.z : c.w;
        }
        else if (kind == kUE4) {
            B.f0 = fmaxf(0.01f, y);
            metallic = z;
        }
        else {
            const float alpha = x * x, aspect = sqrtf(1 - 0.9f * y);
            B.f0 = fmaxf(0.001f, alpha / aspect);
            B.f1 = fmaxf(0.001f, alpha * aspect);
            B.f2 = 2 * kPi * z;
        }
    }
#endif
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
        const float specular = 0.5f;
        B.a = base * (1 - metallic);
        B.b = lerpS(0.08f * specular * S4::one(), base, metallic);
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

// The four texels of the bilinear footprint at (tu, tv), one channel, in
// texture-gather order (w z over x y: w the footprint's first row and
// column); `tex` is point-sampled, so each fetch at a texel centre returns
// that texel, wrapped by the texture's address mode.
__device__ __forceinline__ float4 footprintTexels(cudaTextureObject_t tex, float tu, float tv, uint32_t channel,
                                                  float w, float h) {
    const float i0 = floorf(tu * w - 0.5f), j0 = floorf(tv * h - 0.5f);
    auto at = [&](float i, float j) {
        const float4 c = tex2DLod<float4>(tex, (i + 0.5f) / w, (j + 0.5f) / h, 0.0f);
        return channel == 0 ? c.x : channel == 1 ? c.y : channel == 2 ? c.z : c.w;
    };
    return make_float4(at(i0, j0 + 1), at(i0 + 1, j0 + 1), at(i0 + 1, j0), at(i0, j0));
}

// Image2DTextureShaderNode_Normal3D (shader_nodes.cu:349-391): the normal in
// the shading frame from a normal map (RGB or GBA by plug option, [0,1] ->
// [-1,1], y flipped for DirectX maps) or from height-map differences
// (5/1024 per texel), its tangential part scaled by the bump coefficient.
__device__ __forceinline__ V3 mapNormal(const unsigned long long* textures, const GeomMaps &gm, float tu, float tv) {
    const cudaTextureObject_t tex = textures[gm.normalTex];
    const uint32_t bump = gm.normalInfo & 0xFFu, option = gm.normalInfo >> 8;
    V3 n(0.0f, 0.0f, 1.0f);
    if (bump != kBumpHeight) {
        if (option < 2) {
            const float4 c = tex2DLod<float4>(tex, tu, tv, 0.0f);
            n = option == 0 ? V3(c.x, c.y, c.z) : V3(c.y, c.z, c.w);
            n = V3(2 * n.x - 1.0f, 2 * n.y - 1.0f, 2 * n.z - 1.0f);
            if (bump == kBumpNormalDirectX) n.y = -n.y;
        }
    }
    else {
        const float4 g = footprintTexels(tex, tu, tv, option, gm.texW, gm.texH);
        const float coeff = 5.0f / 1024;
        const float dhdu = (coeff * gm.texW) * (g.y - g.x);
        const float dhdv = (coeff * gm.texH) * (g.x - g.w);
        n = V3(-dhdu, dhdv, 1.0f);
    }
    n.x *= gm.bumpCoeff;
    n.y *= gm.bumpCoeff;
    return normalize(n);
}

// applyBumpMapping (renderer_common.h:554-576): rotate the shading frame by
// the rotation that carries its normal (0, 0, 1) onto n, written as a unit
// quaternion about the axis (-n.y, n.x, 0) by the tilt angle.
__device__ __forceinline__ void bumpFrame(const V3 &n, Frame* frame) {
    if (n.x == 0.0f && n.y == 0.0f) return;
    const float projLength = sqrtf(n.x * n.x + n.y * n.y);
    const float tilt = atanf(projLength / n.z);
    float qSin, qCos;
    sincosf(tilt / 2, &qSin, &qCos);
    const float qX = (-n.y / projLength) * qSin, qY = (n.x / projLength) * qSin, qW = qCos;
    const V3 t(1 - 2 * qY * qY, 2 * qX * qY, -2 * qY * qW);
    const V3 b(2 * qX * qY, 1 - 2 * qX * qX, 2 * qX * qW);
    *frame = Frame(frame->fromLocal(t), frame->fromLocal(b), frame->fromLocal(n));
}

// The shading frame after a group's normal map; kept out of line so that the
// hit shaders of scenes without normal maps do not carry its registers.
static __device__ __noinline__ Frame normalMappedFrame(const GeomMaps* gm, const unsigned long long* textures, float tu,
                                                       float tv, Frame frame) {
    bumpFrame(mapNormal(textures, *gm, tu, tv), &frame);
    return frame;
}

// Alpha of triangle `prim` at barycentrics (b1, b2): its group's alpha map
// channel (Image2DTextureShaderNode_Alpha, shader_nodes.cu:437-455), 1 for a
// group without one (getAlpha, renderer_common.h:532-547).
__device__ __forceinline__ float alphaAt(const SceneGPU &S, uint32_t prim, float b1, float b2) {
    const uint4 t = __ldg(S.tri + prim);
    const GeomMaps &gm = S.geomMaps[t.w];
    if (gm.alphaTex < 0) return 1.0f;
    const float b0 = 1 - b1 - b2;
    const float2 a = __ldg(S.uv + t.x), b = __ldg(S.uv + t.y), c = __ldg(S.uv + t.z);
    const float4 v = tex2DLod<float4>(S.meng.textures[gm.alphaTex], b0 * a.x + b1 * b.x + b2 * c.x,
                                      b0 * a.y + b1 * b.y + b2 * c.y, 0.0f);
    const uint32_t o = gm.alphaOption;
    return o == 0 ? v.x : o == 1 ? v.y : o == 2 ? v.z : o == 3 ? v.w : 0.0f;
}

// Uniform [0, 1) number for the pair (seed, prim): the SplitMix64 finalizer
// (Steele, Lea and Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014) of seed + prim times the golden-ratio increment.
__device__ __forceinline__ float hashUniform(uint64_t seed, uint32_t prim) {
    uint64_t z = seed + (static_cast<uint64_t>(prim) + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return static_cast<float>(static_cast<uint32_t>(z >> 40)) * (1.0f / 16777216.0f);
}

// Stochastic alpha test of a closest-hit ray (pathTracingAnyHitWithAlpha,
// path_tracing.cu:15-25): an intersection is kept when u < alpha.  u comes
// from the path's RNG state mixed with the primitive, so it does not advance
// the path's stream and a ray meets each triangle with one decision.
struct StochasticAlpha {
    static constexpr bool kNeedsBarycentrics = true;
    const SceneGPU* S;
    uint64_t seed;
    __device__ __forceinline__ bool operator()(uint32_t prim, float b1, float b2) const {
        const float a = alphaAt(*S, prim, b1, b2);
        return a >= 1.0f || hashUniform(seed, prim) < a;
    }
};

// Shadow rays (shadowAnyHitWithAlpha, light_transport_common.h:206-219): the
// visibility is the product of (1 - alpha) over the surfaces the segment
// crosses; an intersection ends the ray once that product reaches 0.
struct AlphaVisibility {
    static constexpr bool kNeedsBarycentrics = true;
    const SceneGPU* S;
    float visibility;
    __device__ __forceinline__ bool operator()(uint32_t prim, float b1, float b2) {
        visibility *= 1.0f - alphaAt(*S, prim, b1, b2);
        return visibility == 0.0f;
    }
};

// Fractional visibility of the segment org + t dir, t in (0, tmax).
__device__ __forceinline__ float shadowVisibility(const SceneGPU &S, const V3 &org, const V3 &dir, float tmax) {
    if (!S.hasAlphaMaps) return traceBvh<true>(S.bvh, org, dir, tmax).prim == 0xFFFFFFFFu ? 1.0f : 0.0f;
    AlphaVisibility av{ &S, 1.0f };
    const Hit h = traceBvhWith<true>(S.bvh, org, dir, tmax, av);
    return h.prim == 0xFFFFFFFFu ? av.visibility : 0.0f;
}

// The material whose BSDF shades a hit on triangle `prim` of material `mat`.
// A Multi material (MultiBSDF, materials.cu:2255-2594, the sum of up to four
// BSDFs) picks one of its n sub-BSDFs uniformly and reports scale n: the
// path's throughput times n x f_i is an unbiased estimate of the sum, the
// sub-BSDF's own pdfs serve its sampling and MIS, and a hit's emission (the
// sum of the sub-emitters) is not scaled.  The choice is a function of the
// path's RNG state (not yet advanced between trace and shade) and the
// primitive, so the trace kernel's material sort and the shader agree.
__device__ __forceinline__ uint32_t bsdfMaterial(const SceneGPU &S, uint32_t mat, uint64_t rngState, uint32_t prim,
                                                 float* scale) {
    *scale = 1.0f;
    const MatDesc &m = S.mats[mat];
    if (m.bsdfKind != kMultiBSDF) return mat;
    const uint32_t n = m.numSub;
    const uint32_t i = min(static_cast<uint32_t>(hashUniform(rngState + 0x632BE59BD9B4E019ULL, prim) * n), n - 1);
    *scale = static_cast<float>(n);
    return static_cast<uint32_t>(m.sub[i]);
}

// Closest hit of a path's ray, alpha-tested with the path's RNG state.
__device__ __forceinline__ Hit traceClosest(const SceneGPU &S, const V3 &org, const V3 &dir, float tmax,
                                            uint64_t rngState) {
    if (!S.hasAlphaMaps) return traceBvh<false>(S.bvh, org, dir, tmax);
    StochasticAlpha sa{ &S, rngState };
    return traceBvhWith<false>(S.bvh, org, dir, tmax, sa);
}

// decodeLocalHitPointForTriangle + calcSurfacePoint (triangle.cu:6-53,
// renderer_common.h:609-626) on world-space vertices, the group's normal map
// applied to the shading frame.
// kNormalMaps false: the caller knows the scene has no normal maps (a
// hit shader compiled without the normal-map call keeps its registers).
template <bool kNormalMaps = true>
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
    if (kNormalMaps && S.geomMaps && S.geomMaps[g].normalTex >= 0)
        sp->frame = normalMappedFrame(S.geomMaps + g, S.meng.textures, sp->tu, sp->tv, sp->frame);
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

// Radiance of the environment at texture coordinate (u, v), as the
// reference's spectral build computes it (shader_nodes.cu:457-483): the
// image is held as per-texel Meng-Simon coordinates (u, v) and brightness s
// in half precision (image.cpp:542-566), the texture unit filters those
// bilinearly with repeat wrapping (the node's default linear filter,
// shader_nodes.cpp:1895-1915), and the spectrum is the one at the filtered
// (u, v) with scale s / EqualEnergyReflectance.
__device__ __forceinline__ S4 envRadiance(const SceneGPU &S, float u, float v, const WLS &wls) {
    if (!S.envTex) return mengEvaluate(S.meng, S.envTexels[0], wls);
    const float4 uvs = tex2DLod<float4>(static_cast<cudaTextureObject_t>(S.envTex), u, v, 0.0f);
    UpSpec t;
    mengAdjacents(S.meng, uvs.x, uvs.y, &t);
    t.scale = uvs.z / kMengEqualEnergy;
    return mengEvaluate(S.meng, t, wls);
}

#endif

} // namespace vlrb
