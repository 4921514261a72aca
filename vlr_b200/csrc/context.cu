// Rendering context: scene flattening and upload, light tables, environment
// importance map, camera setup, render orchestration and film readout.
//
// Scene build (replaces Scene::setup, libVLR/scene.cpp:1149-1402, and the
// OptiX GAS/IAS builds at :1318-1328): the node graph is walked from the
// scene root, every (transform chain, triangle mesh) pair becomes one
// instance whose vertices are transformed to world space, and a single LBVH
// is built over all world-space triangles on the GPU.  Light tables keep the
// reference's probabilities: emitting instances (environment first) and
// emitting material groups are chosen uniformly, triangles by area.
#include "context.cuh"
#include "lbvh_build.h"
#include "tables.cuh"
#include "bpt.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <random>
#include <string>

namespace vlrb {

// envmap.cu
void buildEnvDistribution(const float* hostLuminance, uint32_t w, uint32_t h, double* rowCdf, double* margCdf,
                          float* rowPdf, float* margPdf, void* scratch, cudaStream_t stream);
size_t envScratchBytes(uint32_t w, uint32_t h);
namespace api {

namespace {

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Column-major 4x4 helpers.
void matMul(const float a[16], const float b[16], float out[16]) {
    float r[16];
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            float s = 0;
            for (int k = 0; k < 4; ++k) s += a[k * 4 + rr] * b[c * 4 + k];
            r[c * 4 + rr] = s;
        }
    std::memcpy(out, r, sizeof(r));
}
void matIdentity(float m[16]) {
    for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.0f : 0.0f;
}
V3 xfPoint(const float m[16], const V3 &p) {
    return V3(m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12],
              m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
              m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14]);
}
V3 xfVector(const float m[16], const V3 &v) {
    return V3(m[0] * v.x + m[4] * v.y + m[8] * v.z, m[1] * v.x + m[5] * v.y + m[9] * v.z,
              m[2] * v.x + m[6] * v.y + m[10] * v.z);
}
// Normals transform by the inverse transpose (shared/shared.h:316-321).
V3 xfNormal(const float inv[16], const V3 &n) {
    return V3(inv[0] * n.x + inv[1] * n.y + inv[2] * n.z, inv[4] * n.x + inv[5] * n.y + inv[6] * n.z,
              inv[8] * n.x + inv[9] * n.y + inv[10] * n.z);
}

ColorSp parseColorSpace(const std::string &s) {
    std::string l = lower(s);
    if (l == "rec709(d65) srgb gamma") return ColorSp::sRGB;
    if (l == "xyz") return ColorSp::XYZ;
    if (l == "xyy") return ColorSp::xyY;
    return ColorSp::Rec709;
}

UpSpec upsampleImm(const ImmSpectrum &s, SpType t) {
    return mengUpsample(hostMengTables(), hostColorMatrices(), t, parseColorSpace(s.colorSpace), s.e[0], s.e[1], s.e[2]);
}

// Reference-style discrete distribution: PMF = w / sum, CDF prefix / sum with
// a compensated (Kahan) running sum, CDF[n] = 1 (context.cpp:1796-1819).
struct HostDist {
    std::vector<float> pmf, cdf;
    float integral = 0;
};
HostDist makeDist(const std::vector<float> &w) {
    HostDist d;
    const size_t n = w.size();
    d.pmf = w;
    d.cdf.assign(n + 1, 0.0f);
    float sum = 0, comp = 0;
    for (size_t i = 0; i < n; ++i) {
        d.cdf[i] = sum;
        float y = w[i] - comp;
        float t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    d.integral = sum;
    for (size_t i = 0; i < n; ++i) { d.pmf[i] /= d.integral; d.cdf[i] /= d.integral; }
    d.cdf[n] = 1.0f;
    return d;
}

} // namespace

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void DeviceBuffer::resize(size_t b) {
    if (b <= bytes && ptr) return;
    release();
    ck(cudaMalloc(&ptr, b > 0 ? b : 1), "cudaMalloc");
    bytes = b;
}

Context::Context(CUcontext cu, bool log) : Object(Kind::Context), cuContext(cu), logging(log) {
    typeName = "Context";
    ctx = this;
    ck(cudaGetDevice(&device), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, device), "SM count");
    ck(cudaMallocHost(reinterpret_cast<void**>(&hostCounters), (kMaxBounces + 1) * kCountersPerBounce * 4),
       "pinned counters");
}

Context::~Context() {
    for (Object* o : objects) delete o;
    objects.clear();
    if (outArray) cudaFreeArray(reinterpret_cast<cudaArray_t>(outArray));
    if (hostCounters) cudaFreeHost(hostCounters);
}

void Context::destroy(Object* o) {
    if (!owns(o)) return;
    objects.erase(o);
    if (o == scene) scene = nullptr;
    delete o;
    markDirty();
}

template <typename T>
T* Context::upload(const std::vector<T> &v, cudaStream_t stream) {
    auto buf = std::make_unique<DeviceBuffer>();
    buf->resize(std::max<size_t>(v.size() * sizeof(T), 16));
    if (!v.empty())
        ck(cudaMemcpyAsync(buf->ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
    T* p = buf->as<T>();
    sceneBufs.push_back(std::move(buf));
    return p;
}

void Context::bindOutput(uint32_t w, uint32_t h) {
    width = w;
    height = h;
    film.resize(size_t(w) * h * kNumStrata * 8 + 256);
    output.resize(size_t(w) * h * 16);
    ck(cudaMemset(film.ptr, 0, film.bytes), "film clear");
    ck(cudaMemset(output.ptr, 0, size_t(w) * h * 16), "output clear");
    if (outArray) { cudaFreeArray(reinterpret_cast<cudaArray_t>(outArray)); outArray = nullptr; }
    pathCapacity = 0;
    numAccumFrames = 0;
}

CUarray Context::outputArray() {
    // A CUDA array of RGBA32F texels refreshed from the output image; runtime
    // API only so the library needs no link-time dependency on the driver.
    if (!outArray && width > 0) {
        cudaChannelFormatDesc desc = cudaCreateChannelDesc<float4>();
        cudaArray_t a = nullptr;
        ck(cudaMallocArray(&a, &desc, width, height), "cudaMallocArray");
        outArray = reinterpret_cast<CUarray>(a);
    }
    if (outArray)
        ck(cudaMemcpy2DToArray(reinterpret_cast<cudaArray_t>(outArray), 0, 0, output.ptr, size_t(width) * 16,
                               size_t(width) * 16, height, cudaMemcpyDeviceToDevice), "output array copy");
    return outArray;
}

void Context::readOutput(float* host) {
    ck(cudaMemcpy(host, output.ptr, size_t(width) * height * 16, cudaMemcpyDeviceToHost), "read output");
}

bool Context::readAux(float* albedo, float* normal) {
    if (!auxCurrent || auxSamples == 0) return false;
    const size_t bytes = size_t(width) * height * sizeof(float4);
    if (albedo) ck(cudaMemcpy(albedo, aux.linAlbedo, bytes, cudaMemcpyDeviceToHost), "read aux");
    if (normal) ck(cudaMemcpy(normal, aux.linNormal, bytes, cudaMemcpyDeviceToHost), "read aux");
    return true;
}

void Context::readFilm(double* host) {
    ck(cudaMemcpy(host, film.ptr, size_t(width) * height * kNumStrata * 8, cudaMemcpyDeviceToHost), "read film");
}

namespace {

// Material descriptor from the material's parameters, following each
// material's setupMaterialDescriptor / setupBSDF pair in the reference
// (libVLR/materials.cpp and GPU_kernels/materials.cu).
MatDesc describeMaterial(const SurfaceMaterial* m) {
    MatDesc d{};
    std::memset(&d, 0, sizeof(d));
    for (int32_t &k : d.table) k = -1;
    for (int32_t &k : d.tex) k = -1;
    for (int32_t &k : d.sub) k = -1;
    d.texF = -1;
    d.bsdfKind = kNullBSDF;
    d.emitScale = 1.0f;
    const std::string t = lower(m->typeName);
    auto spec = [&](const char* name) { return m->spectra.at(lower(name)); };
    auto roughAniso = [&](float* out) {
        float r = m->getFloat("roughness", 0.1f), a = m->getFloat("anisotropy", 0.0f), rot = m->getFloat("rotation", 0.0f);
        float alpha = r * r;
        float aspect = std::sqrt(1.0f - 0.9f * a);
        out[0] = std::fmax(0.001f, alpha / aspect);
        out[1] = std::fmax(0.001f, alpha * aspect);
        out[2] = 2 * kPi * rot;
    };
    if (t == "matte") {
        d.bsdfKind = kMatte;
        d.sp[0] = upsampleImm(spec("albedo"), SpType::Reflectance);
    }
    else if (t == "specularreflection") {
        d.bsdfKind = kSpecularBRDF;
        d.sp[0] = upsampleImm(spec("coeff"), SpType::Reflectance);
        d.sp[1] = upsampleImm(spec("eta"), SpType::IOR);
        d.sp[2] = upsampleImm(spec("k"), SpType::IOR);
    }
    else if (t == "specularscattering") {
        d.bsdfKind = kSpecularBSDF;
        d.sp[0] = upsampleImm(spec("coeff"), SpType::Reflectance);
        d.sp[1] = upsampleImm(spec("eta ext"), SpType::IOR);
        d.sp[2] = upsampleImm(spec("eta int"), SpType::IOR);
    }
    else if (t == "microfacetreflection") {
        d.bsdfKind = kMicrofacetBRDF;
        d.sp[1] = upsampleImm(spec("eta"), SpType::IOR);
        d.sp[2] = upsampleImm(spec("k"), SpType::IOR);
        roughAniso(d.f);
    }
    else if (t == "microfacetscattering") {
        d.bsdfKind = kMicrofacetBSDF;
        d.sp[0] = upsampleImm(spec("coeff"), SpType::Reflectance);
        d.sp[1] = upsampleImm(spec("eta ext"), SpType::IOR);
        d.sp[2] = upsampleImm(spec("eta int"), SpType::IOR);
        roughAniso(d.f);
    }
    else if (t == "lambertianscattering") {
        d.bsdfKind = kLambertianBSDF;
        d.sp[0] = upsampleImm(spec("coeff"), SpType::Reflectance);
        d.f[0] = m->getFloat("f0", 0.04f);
    }
    else if (t == "ue4") {
        d.bsdfKind = kUE4;
        d.sp[0] = upsampleImm(spec("base color"), SpType::Reflectance);
        d.f[0] = std::fmax(0.01f, m->getFloat("roughness", 0.1f));
        d.f[1] = m->getFloat("metallic", 0.0f);
    }
    else if (t == "diffuseemitter") {
        d.emitter = 1;
        d.emit = upsampleImm(spec("emittance"), SpType::LightSource);
        d.emitScale = m->getFloat("scale", 1.0f);
    }
    else if (t == "pointemitter") {
        d.emitter = kEmitPoint;
        d.emit = upsampleImm(spec("intensity"), SpType::LightSource);
        d.emitScale = m->getFloat("scale", 1.0f);
    }
    else if (t == "directionalemitter") {
        d.emitter = kEmitDirectional;
        d.emit = upsampleImm(spec("emittance"), SpType::LightSource);
        d.emitScale = m->getFloat("scale", 1.0f);
    }
    else if (t == "environmentemitter") {
        d.emitter = 2;
        d.emit = upsampleImm(spec("emittance"), SpType::LightSource);
        d.emitScale = m->getFloat("scale", 1.0f);
    }
    return d;
}

struct FlatScene {
    std::vector<float4> pos, nrm, tan;
    std::vector<float2> uv;
    std::vector<uint4> tri;
    std::vector<uint32_t> triMaterial;
    std::vector<float> triVerts;                 // 9 floats per triangle for the BVH build
    std::vector<MatDesc> mats;
    std::vector<const SurfaceMaterial*> matObjs;
    // geometry instances (one per instance x material group)
    std::vector<uint32_t> geomInstInstance;
    std::vector<uint32_t> geomInstMaterial;
    std::vector<std::vector<uint32_t>> geomInstTris;
    std::vector<std::vector<float>> geomInstAreas;
    std::vector<uint32_t> geomInstPoints;        // 1: the geometry instance is points (ids into pt*)
    std::vector<VLRShaderNodePlug> geomInstNormal, geomInstAlpha;   // the group's nodeNormal / nodeAlpha
    std::vector<float4> ptPos, ptNrm, ptTan;     // points of PointSurfaceNodes, world space
    uint32_t numInstances = 0;
    V3 lo{ FLT_MAX, FLT_MAX, FLT_MAX }, hi{ -FLT_MAX, -FLT_MAX, -FLT_MAX };
};

uint32_t materialIndex(FlatScene &f, const SurfaceMaterial* m) {
    for (size_t i = 0; i < f.matObjs.size(); ++i)
        if (f.matObjs[i] == m) return static_cast<uint32_t>(i);
    f.matObjs.push_back(m);
    f.mats.push_back(describeMaterial(m));
    const uint32_t index = static_cast<uint32_t>(f.mats.size() - 1);
    if (lower(m->typeName) == "multi") {
        // MultiSurfaceMaterial::setupMaterialDescriptor (materials.cpp:2098-2113)
        // keeps the set sub-materials in order.  Here the BSDF-bearing ones
        // (not nested Multis) become sub[]; the diffuse emitters' emittance
        // is summed into this material's emission when the tables are built.
        uint32_t n = 0;
        bool emits = false;
        for (const char* k : { "0", "1", "2", "3" }) {
            auto it = m->objects.find(k);
            if (it == m->objects.end() || !it->second) continue;
            const auto* sub = static_cast<const SurfaceMaterial*>(it->second);
            if (sub == m || lower(sub->typeName) == "multi") continue;
            const uint32_t si = materialIndex(f, sub);
            if (f.mats[si].emitter == kEmitDiffuse) emits = true;
            if (f.mats[si].bsdfKind != kNullBSDF) f.mats[index].sub[n++] = static_cast<int32_t>(si);
        }
        f.mats[index].numSub = n;
        f.mats[index].bsdfKind = n > 0 ? kMultiBSDF : kNullBSDF;
        f.mats[index].emitter = emits ? kEmitDiffuse : kEmitNone;
        f.mats[index].emitScale = 1.0f;
    }
    return index;
}

void flattenNode(FlatScene &f, const Node* n, const float world[16], const float worldInv[16]) {
    if (n->kind == Kind::TriangleMeshSurfaceNode) {
        const auto* mesh = static_cast<const TriangleMeshNode*>(n);
        const uint32_t inst = f.numInstances++;
        const uint32_t base = static_cast<uint32_t>(f.pos.size());
        for (const VLRVertex &v : mesh->vertices) {
            V3 p = xfPoint(world, V3(v.position.x, v.position.y, v.position.z));
            V3 nn = xfNormal(worldInv, V3(v.normal.x, v.normal.y, v.normal.z));
            V3 tt = xfVector(world, V3(v.tc0Direction.x, v.tc0Direction.y, v.tc0Direction.z));
            f.pos.push_back(make_float4(p.x, p.y, p.z, 0.0f));
            f.nrm.push_back(make_float4(nn.x, nn.y, nn.z, 0.0f));
            f.tan.push_back(make_float4(tt.x, tt.y, tt.z, 0.0f));
            f.uv.push_back(make_float2(v.texCoord.u, v.texCoord.v));
            f.lo = vmin3(f.lo, p);
            f.hi = vmax3(f.hi, p);
        }
        for (const MaterialGroup &g : mesh->groups) {
            if (!g.material) continue;
            const uint32_t gi = static_cast<uint32_t>(f.geomInstMaterial.size());
            const uint32_t mi = materialIndex(f, g.material);
            f.geomInstInstance.push_back(inst);
            f.geomInstMaterial.push_back(mi);
            f.geomInstTris.emplace_back();
            f.geomInstAreas.emplace_back();
            f.geomInstPoints.push_back(0u);
            f.geomInstNormal.push_back(g.nodeNormal);
            f.geomInstAlpha.push_back(g.nodeAlpha);
            for (size_t k = 0; k + 2 < g.indices.size(); k += 3) {
                uint32_t i0 = g.indices[k], i1 = g.indices[k + 1], i2 = g.indices[k + 2];
                if (i0 >= mesh->vertices.size() || i1 >= mesh->vertices.size() || i2 >= mesh->vertices.size())
                    throw std::runtime_error("triangle index out of range");
                const uint32_t t = static_cast<uint32_t>(f.tri.size());
                f.tri.push_back(make_uint4(base + i0, base + i1, base + i2, gi));
                f.triMaterial.push_back(mi);
                const float4 &a = f.pos[base + i0], &b = f.pos[base + i1], &c = f.pos[base + i2];
                f.triVerts.insert(f.triVerts.end(), { a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z });
                // Triangle area in the mesh's own space, as the reference computes it
                // before instancing (scene.cpp:206-207).
                const VLRVertex &va = mesh->vertices[i0], &vb = mesh->vertices[i1], &vc = mesh->vertices[i2];
                V3 e1(vb.position.x - va.position.x, vb.position.y - va.position.y, vb.position.z - va.position.z);
                V3 e2(vc.position.x - va.position.x, vc.position.y - va.position.y, vc.position.z - va.position.z);
                f.geomInstTris.back().push_back(t);
                f.geomInstAreas.back().push_back(0.5f * cross(e1, e2).length());
            }
        }
        return;
    }
    if (n->kind == Kind::PointSurfaceNode) {
        // points are light sources only: rays never hit them (point.cu:40-80
        // samples them; a point of zero radius has no intersection)
        const auto* pts = static_cast<const PointNode*>(n);
        const uint32_t inst = f.numInstances++;
        const uint32_t base = static_cast<uint32_t>(f.ptPos.size());
        for (const VLRVertex &v : pts->vertices) {
            V3 p = xfPoint(world, V3(v.position.x, v.position.y, v.position.z));
            V3 nn = xfNormal(worldInv, V3(v.normal.x, v.normal.y, v.normal.z));
            V3 tt = xfVector(world, V3(v.tc0Direction.x, v.tc0Direction.y, v.tc0Direction.z));
            f.ptPos.push_back(make_float4(p.x, p.y, p.z, 0.0f));
            f.ptNrm.push_back(make_float4(nn.x, nn.y, nn.z, 0.0f));
            f.ptTan.push_back(make_float4(tt.x, tt.y, tt.z, 0.0f));
            f.lo = vmin3(f.lo, p);
            f.hi = vmax3(f.hi, p);
        }
        for (const MaterialGroup &g : pts->groups) {
            if (!g.material) continue;
            const uint32_t mi = materialIndex(f, g.material);
            f.geomInstInstance.push_back(inst);
            f.geomInstMaterial.push_back(mi);
            f.geomInstTris.emplace_back();
            f.geomInstAreas.emplace_back();
            f.geomInstPoints.push_back(1u);
            f.geomInstNormal.push_back(VLRShaderNodePlug{});
            f.geomInstAlpha.push_back(VLRShaderNodePlug{});
            for (uint32_t idx : g.indices) {
                if (idx >= pts->vertices.size()) throw std::runtime_error("point index out of range");
                f.geomInstTris.back().push_back(base + idx);
                f.geomInstAreas.back().push_back(1.0f);   // uniform over the group's points (scene.cpp:380-393)
            }
        }
        return;
    }
    if (n->kind == Kind::InternalNode || n->kind == Kind::Scene) {
        const auto* p = static_cast<const ParentNode*>(n);
        float w[16], wi[16];
        if (p->transform) {
            matMul(world, p->transform->m, w);
            matMul(p->transform->inv, worldInv, wi);
        }
        else {
            std::memcpy(w, world, sizeof(w));
            std::memcpy(wi, worldInv, sizeof(wi));
        }
        for (const Node* c : p->children) flattenNode(f, c, w, wi);
    }
}

} // namespace

Context::SceneTexture::~SceneTexture() {
    if (tex) cudaDestroyTextureObject(tex);
    if (array) cudaFreeArray(array);
}

namespace {

// Material parameters whose Spectrum plug may be an Image2DTexture, with the
// MatDesc spectrum slot each drives (the slots describeMaterial fills).
const std::map<std::string, std::vector<std::pair<std::string, int>>> &textureSlots() {
    static const std::map<std::string, std::vector<std::pair<std::string, int>>> m = {
        { "matte", { { "albedo", 0 } } },
        { "specularreflection", { { "coeff", 0 }, { "eta", 1 }, { "k", 2 } } },
        { "specularscattering", { { "coeff", 0 }, { "eta ext", 1 }, { "eta int", 2 } } },
        { "microfacetreflection", { { "eta", 1 }, { "k", 2 } } },
        { "microfacetscattering", { { "coeff", 0 }, { "eta ext", 1 }, { "eta int", 2 } } },
        { "lambertianscattering", { { "coeff", 0 } } },
        { "ue4", { { "base color", 0 } } },
    };
    return m;
}

SpType parseSpectrumType(const std::string &s) {
    const std::string l = lower(s);
    if (l.find("light") != std::string::npos) return SpType::LightSource;
    if (l.find("ior") != std::string::npos || l.find("refraction") != std::string::npos) return SpType::IOR;
    return SpType::Reflectance;
}

// Image2DTexture's bump coefficient as kernels see it: stored in 5 bits as
// min(round(31 * c / 2), 31) and read back as (stored + 1) / 16
// (shader_nodes.cpp:1684-1686, shared/shared.h:743-746).
float decodedBumpCoeff(float c) {
    const uint32_t maxInt = 31;
    const float r = std::round(maxInt * c * 0.5f);
    const uint32_t stored = r <= 0.0f ? 0u : std::min<uint32_t>(static_cast<uint32_t>(r), maxInt);
    return static_cast<float>(stored + 1) / 16.0f;
}

cudaTextureAddressMode parseWrap(const std::string &s) {
    const std::string l = lower(s);
    if (l == "clamp to edge") return cudaAddressModeClamp;
    if (l == "mirror") return cudaAddressModeMirror;
    if (l == "clamp to border") return cudaAddressModeBorder;
    return cudaAddressModeWrap;
}

} // namespace

// Meng (u, v) and brightness s of a linear Rec.709 (D65) texel, the
// reference's per-pixel conversion for light-source images in spectral mode
// (image.cpp:542-566, xy_to_uv spectrum_types.h:382-391).
static void envTexelUVS(const float* rgb, float* u, float* v, float* s) {
    float c[3] = { rgb[0], rgb[1], rgb[2] }, xyz[3];
    mulColMajor(hostColorMatrices().rec709D65ToXYZ, c, xyz);
    const float b = xyz[0] + xyz[1] + xyz[2];
    const float x = b > 0.0f ? xyz[0] / b : (1.0f / 3.0f);
    const float y = b > 0.0f ? xyz[1] / b : (1.0f / 3.0f);
    *u = 16.730260708356887f * x + 7.7801960340706f * y - 2.170152247475828f;
    *v = -7.530081094743006f * x + 16.192422314095225f * y + 1.1125529268825947f;
    *s = b;
}

void Context::buildScene(cudaStream_t stream) {
    if (!sceneTextures.empty()) {
        // kernels of earlier frames may still read the textures
        ck(cudaDeviceSynchronize(), "texture release");
        sceneTextures.clear();
    }
    sceneBufs.clear();
    std::memset(&sg, 0, sizeof(sg));
    sg.meng = deviceMengTables();
    sg.envInst = -1;
    FlatScene f;
    if (scene) {
        float id[16];
        matIdentity(id);
        flattenNode(f, scene, id, id);
    }
    const uint32_t numTris = static_cast<uint32_t>(f.tri.size());
    // environment material
    const SurfaceMaterial* envMat = scene ? scene->envMaterial : nullptr;
    uint32_t envMatIndex = 0;
    if (envMat) envMatIndex = materialIndex(f, envMat);
    if (f.mats.empty()) f.mats.push_back(MatDesc{});

    // ---- light tables (scene.cpp:1237-1402)
    struct LightInst { std::vector<uint32_t> groups; };
    std::vector<LightInst> lightInsts;
    std::vector<uint32_t> geomInstGroup(f.geomInstMaterial.size(), 0xFFFFFFFFu);
    std::vector<EmitGroup> groups;
    std::vector<uint32_t> lightTris;
    std::vector<HostDist> groupDists;
    const bool envEmitting = envMat && envMat->isEmitting();
    if (envEmitting) lightInsts.push_back(LightInst{ { 0xFFFFFFFEu } });
    {
        std::map<uint32_t, size_t> instToLight;
        for (size_t g = 0; g < f.geomInstMaterial.size(); ++g) {
            if (!f.mats[f.geomInstMaterial[g]].emitter) continue;
            if (f.geomInstTris[g].empty()) continue;
            uint32_t inst = f.geomInstInstance[g];
            auto it = instToLight.find(inst);
            if (it == instToLight.end()) {
                it = instToLight.emplace(inst, lightInsts.size()).first;
                lightInsts.emplace_back();
            }
            const uint32_t grp = static_cast<uint32_t>(groups.size());
            lightInsts[it->second].groups.push_back(grp);
            geomInstGroup[g] = grp;
            EmitGroup eg{};
            eg.firstTri = static_cast<uint32_t>(lightTris.size());
            eg.numTris = static_cast<uint32_t>(f.geomInstTris[g].size());
            eg.material = f.geomInstMaterial[g];
            eg.points = f.geomInstPoints[g];
            const uint32_t kind = f.mats[eg.material].emitter;
            if (kind == kEmitPoint || kind == kEmitDirectional) sg.hasDeltaEmitters = 1u;
            lightTris.insert(lightTris.end(), f.geomInstTris[g].begin(), f.geomInstTris[g].end());
            groupDists.push_back(makeDist(f.geomInstAreas[g]));
            groups.push_back(eg);
        }
    }
    // Device distributions.
    std::vector<Dist1D> instGroupDists;
    std::vector<uint32_t> instFirstGroup;
    std::vector<float> geomLightProb(f.geomInstMaterial.size() + 1, 0.0f);
    const float numLightInsts = static_cast<float>(lightInsts.size());
    HostDist instDist = makeDist(std::vector<float>(lightInsts.size(), 1.0f));
    for (size_t i = 0; i < lightInsts.size(); ++i) {
        const size_t G = lightInsts[i].groups.size();
        HostDist gd = makeDist(std::vector<float>(G, 1.0f));
        Dist1D d{ upload(gd.pmf, stream), upload(gd.cdf, stream), gd.integral, static_cast<uint32_t>(G) };
        instGroupDists.push_back(d);
        const bool isEnv = envEmitting && i == 0;
        instFirstGroup.push_back(isEnv ? 0u : lightInsts[i].groups[0]);
        // Selection probabilities as the reference's MIS uses them
        // (path_tracing.cu:168-170): instProb = groups(inst) / sum of instance
        // importances, geomInstProb = 1 / groups(inst).
        const float instProb = static_cast<float>(G) / numLightInsts;
        const float geomInstProb = 1.0f / static_cast<float>(G);
        if (isEnv) { sg.envInst = 0; sg.envLightProb = instProb * geomInstProb; }
        else
            for (size_t g = 0; g < f.geomInstMaterial.size(); ++g)
                if (geomInstGroup[g] != 0xFFFFFFFFu &&
                    std::find(lightInsts[i].groups.begin(), lightInsts[i].groups.end(), geomInstGroup[g]) !=
                        lightInsts[i].groups.end())
                    geomLightProb[g] = instProb * geomInstProb;
    }
    for (size_t g = 0; g < groups.size(); ++g) {
        const HostDist &hd = groupDists[g];
        groups[g].prims = Dist1D{ upload(hd.pmf, stream), upload(hd.cdf, stream), hd.integral, groups[g].numTris };
    }
    sg.lightInsts = Dist1D{ upload(instDist.pmf, stream), upload(instDist.cdf, stream), instDist.integral,
                            static_cast<uint32_t>(lightInsts.size()) };
    sg.instGroups = upload(instGroupDists, stream);
    sg.instFirstGroup = upload(instFirstGroup, stream);
    sg.groups = upload(groups, stream);
    sg.geomLightPdfArea = upload(geomLightProb, stream);
    geomInstGroup.push_back(0xFFFFFFFFu);
    sg.geomInstGroup = upload(geomInstGroup, stream);
    sg.lightTris = upload(lightTris, stream);
    sg.ptPos = upload(f.ptPos, stream);
    sg.ptNrm = upload(f.ptNrm, stream);
    sg.ptTan = upload(f.ptTan, stream);

    // ---- geometry
    sg.numTris = numTris;
    sg.pos = upload(f.pos, stream);
    sg.nrm = upload(f.nrm, stream);
    sg.tan = upload(f.tan, stream);
    sg.tri = upload(f.tri, stream);
    sg.triMaterial = upload(f.triMaterial, stream);
    for (MatDesc &md : f.mats) md.bsdfFlags = options.consistentDielectricPdf ? kBsdfConsistentPdf : 0u;
    // Image2DTexture plugs: material spectra, then the groups' normal and alpha maps
    {
        std::map<std::pair<const Object*, bool>, int32_t> texIndex;
        std::vector<unsigned long long> texObjs;
        std::vector<uint32_t> texTypes;
        // Texture index of an Image2DTexture node (-1: not one, or no image);
        // pointSampled: a nearest-filtered object of the same image (height maps).
        auto textureOf = [&](const VLRShaderNodePlug &plug, bool pointSampled, const Image2D** imgOut) -> int32_t {
            if (!plug.nodeRef) return -1;
            const auto* node = reinterpret_cast<const ShaderNode*>(plug.nodeRef);
            if (lower(node->typeName) != "image2dtexture") return -1;
            auto io = node->objects.find("image");
            const auto* img = io != node->objects.end() ? static_cast<const Image2D*>(io->second) : nullptr;
            if (!img || img->width == 0 || img->height == 0 ||
                img->rgba.size() < size_t(img->width) * img->height * 4)
                return -1;
            if (imgOut) *imgOut = img;
            auto it = texIndex.find({ node, pointSampled });
            if (it != texIndex.end()) return it->second;
            auto st = std::make_unique<SceneTexture>();
            const cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
            ck(cudaMallocArray(&st->array, &ch, img->width, img->height), "texture array");
            ck(cudaMemcpy2DToArray(st->array, 0, 0, img->rgba.data(), size_t(img->width) * 16,
                                   size_t(img->width) * 16, img->height, cudaMemcpyHostToDevice),
               "texture upload");
            cudaResourceDesc rd{};
            rd.resType = cudaResourceTypeArray;
            rd.res.array.array = st->array;
            cudaTextureDesc td{};
            auto en = [&](const char* k, const char* d) {
                auto e = node->enums.find(k);
                return e != node->enums.end() ? e->second : std::string(d);
            };
            td.addressMode[0] = parseWrap(en("wrap u", "Repeat"));
            td.addressMode[1] = parseWrap(en("wrap v", "Repeat"));
            td.filterMode = pointSampled || lower(en("mag filter", "Linear")) == "nearest" ? cudaFilterModePoint
                                                                                          : cudaFilterModeLinear;
            td.readMode = cudaReadModeElementType;
            td.normalizedCoords = 1;
            ck(cudaCreateTextureObject(&st->tex, &rd, &td, nullptr), "texture object");
            const int32_t index = static_cast<int32_t>(texObjs.size());
            texIndex.emplace(std::make_pair(static_cast<const Object*>(node), pointSampled), index);
            texObjs.push_back(static_cast<unsigned long long>(st->tex));
            // 8-bit sRGB images are linearised when created (vlrLinearImage2DCreate)
            const bool eightBit = img->format != "RGBA32Fx4" && img->format != "Gray32F";
            const ColorSp cs = eightBit && parseColorSpace(img->colorSpace) == ColorSp::sRGB
                                   ? ColorSp::Rec709 : parseColorSpace(img->colorSpace);
            texTypes.push_back(static_cast<uint32_t>(parseSpectrumType(img->spectrumType)) |
                               (static_cast<uint32_t>(cs) << 8));
            sceneTextures.push_back(std::move(st));
            return index;
        };
        for (size_t i = 0; i < f.matObjs.size() && i < f.mats.size(); ++i) {
            const SurfaceMaterial* m = f.matObjs[i];
            auto slots = textureSlots().find(lower(m->typeName));
            if (slots == textureSlots().end()) continue;
            for (const auto &ps : slots->second) {
                auto pl = m->plugs.find(ps.first);
                if (pl == m->plugs.end()) continue;
                const int32_t t = textureOf(pl->second, false, nullptr);
                if (t >= 0) f.mats[i].tex[ps.second] = t;
            }
        }
        // float3 plugs of the scalar parameters
        for (size_t i = 0; i < f.matObjs.size() && i < f.mats.size(); ++i) {
            const std::string t = lower(f.matObjs[i]->typeName);
            const bool lambert = t == "lambertianscattering";
            const char* param = t == "ue4" ? "occlusion/roughness/metallic"
                                : (t == "microfacetreflection" || t == "microfacetscattering")
                                    ? "roughness/anisotropy/rotation"
                                : lambert ? "f0" : nullptr;
            if (!param) continue;
            auto pl = f.matObjs[i]->plugs.find(param);
            const uint32_t want = lambert ? VLRShaderNodePlugType_float1 : VLRShaderNodePlugType_float3;
            if (pl == f.matObjs[i]->plugs.end() || (pl->second.info & 0xFFu) != want) continue;
            const int32_t tx = textureOf(pl->second, false, nullptr);
            if (tx < 0) continue;
            const uint32_t option = (pl->second.info >> 8) & 0xFFu;
            f.mats[i].texF = tx;
            f.mats[i].texFOpt = lambert ? std::min<uint32_t>(option, 3u) << 8 : (option == 1 ? 1u : 0u);
            sg.hasScalarTextures = 1;
        }
        std::vector<GeomMaps> maps(f.geomInstMaterial.size() + 1);
        bool anyMap = false;
        for (size_t g = 0; g < f.geomInstMaterial.size(); ++g) {
            if (f.geomInstPoints[g]) continue;
            const VLRShaderNodePlug &np = f.geomInstNormal[g];
            if (np.nodeRef && (np.info & 0xFFu) == VLRShaderNodePlugType_Normal3D) {
                const auto* node = reinterpret_cast<const ShaderNode*>(np.nodeRef);
                auto bt = node->enums.find("bump type");
                const std::string b = lower(bt != node->enums.end() ? bt->second : std::string("Normal Map (DirectX)"));
                const uint32_t bump = b == "height map" ? kBumpHeight
                                      : b == "normal map (opengl)" ? kBumpNormalOpenGL : kBumpNormalDirectX;
                const Image2D* img = nullptr;
                const int32_t t = textureOf(np, bump == kBumpHeight, &img);
                if (t >= 0) {
                    maps[g].normalTex = t;
                    maps[g].normalInfo = bump | (((np.info >> 8) & 0xFFu) << 8);
                    maps[g].bumpCoeff = decodedBumpCoeff(node->getFloat("bump coeff", 1.0f));
                    maps[g].texW = static_cast<float>(img->width);
                    maps[g].texH = static_cast<float>(img->height);
                    anyMap = true;
                }
            }
            const VLRShaderNodePlug &ap = f.geomInstAlpha[g];
            if (ap.nodeRef && (ap.info & 0xFFu) == VLRShaderNodePlugType_Alpha) {
                const int32_t t = textureOf(ap, false, nullptr);
                if (t >= 0) {
                    maps[g].alphaTex = t;
                    maps[g].alphaOption = (ap.info >> 8) & 0xFFu;
                    sg.hasAlphaMaps = 1;
                    anyMap = true;
                }
            }
        }
        if (!texObjs.empty()) {
            sg.meng.textures = upload(texObjs, stream);
            sg.meng.texSpType = upload(texTypes, stream);
            sg.meng.colorMats = deviceColorMatrices();
            sg.uv = upload(f.uv, stream);
        }
        if (anyMap) sg.geomMaps = upload(maps, stream);
    }
    // Material spectra are immediate colours: each is tabulated once here on
    // the 95-sample grid, so a hit interpolates one table per spectrum.
    {
        std::vector<float> blended(f.mats.size() * 4 * kMengSamples);
        const MengTables hostT = hostMengTables();
        for (size_t i = 0; i < f.mats.size(); ++i)
            for (int k = 0; k < 4; ++k) {
                mengBlend(hostT, k < 3 ? f.mats[i].sp[k] : f.mats[i].emit, blended.data() + (i * 4 + k) * kMengSamples);
                f.mats[i].table[k] = static_cast<int32_t>(i * 4 + k);
            }
        // A Multi material emits the sum of its diffuse emitters' scaled
        // emittance (MultiEDF::evaluateEmittanceInternal, materials.cu:2700-2715).
        for (size_t i = 0; i < f.mats.size(); ++i) {
            if (lower(f.matObjs[i]->typeName) != "multi") continue;
            float* dst = blended.data() + (i * 4 + 3) * kMengSamples;
            std::fill(dst, dst + kMengSamples, 0.0f);
            for (const char* k : { "0", "1", "2", "3" }) {
                auto it = f.matObjs[i]->objects.find(k);
                if (it == f.matObjs[i]->objects.end() || !it->second) continue;
                for (size_t j = 0; j < f.matObjs.size(); ++j) {
                    if (f.matObjs[j] != it->second || j == i || f.mats[j].emitter != kEmitDiffuse) continue;
                    const float* src = blended.data() + (j * 4 + 3) * kMengSamples;
                    for (uint32_t w = 0; w < kMengSamples; ++w) dst[w] += f.mats[j].emitScale * src[w];
                }
            }
        }
        sg.meng.blended = upload(blended, stream);
    }
    sg.mats = upload(f.mats, stream);
    if (f.pos.empty()) { f.lo = V3(0.0f); f.hi = V3(0.0f); }
    sg.bounds.lo = f.lo;
    sg.bounds.hi = f.hi;
    sg.bounds.center = (f.lo + f.hi) * 0.5f;
    sg.bounds.worldRadius = (f.hi - sg.bounds.center).length();
    // A scene without extent (no geometry, or one point) still needs a disc
    // for the environment's light subpaths and its density: a unit radius.
    if (!(sg.bounds.worldRadius > 0.0f)) sg.bounds.worldRadius = 1.0f;
    sg.bounds.worldDiscArea = kPi * sg.bounds.worldRadius * sg.bounds.worldRadius;

    // ---- BVH
    if (numTris > 0) {
        const float* dVerts = upload(f.triVerts, stream);
        auto out = std::make_unique<DeviceBuffer>();
        const size_t n = numTris;
        size_t off[6];
        size_t total = 0;
        const size_t sizes[6] = { n * 4, n * 4, n * 8, n * 24, n * sizeof(BvhNode), n * sizeof(BvhTri) };
        for (int i = 0; i < 6; ++i) { off[i] = total; total += (sizes[i] + 255) & ~size_t(255); }
        out->resize(total);
        char* b = out->as<char>();
        LbvhOutput lo{ reinterpret_cast<uint32_t*>(b + off[0]), reinterpret_cast<uint32_t*>(b + off[1]),
                       reinterpret_cast<int32_t*>(b + off[2]), reinterpret_cast<float*>(b + off[3]),
                       reinterpret_cast<BvhNode*>(b + off[4]), reinterpret_cast<BvhTri*>(b + off[5]) };
        lbvhScratch.resize(lbvhTraversableScratchBytes(numTris));
        bvhMaxDepth = lbvhBuildTraversable(dVerts, numTris, options.bvhTreeletRounds, lbvhScratch.ptr, &lo, nullptr,
                                           stream);
        auto flag = std::make_unique<DeviceBuffer>();
        flag->resize(256);
        ck(cudaMemsetAsync(flag->ptr, 0, 4, stream), "bvh flag");
        sg.bvh = Bvh{ lo.nodes, lo.tris, numTris, flag->as<uint32_t>() };
        sceneBufs.push_back(std::move(flag));
        sceneBufs.push_back(std::move(out));
    }

    // ---- environment (EnvironmentEmitter with an EnvironmentTexture node)
    if (envMat) {
        sg.envMaterial = envMatIndex;
        sg.envRotation = scene->envRotation;
        const Image2D* img = nullptr;
        auto pit = envMat->plugs.find("emittance");
        if (pit != envMat->plugs.end() && pit->second.nodeRef) {
            const auto* node = reinterpret_cast<const ShaderNode*>(pit->second.nodeRef);
            auto iit = node->objects.find("image");
            if (iit != node->objects.end()) img = static_cast<const Image2D*>(iit->second);
        }
        uint32_t w = 1, h = 1;
        std::vector<float> lum;
        // untextured: the immediate emittance everywhere (textured: unused)
        sg.envTexels = upload(std::vector<UpSpec>{ f.mats[envMatIndex].emit }, stream);
        sg.envTex = 0;
        if (img && img->width > 0) {
            w = img->width;
            h = img->height;
            lum.resize(size_t(w) * h);
            // Per texel, the reference's spectral-mode image conversion
            // (image.cpp:542-566): Rec.709 (D65) RGB -> XYZ, b = X + Y + Z,
            // chromaticity -> Meng (u, v), stored with s = b as halves.  The
            // importance map's luminance is the reference's for that format
            // (image.cpp:1010-1017): y(u, v) * s of the stored halves.
            std::vector<__half> uvs(size_t(w) * h * 4);
            for (size_t i = 0; i < lum.size(); ++i) {
                float hu, hv, hs;
                envTexelUVS(&img->rgba[4 * i], &hu, &hv, &hs);
                uvs[4 * i + 0] = __float2half_rn(hu);
                uvs[4 * i + 1] = __float2half_rn(hv);
                uvs[4 * i + 2] = __float2half_rn(hs);
                uvs[4 * i + 3] = __float2half_rn(img->rgba[4 * i + 3]);
                const float su = __half2float(uvs[4 * i + 0]), sv = __half2float(uvs[4 * i + 1]);
                const float sY = 0.022853819546830627f * su + 0.05077639329371236f * sv - 0.006895157122499944f;
                lum[i] = std::fmax(sY * __half2float(uvs[4 * i + 2]), 0.0f);
            }
            // the (u, v, s) image in a texture object the renderers fetch bilinearly
            auto st = std::make_unique<SceneTexture>();
            cudaChannelFormatDesc cd = cudaCreateChannelDescHalf4();
            ck(cudaMallocArray(&st->array, &cd, w, h), "env array");
            ck(cudaMemcpy2DToArray(st->array, 0, 0, uvs.data(), size_t(w) * 8, size_t(w) * 8, h,
                                   cudaMemcpyHostToDevice), "env upload");
            cudaResourceDesc rd{};
            rd.resType = cudaResourceTypeArray;
            rd.res.array.array = st->array;
            cudaTextureDesc td{};
            td.addressMode[0] = cudaAddressModeWrap;
            td.addressMode[1] = cudaAddressModeWrap;
            td.filterMode = cudaFilterModeLinear;
            td.readMode = cudaReadModeElementType;
            td.normalizedCoords = 1;
            ck(cudaCreateTextureObject(&st->tex, &rd, &td, nullptr), "env texture");
            sg.envTex = static_cast<unsigned long long>(st->tex);
            sceneTextures.push_back(std::move(st));
        }
        else {
            lum.push_back(1.0f);
        }
        auto dist = std::make_unique<DeviceBuffer>();
        const size_t bRow = (size_t(h) * (w + 1) * 8 + 255) & ~size_t(255);
        const size_t bMarg = ((h + 1) * 8 + 255) & ~size_t(255);
        const size_t bRowPdf = (size_t(h) * w * 4 + 255) & ~size_t(255);
        const size_t bMargPdf = (h * 4 + 255) & ~size_t(255);
        dist->resize(bRow + bMarg + bRowPdf + bMargPdf);
        char* d = dist->as<char>();
        sg.env.rowCdf = reinterpret_cast<double*>(d);
        sg.env.margCdf = reinterpret_cast<double*>(d + bRow);
        sg.env.rowPdf = reinterpret_cast<float*>(d + bRow + bMarg);
        sg.env.margPdf = reinterpret_cast<float*>(d + bRow + bMarg + bRowPdf);
        sg.env.w = w;
        sg.env.h = h;
        DeviceBuffer scratch;
        scratch.resize(envScratchBytes(w, h));
        buildEnvDistribution(lum.data(), w, h, const_cast<double*>(sg.env.rowCdf), const_cast<double*>(sg.env.margCdf),
                             const_cast<float*>(sg.env.rowPdf), const_cast<float*>(sg.env.margPdf), scratch.ptr, stream);
        ck(cudaStreamSynchronize(stream), "env build");
        sceneBufs.push_back(std::move(dist));
    }
    ck(cudaStreamSynchronize(stream), "scene build");
    builtGeneration = generation;
}

void Context::setupCamera(const Camera* cam) {
    // PerspectiveCamera::setImagePlaneArea (shared/shared.h:895-900) and the
    // quaternion-to-matrix conversion (include/vlr/basic_types.h:1386-1393).
    auto f3 = [&](const char* n, std::vector<float> def) {
        auto it = cam->floats.find(n);
        return it != cam->floats.end() ? it->second : def;
    };
    std::vector<float> pos = f3("position", { 0, 0, 0 });
    std::vector<float> q = f3("orientation", { 0, 0, 0, 1 });
    const float aspect = cam->getFloat("aspect", 1.0f);
    const float fovY = cam->getFloat("fovy", 45 * kPi / 180);
    const float lensRadius = cam->getFloat("lens radius", 1.0f);
    const float sensitivity = cam->getFloat("sensitivity", 1.0f);
    const float objPlaneDistance = cam->getFloat("op distance", 1.0f);
    vlrb::Camera &C = sg.cam;
    C.position = V3(pos[0], pos[1], pos[2]);
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, zx = z * x, xw = x * w, yw = y * w, zw = z * w;
    C.right = V3(1 - 2 * (yy + zz), 2 * (xy + zw), 2 * (zx - yw));
    C.up = V3(2 * (xy - zw), 1 - 2 * (xx + zz), 2 * (yz + xw));
    C.forward = V3(2 * (zx + yw), 2 * (yz - xw), 1 - 2 * (xx + yy));
    C.sensitivity = sensitivity;
    C.lensRadius = lensRadius;
    C.objPlaneDistance = objPlaneDistance;
    C.opHeight = 2.0f * objPlaneDistance * std::tan(fovY * 0.5f);
    C.opWidth = C.opHeight * aspect;
    C.imgPlaneDistance = 1.0f;
    C.imgPlaneArea = C.opWidth * C.opHeight * sq(C.imgPlaneDistance / objPlaneDistance);
    C.kind = kCameraPerspective;
    C.phiAngle = C.thetaAngle = 0.0f;
    if (cam->type == "equirectangular") {
        // EquirectangularCamera::set clamps the angles (scene.cpp:1805-1822);
        // the camera is a point (cameras.cu:226-255)
        C.kind = kCameraEquirectangular;
        C.lensRadius = 0.0f;
        C.sensitivity = std::isfinite(sensitivity) ? std::max(0.0f, sensitivity) : 1.0f;
        C.phiAngle = std::min(std::max(cam->getFloat("h angle", 2 * kPi), 0.01f), 2 * kPi);
        C.thetaAngle = std::min(std::max(cam->getFloat("v angle", kPi), 0.01f), kPi);
    }
}

void Context::ensurePathBuffers(uint32_t paths, uint32_t imageW, uint32_t imageH) {
    const uint64_t seed = options.rngSeed ? options.rngSeed : 591842031321323413ull;
    if (paths <= pathCapacity && seed == pathSeed && imageW == pathSeedW && imageH == pathSeedH) return;
    if (paths > pathCapacity) {
        if (pathCapacity > 0) {
            // keep the running totals across the reallocation
            unsigned long long t[2];
            ck(cudaMemcpy(t, pb.totals, 16, cudaMemcpyDeviceToHost), "totals");
            totalsBase[0] += t[0];
            totalsBase[1] += t[1];
        }
        pathMem.resize(pathBufferBytes(paths));
        carvePathBuffers(pathMem.ptr, paths, &pb);
        ck(cudaMemset(pb.totals, 0, 16), "totals");
        pathCapacity = paths;
    }
    pathSeed = seed;
    pathSeedW = imageW;
    pathSeedH = imageH;
    paths = pathCapacity;
    std::vector<uint64_t> gen(paths), seeds(paths);
    // Per-slot PCG32 states from std::mt19937_64 (context.cpp:1176-1190): the
    // reference seeds pixel y*W+x with the generator's (y*W+x)-th output, so
    // slot p of each full image block takes the output of the pixel it
    // renders (pixelOfPath) and keeps that pixel's stream across launches.
    seedPathRngs(gen.data(), paths, seed);
    const uint32_t pixels = imageW * imageH;
    const uint32_t fullBlocks = pixels ? paths / pixels : 0;
    for (uint32_t p = 0; p < paths; ++p) {
        const uint32_t block = pixels ? p / pixels : 0;
        seeds[p] = block < fullBlocks ? gen[block * pixels + pixelOfPath(p, imageW, imageH)] : gen[p];
    }
    ck(cudaMemcpy(pb.rng, seeds.data(), size_t(paths) * 8, cudaMemcpyHostToDevice), "seed rngs");
}

bool Context::readPixelRngStates(uint64_t* states, uint32_t count) {
    const uint32_t pixels = imgW * imgH;
    if (count > pixels || count > pathCapacity || pathSeedW != imgW || pathSeedH != imgH) return false;
    std::vector<uint64_t> slots(pixels);
    ck(cudaMemcpy(slots.data(), pb.rng, size_t(pixels) * 8, cudaMemcpyDeviceToHost), "read rngs");
    std::vector<uint64_t> byPixel(pixels);
    for (uint32_t p = 0; p < pixels; ++p) byPixel[pixelOfPath(p, imgW, imgH)] = slots[p];
    std::copy(byPixel.begin(), byPixel.begin() + count, states);
    return true;
}

uint64_t Context::lightSeedOf(uint64_t rngSeed) {
    // the reference's constant (context.cpp:618-626) unless the caller chose
    // its own seed: then one derived from it (SplitMix64), so contexts or
    // ranks with different seeds also draw different light subpaths
    if (rngSeed == 0 || rngSeed == 591842031321323413ull) return 459182033132123413ull;
    uint64_t z = rngSeed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

bool Context::persistentScene(uint32_t spp, PersistentScene* out) const {
    const uint32_t pixels = imgW * imgH;
    if (pixels == 0 || pathCapacity < pixels || pathSeedW != imgW || pathSeedH != imgH) return false;
    out->scene = sg;
    out->rng = pb.rng;
    out->film = filmDesc();
    out->totals = pb.totals;
    out->width = imgW;
    out->height = imgH;
    out->stride = width;
    out->spp = spp;
    out->maxPathLength = options.maxPathLength;
    out->firstUnit = 0;
    return true;
}

bool Context::readBounceCounters(uint32_t* counters, uint32_t bounces) {
    if (!pb.counters || bounces > kMaxBounces + 1) return false;
    ck(cudaMemcpy(counters, pb.counters, size_t(bounces) * kCountersPerBounce * 4, cudaMemcpyDeviceToHost),
       "read counters");
    return true;
}

void Context::ensureGuiding(uint32_t paths) {
    const GuidingOptions &g = guiding;
    if (!guideNet || guideNet->net.log2Table != g.log2TableSize) {
        guideNet.reset(new guide::GuideNet(g.log2TableSize, 0x5EED0001ull));
        guideLaunches = 0;
        guidingStats = GuidingStats{};
    }
    const float lo[3] = { sg.bounds.lo.x, sg.bounds.lo.y, sg.bounds.lo.z };
    const float hi[3] = { sg.bounds.hi.x, sg.bounds.hi.y, sg.bounds.hi.z };
    guideNet->setBounds(lo, hi);
    guideNet->weightClamp = g.weightClamp;
    const uint32_t rec = std::min<uint32_t>(std::max<uint32_t>(g.recordBounces, 1u), kMaxRecBounces);
    const uint32_t cap = 2 * g.samplesPerStep;
    if (paths > guideCapacityPaths || rec != guideRecBounces || cap != guideSampleCapacity) {
        guideMem.resize(guideBufferBytes(paths, rec, cap));
        ck(cudaMemset(guideMem.ptr, 0, guideMem.bytes), "guide buffers");
        carveGuideBuffers(guideMem.ptr, paths, rec, cap, &gframe);
        guideCapacityPaths = paths;
        guideRecBounces = rec;
        guideSampleCapacity = cap;
    }
}

uint32_t Context::guideSamplesRecorded() const {
    if (!gframe.counts) return 0;
    uint32_t n = 0;
    ck(cudaMemcpy(&n, gframe.counts, 4, cudaMemcpyDeviceToHost), "guide counts");
    return std::min(n, guideSampleCapacity);
}

// Training steps on the samples the last launch recorded; the sample count
// stays on the device.
void Context::trainGuide(cudaStream_t stream) {
    for (uint32_t s = 0; s < guiding.stepsPerLaunch; ++s) {
        timer.begin(kStageGuide, stream, 64);
        guideNet->gradients(gframe.samples, guideSampleCapacity, stream, gframe.counts);
        guideNet->step(guiding.learningRate, stream);
        timer.end(stream);
        timer.totalLaunches += 5;
        ++guidingStats.trainingSteps;
    }
}

void Context::render(cudaStream_t stream, const Camera* cam, bool firstFrame, uint32_t limitFrames,
                     uint32_t samples, uint32_t* numAccumFramesOut, uint32_t shrink, bool denoise) {
    if (width == 0 || height == 0) throw std::runtime_error("no output buffer bound");
    if (builtGeneration != generation) buildScene(stream);
    if (firstFrame || imgW == 0 || imgW > width || imgH > height) {
        const uint32_t s = std::max<uint32_t>(shrink, 1u);
        imgW = std::max<uint32_t>(width / s, 1u);
        imgH = std::max<uint32_t>(height / s, 1u);
    }
    if (firstFrame) {
        setupCamera(cam);
        numAccumFrames = 0;
        filmClear(filmDesc(), stream);
    }
    const uint32_t pixels = imgW * imgH;
    if (numAccumFrames + samples > limitFrames)
        samples = limitFrames > numAccumFrames ? limitFrames - numAccumFrames : 0;
    Film fl = filmDesc();
    if (samples > 0) {
        uint32_t perLaunch = std::max<uint32_t>(1, std::min<uint32_t>(samples, options.maxPathsInFlight / pixels));
        ensurePathBuffers(pixels * perLaunch, imgW, imgH);
        uint32_t done = 0;
        while (done < samples) {
            uint32_t k = std::min(perLaunch, samples - done);
            FrameParams fp{};
            fp.width = imgW;
            fp.height = imgH;
            fp.stride = width;
            fp.sppPerLaunch = k;
            fp.numPaths = pixels * k;
            fp.maxPathLength = options.maxPathLength;
            fp.blocksPerSM = options.blocksPerSM;
            if (renderer == VLRRenderer_BPT) {
                // One frame per launch: all paths of a frame share its
                // wavelength samples.  Light subpaths per frame default to
                // one per pixel path (the pixel count), and the cache holds
                // ten vertices per light subpath, the reference's ratio
                // (500,000 subpaths, 5,000,000 vertices: context.h:303,
                // context.cpp:628); overflow is counted, see vlrbContextGetStats.
                const uint32_t lightPaths = options.lightPathsPerFrame ? options.lightPathsPerFrame
                                                                       : std::max<uint32_t>(1, pixels);
                const uint32_t capacity = static_cast<uint32_t>(
                    std::min<uint64_t>(uint64_t(10) * lightPaths, 0xFFFFFFFFull / 2));
                const uint64_t lightSeed = lightSeedOf(options.rngSeed);
                const bool reseed = bptLightSeed != lightSeed;
                if (reseed) {
                    bptLightSeed = lightSeed;
                    bptRng.seed(lightSeed);
                }
                if (bptCapacityPaths < lightPaths || bptCapacityVerts < capacity || bptEyeCapacity < pixels || reseed) {
                    bptCapacityPaths = lightPaths;
                    bptCapacityVerts = capacity;
                    bptEyeCapacity = pixels;
                    bptMem.resize(bptBufferBytes(lightPaths, pixels, capacity));
                    carveBptBuffers(bptMem.ptr, lightPaths, pixels, capacity, &lightPb, &bb);
                    std::vector<uint64_t> seeds(lightPaths);
                    // The reference seeds its light-path RNGs from this generator (context.cpp:618-626).
                    seedPathRngs(seeds.data(), lightPaths, lightSeed);
                    ck(cudaMemcpy(lightPb.rng, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice), "seed light rngs");
                    ck(cudaMemset(lightPb.totals, 0, 16), "totals");
                }
                // One common wavelength set per frame from a host generator
                // (context.cpp:1462-1470).
                std::uniform_real_distribution<float> u01(0.0f, 1.0f);
                float wlPdf;
                float o = u01(bptRng), sel = u01(bptRng);
                WLS wls = WLS::equalOffsets(o, sel, &wlPdf);
                FrameParams bf = fp;
                bf.sppPerLaunch = 1;
                bf.numPaths = pixels;
                bptRenderLaunch(sg, pb, lightPb, bb, fl, bf, lightPaths, wls, wlPdf, numSMs, stream, &timer);
                k = 1;
            }
            else if (renderer == VLRRenderer_LightTracing) {
                // One frame per launch: light subpaths per frame default to
                // the pixel count (the reference launches a fixed 500,000,
                // context.h:303); each carries its own wavelength samples.
                // As many frames per launch as the path budget holds.
                const uint32_t lightPaths = options.lightPathsPerFrame ? options.lightPathsPerFrame : pixels;
                const uint32_t frames = std::max<uint32_t>(
                    1u, std::min<uint32_t>(samples - done, options.maxPathsInFlight / lightPaths));
                const uint32_t slots = lightPaths * frames;
                const uint64_t lightSeed = lightSeedOf(options.rngSeed);
                if (ltCapacity < slots || ltLightSeed != lightSeed) {
                    ltLightSeed = lightSeed;
                    ltCapacity = slots;
                    const size_t pathBytes = pathBufferBytes(slots);
                    ltMem.resize(pathBytes + ltConnectionBytes(slots));
                    carvePathBuffers(ltMem.ptr, slots, &ltPb);
                    ltConn = ltMem.as<char>() + pathBytes;
                    std::vector<uint64_t> seeds(slots);
                    seedPathRngs(seeds.data(), slots, lightSeed);
                    ck(cudaMemcpy(ltPb.rng, seeds.data(), seeds.size() * 8, cudaMemcpyHostToDevice), "seed light rngs");
                    ck(cudaMemset(ltPb.totals, 0, 16), "totals");
                }
                FrameParams lf = fp;
                lf.sppPerLaunch = frames;
                lf.numPaths = slots;
                ltRenderLaunch(sg, ltPb, ltConn, fl, lf, lightPaths, frames, numSMs, stream, &timer);
                k = frames;
            }
            else if (guiding.enabled || guiding.train) {
                ensureGuiding(pathCapacity);
                // record and train on every trainInterval-th launch once
                // the warm-up launches are done
                const uint32_t interval = std::max<uint32_t>(guiding.trainInterval, 1u);
                gframe.record = guiding.train &&
                                (guideLaunches < guiding.warmupLaunches || guideLaunches % interval == 0);
                gframe.sample = guiding.enabled && (!guiding.train || guideLaunches >= guiding.warmupLaunches);
                gframe.net = guideNet->net;
                gframe.targetSamples = guiding.samplesPerStep;
                ptRenderLaunch(sg, pb, fl, fp, numSMs, stream, &timer, &gframe);
                if (gframe.sample) ++guidingStats.guidedLaunches;
                if (gframe.record) trainGuide(stream);
                ++guideLaunches;
            }
            else {
                ptRenderLaunch(sg, pb, fl, fp, numSMs, stream, &timer);
            }
            done += k;
        }
        numAccumFrames += samples;
        stats.frames += samples;
    }
    if (samples > 0) filmAddFrames(fl, samples, stream);
    filmToRGBA(fl, output.as<float4>(), stream);
    // Guide buffers (auxBufferGenerator, run with every frame of every
    // renderer in the reference, context.cpp:1440-1530): up to 4 first-hit
    // samples per call; restarted with the accumulation.
    const bool wantAux = denoise || options.auxBuffers;
    if (wantAux) {
        const size_t bytes = auxBufferBytes(width, height);
        if (auxMem.bytes < bytes || aux.stride != width) {
            auxMem.resize(bytes);
            carveAuxBuffers(auxMem.ptr, width, height, &aux);
            auxCurrent = false;
        }
        if (firstFrame || !auxCurrent) {
            auxClear(aux, height, stream);
            auxSamples = 0;
        }
        const uint32_t auxNow = std::min<uint32_t>(std::max<uint32_t>(samples, 1u), 4u);
        auxLaunch(sg, aux, imgW, imgH, auxNow, 0x2545F4914F6CDD1DULL * ++auxSeed, stream);
        auxSamples += auxNow;
        auxToLinear(sg, aux, imgW, imgH, auxSamples, stream);
        if (denoise) denoiseLaunch(aux, output.as<float4>(), imgW, imgH, stream);
    }
    auxCurrent = wantAux;
    ++timer.totalLaunches;
    timer.paramBytes += sizeof(Film) + 4 + 40 + sizeof(void*);
    if (numAccumFramesOut) *numAccumFramesOut = numAccumFrames;
}

std::vector<AutotuneTrial> Context::autotune(cudaStream_t stream, const Camera* cam, uint32_t samplesPerTrial) {
    if (width == 0 || height == 0) throw std::runtime_error("no output buffer bound");
    const RenderOptions saved = options;
    const uint32_t pixels = width * height;
    std::vector<AutotuneTrial> trials;
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    uint32_t frames = 0;
    // Path slots cost ~250 bytes each; candidates stay within half the free
    // device memory, and above the paths one trial renders (pixels x
    // samplesPerTrial) a candidate behaves like the one that holds them all.
    size_t freeBytes = 0, totalBytes = 0;
    ck(cudaMemGetInfo(&freeBytes, &totalBytes), "memory info");
    const uint64_t trialPaths = uint64_t(pixels) * samplesPerTrial;
    for (uint32_t paths : { 1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25 }) {
        // below one sample per pixel per launch the candidate equals the
        // smallest one that holds a full frame
        if (paths < pixels && !trials.empty() && trials.back().maxPathsInFlight >= pixels) continue;
        if (!trials.empty() && uint64_t(trials.back().maxPathsInFlight) >= trialPaths) break;
        if (!trials.empty() && uint64_t(std::max(paths, pixels)) * 256 > freeBytes / 2) break;
        for (uint32_t bps : { 4u, 8u, 16u, 32u }) {
            options.maxPathsInFlight = std::max(paths, pixels);
            options.blocksPerSM = bps;
            render(stream, cam, true, 1u << 30, samplesPerTrial, &frames);    // warm-up / allocation
            unsigned long long t0[2], t1[2];
            ck(cudaStreamSynchronize(stream), "sync");
            ck(cudaMemcpy(t0, pb.totals, 16, cudaMemcpyDeviceToHost), "totals");
            ck(cudaEventRecord(e0, stream), "record");
            render(stream, cam, false, 1u << 30, samplesPerTrial, &frames);
            ck(cudaEventRecord(e1, stream), "record");
            ck(cudaEventSynchronize(e1), "sync");
            ck(cudaMemcpy(t1, pb.totals, 16, cudaMemcpyDeviceToHost), "totals");
            float ms = 0.0f;
            ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
            trials.push_back({ options.maxPathsInFlight, bps, double(t1[0] - t0[0]) / (ms * 1e-3) });
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    options = saved;
    const AutotuneTrial* best = &trials[0];
    for (const auto &t : trials)
        if (t.segmentsPerSecond > best->segmentsPerSecond) best = &t;
    options.maxPathsInFlight = best->maxPathsInFlight;
    options.blocksPerSM = best->blocksPerSM;
    return trials;
}

RenderBatch::RenderBatch(std::vector<BatchItem> its, cudaStream_t stream, bool persistentMode)
    : items(std::move(its)), persistent(persistentMode) {
    for (const BatchItem &it : items) {
        if (!it.ctx || !it.cam || it.samples == 0) throw std::runtime_error("batch item without context, camera or samples");
        if (it.ctx->renderer != VLRRenderer_PathTracing) throw std::runtime_error("batch rendering is path tracing only");
    }
    const size_t n = items.size();
    streams.resize(n);
    evBegin.resize(n);
    evEnd.resize(n);
    evJoin.resize(n);
    // Each item's stream gets a priority by its work (pixels x samples): the
    // smallest items the highest, so the block scheduler starts their kernels
    // first and short frames are not held behind long ones.  The captured
    // nodes keep their stream's priority (instantiated with node priorities).
    int leastPrio = 0, greatestPrio = 0;
    ck(cudaDeviceGetStreamPriorityRange(&leastPrio, &greatestPrio), "priority range");
    std::vector<uint32_t> byWork(n);
    for (size_t i = 0; i < n; ++i) byWork[i] = static_cast<uint32_t>(i);
    auto itemWork = [&](uint32_t i) {
        const Context* c = items[i].ctx;
        return uint64_t(c->width) * c->height * items[i].samples;
    };
    std::stable_sort(byWork.begin(), byWork.end(), [&](uint32_t a, uint32_t b) { return itemWork(a) < itemWork(b); });
    std::vector<int> prio(n, leastPrio);
    const int levels = leastPrio - greatestPrio + 1;
    for (size_t r = 0; r < n; ++r)
        prio[byWork[r]] = greatestPrio + static_cast<int>(r * levels / n);
    for (size_t i = 0; i < n; ++i) {
        ck(cudaStreamCreateWithPriority(&streams[i], cudaStreamNonBlocking, prio[i]), "batch stream");
        ck(cudaEventCreate(&evBegin[i]), "event");
        ck(cudaEventCreate(&evEnd[i]), "event");
        ck(cudaEventCreateWithFlags(&evJoin[i], cudaEventDisableTiming), "event");
    }
    ck(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
    // One plain render per item outside capture: builds scenes, allocates
    // path and guiding buffers, and gets guided contexts past their warm-up.
    for (BatchItem &it : items) {
        const bool profiling = it.ctx->timer.enabled;
        it.ctx->timer.enabled = false;
        uint32_t frames;
        const uint32_t warm = it.ctx->guiding.train ? std::max(it.samples, it.ctx->guiding.warmupLaunches) : it.samples;
        it.ctx->render(stream, it.cam, true, 1u << 30, warm, &frames);
        it.ctx->timer.enabled = profiling;
    }
    ck(cudaStreamSynchronize(stream), "batch warm-up");
    slotOfItem.assign(n, ~0u);
    if (persistent) {
        for (size_t i = 0; i < n; ++i) {
            const Context* c = items[i].ctx;
            if (!(c->guiding.enabled || c->guiding.train)) plainOrder.push_back(static_cast<uint32_t>(i));
        }
        auto cost = [&](uint32_t i) { return uint64_t(items[i].ctx->imgW) * items[i].ctx->imgH * items[i].samples; };
        std::stable_sort(plainOrder.begin(), plainOrder.end(), [&](uint32_t a, uint32_t b) { return cost(a) < cost(b); });
        std::vector<PersistentScene> ps(plainOrder.size());
        unsigned long long units = 0;
        for (size_t k = 0; k < plainOrder.size(); ++k) {
            BatchItem &it = items[plainOrder[k]];
            if (!it.ctx->persistentScene(it.samples, &ps[k]))
                throw std::runtime_error("batch item without path buffers for its image");
            ps[k].firstUnit = units;
            units += uint64_t(ps[k].width) * ps[k].height;
            maps = maps || it.ctx->shadingNeedsMaps();
            slotOfItem[plainOrder[k]] = static_cast<uint32_t>(k);
        }
        if (!ps.empty()) {
            scenesBuf.resize(ps.size() * sizeof(PersistentScene));
            ck(cudaMemcpy(scenesBuf.ptr, ps.data(), ps.size() * sizeof(PersistentScene), cudaMemcpyHostToDevice),
               "persistent scenes");
            countersBuf.resize(persistentCounterBytes(static_cast<uint32_t>(ps.size())));
            work = persistentWorkDesc(scenesBuf.as<PersistentScene>(), static_cast<uint32_t>(ps.size()), units,
                                      countersBuf.ptr);
            grid = persistentGrid(items[plainOrder[0]].ctx->numSMs, maps);
            ck(cudaStreamCreateWithFlags(&pStream, cudaStreamNonBlocking), "persistent stream");
            ck(cudaEventCreateWithFlags(&pJoin, cudaEventDisableTiming), "event");
        }
    }
    // Captured on a stream of its own: the caller's may be the legacy default
    // stream, which cannot be captured.  Launches go to the caller's stream.
    ck(cudaStreamCreateWithFlags(&captureStream, cudaStreamNonBlocking), "capture stream");
    ck(cudaStreamBeginCapture(captureStream, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        ck(cudaEventRecord(fork, captureStream), "fork");
        if (!plainOrder.empty()) {
            ck(cudaStreamWaitEvent(pStream, fork, 0), "wait fork");
            for (uint32_t i : plainOrder)
                if (items[i].firstFrame) items[i].ctx->clearFilm(pStream);
            persistentPtLaunch(work, maps, grid, pStream);
            for (uint32_t i : plainOrder) items[i].ctx->convertFilm(pStream);
            ck(cudaEventRecord(pJoin, pStream), "join");
            ck(cudaStreamWaitEvent(captureStream, pJoin, 0), "wait join");
        }
        for (size_t i = 0; i < n; ++i) {
            BatchItem &it = items[i];
            if (slotOfItem[i] != ~0u) continue;
            ck(cudaStreamWaitEvent(streams[i], fork, 0), "wait fork");
            ck(cudaEventRecordWithFlags(evBegin[i], streams[i], cudaEventRecordExternal), "begin");
            const bool profiling = it.ctx->timer.enabled;
            it.ctx->timer.enabled = false;
            uint32_t frames;
            it.ctx->render(streams[i], it.cam, it.firstFrame, 1u << 30, it.samples, &frames);
            it.ctx->timer.enabled = profiling;
            ck(cudaEventRecordWithFlags(evEnd[i], streams[i], cudaEventRecordExternal), "end");
            ck(cudaEventRecord(evJoin[i], streams[i]), "join");
            ck(cudaStreamWaitEvent(captureStream, evJoin[i], 0), "wait join");
        }
    }
    catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(captureStream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    ck(cudaStreamEndCapture(captureStream, &graph), "end capture");
    ck(cudaGraphInstantiateWithFlags(&exec, graph, cudaGraphInstantiateFlagUseNodePriority), "instantiate");
}

RenderBatch::~RenderBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto s : streams) cudaStreamDestroy(s);
    for (auto e : evBegin) cudaEventDestroy(e);
    for (auto e : evEnd) cudaEventDestroy(e);
    for (auto e : evJoin) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (captureStream) cudaStreamDestroy(captureStream);
    if (pStream) cudaStreamDestroy(pStream);
    if (pJoin) cudaEventDestroy(pJoin);
}

void RenderBatch::launch(cudaStream_t stream) {
    ck(cudaGraphLaunch(exec, stream), "graph launch");
    // host-side bookkeeping the replayed graph cannot do
    for (BatchItem &it : items) {
        it.ctx->numAccumFrames = it.firstFrame ? it.samples : it.ctx->numAccumFrames + it.samples;
        it.ctx->stats.frames += it.samples;
    }
}

void RenderBatch::itemTimes(std::vector<float>* ms) const {
    ms->resize(items.size());
    std::vector<unsigned long long> ends(plainOrder.size());
    unsigned long long start = 0;
    if (!plainOrder.empty()) {
        // the persistent items: each scene's last pixel against the launch's start
        ck(cudaStreamSynchronize(pStream), "sync");
        ck(cudaMemcpy(&start, work.startNs, 8, cudaMemcpyDeviceToHost), "start stamp");
        ck(cudaMemcpy(ends.data(), work.endNs, ends.size() * 8, cudaMemcpyDeviceToHost), "end stamps");
    }
    for (size_t i = 0; i < items.size(); ++i) {
        if (slotOfItem[i] != ~0u) {
            (*ms)[i] = static_cast<float>(double(ends[slotOfItem[i]] - start) * 1e-6);
            continue;
        }
        ck(cudaEventSynchronize(evEnd[i]), "sync");
        ck(cudaEventElapsedTime(&(*ms)[i], evBegin[i], evEnd[i]), "elapsed");
    }
}

void Context::readStats(RenderStats* out) {
    unsigned long long t[2] = { 0, 0 };
    if (pathCapacity > 0) ck(cudaMemcpy(t, pb.totals, 16, cudaMemcpyDeviceToHost), "stats");
    unsigned long long tl[2] = { 0, 0 };
    if (bptCapacityPaths > 0) ck(cudaMemcpy(tl, lightPb.totals, 16, cudaMemcpyDeviceToHost), "light stats");
    unsigned long long tt[2] = { 0, 0 };
    if (ltCapacity > 0) ck(cudaMemcpy(tt, ltPb.totals, 16, cudaMemcpyDeviceToHost), "light tracing stats");
    tl[0] += tt[0];
    tl[1] += tt[1];
    *out = stats;
    if (sg.bvh.errorFlag) {
        uint32_t e = 0;
        ck(cudaMemcpy(&e, sg.bvh.errorFlag, 4, cudaMemcpyDeviceToHost), "bvh flag");
        if (e & 1u) throw std::runtime_error("BVH traversal met an out-of-range node reference");
        if (e & 2u) throw std::runtime_error("BVH traversal stack overflowed (a hierarchy deeper than 64 levels)");
    }
    out->segments = t[0] + tl[0] + totalsBase[0];
    out->shadowRays = t[1] + tl[1] + totalsBase[1];
    if (bptCapacityPaths > 0) {
        uint32_t c[2];
        ck(cudaMemcpy(c, bb.counters, 8, cudaMemcpyDeviceToHost), "overflow");
        out->lightVertexOverflow = c[1];
    }
}

} // namespace api
} // namespace vlrb
