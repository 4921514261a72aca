// The VLR C API (include/vlr/vlr.h) over the host object model.
//
// Error behaviour follows the reference's C layer (libVLR/vlr.cpp:13-34):
// a null handle is VLRResult_InvalidArgument, a handle of the wrong kind is
// VLRResult_InvalidInstance, an exception becomes VLRResult_InternalError.
#include "context.cuh"
#include "tables.cuh"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

using namespace vlrb;
using namespace vlrb::api;

namespace vlrb {
namespace api {

std::string lower(const std::string &s) {
    std::string r(s);
    for (char &c : r) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return r;
}

void Queryable::addParam(const char* name, uint32_t form, const char* type, uint32_t tuple) {
    auto p = std::make_unique<ParameterInfoObj>();
    p->typeName = "ParameterInfo";
    p->info = ParamInfo{ name, form, type, tuple };
    p->ctx = ctx;
    infos.push_back(std::move(p));
}

const ParamInfo* Queryable::find(const std::string &name) const {
    const std::string l = lower(name);
    for (const auto &p : infos)
        if (lower(p->info.name) == l) return &p->info;
    return nullptr;
}

float Queryable::getFloat(const char* name, float def) const {
    auto it = floats.find(lower(name));
    return (it != floats.end() && !it->second.empty()) ? it->second[0] : def;
}

bool SurfaceMaterial::isEmitting() const {
    const std::string t = lower(typeName);
    return t == "diffuseemitter" || t == "environmentemitter" || t == "directionalemitter" || t == "pointemitter";
}

bool isImage(const Object* o) { return o->kind == Kind::LinearImage2D || o->kind == Kind::BlockCompressedImage2D; }
bool isQueryable(const Object* o) {
    return isImage(o) || o->kind == Kind::ShaderNode || o->kind == Kind::SurfaceMaterial || o->kind == Kind::Camera;
}
bool isParentNode(const Object* o) { return o->kind == Kind::InternalNode || o->kind == Kind::Scene; }
bool isNode(const Object* o) {
    return isParentNode(o) || o->kind == Kind::TriangleMeshSurfaceNode || o->kind == Kind::PointSurfaceNode;
}

} // namespace api
} // namespace vlrb

namespace {

constexpr uint32_t kImm = VLRParameterFormFlag_ImmediateValue, kNode = VLRParameterFormFlag_Node,
                   kBoth = VLRParameterFormFlag_Both;

// Enum tables (queryable.cpp:31-104).
const std::vector<std::pair<std::string, std::vector<const char*>>> &enumTables() {
    static const std::vector<std::pair<std::string, std::vector<const char*>>> t = {
        { "SpectrumType", { "Reflectance", "Transmittance", "Light Source", "NA" } },
        { "ColorSpace", { "Rec709(D65) sRGB Gamma", "Rec709(D65)", "XYZ", "xyY" } },
        { "DataFormat", { "RGB8x3", "RGB_8x4", "RGBA8x4", "RGBA16Fx4", "RGBA32Fx4", "RG32Fx2", "Gray32F", "Gray8",
                          "GrayA8x2", "BC1", "BC2", "BC3", "BC4", "BC4_Signed", "BC5", "BC5_Signed", "BC6H",
                          "BC6H_Signed", "BC7" } },
        { "BumpType", { "Normal Map (DirectX)", "Normal Map (OpenGL)", "Height Map" } },
        { "TextureFilter", { "Nearest", "Linear", "None" } },
        { "TextureWrapMode", { "Repeat", "Clamp to Edge", "Mirror", "Clamp to Border" } },
        { "TangentType", { "TC0 Direction", "Radial X", "Radial Y", "Radial Z" } },
    };
    return t;
}

const std::vector<const char*>* enumMembers(const std::string &type) {
    for (const auto &e : enumTables())
        if (e.first == type) return &e.second;
    return nullptr;
}

void setSpectrumDefault(Queryable* q, const char* name, float v0, float v1, float v2) {
    ImmSpectrum s;
    s.colorSpace = "Rec709(D65)";
    s.e[0] = v0; s.e[1] = v1; s.e[2] = v2;
    q->spectra[lower(name)] = s;
}

// Parameter tables and defaults of each material (libVLR/materials.cpp
// initialize() lists and constructors).
bool initMaterial(SurfaceMaterial* m, const std::string &type) {
    const std::string t = lower(type);
    const float pi = kPi;
    if (t == "matte") {
        m->addParam("albedo", kBoth, "Spectrum");
        setSpectrumDefault(m, "albedo", 0.18f, 0.18f, 0.18f);
    }
    else if (t == "specularreflection") {
        m->addParam("coeff", kBoth, "Spectrum");
        m->addParam("eta", kBoth, "Spectrum");
        m->addParam("k", kBoth, "Spectrum");
        setSpectrumDefault(m, "coeff", 0.8f, 0.8f, 0.8f);
        setSpectrumDefault(m, "eta", 1.0f, 1.0f, 1.0f);
        setSpectrumDefault(m, "k", 0.0f, 0.0f, 0.0f);
    }
    else if (t == "specularscattering") {
        m->addParam("coeff", kBoth, "Spectrum");
        m->addParam("eta ext", kBoth, "Spectrum");
        m->addParam("eta int", kBoth, "Spectrum");
        setSpectrumDefault(m, "coeff", 0.8f, 0.8f, 0.8f);
        setSpectrumDefault(m, "eta ext", 1.0f, 1.0f, 1.0f);
        setSpectrumDefault(m, "eta int", 1.5f, 1.5f, 1.5f);
    }
    else if (t == "microfacetreflection") {
        m->addParam("eta", kBoth, "Spectrum");
        m->addParam("k", kBoth, "Spectrum");
        m->addParam("roughness/anisotropy/rotation", kNode, "Float", 3);
        m->addParam("roughness", kImm, "Float");
        m->addParam("anisotropy", kImm, "Float");
        m->addParam("rotation", kImm, "Float");
        setSpectrumDefault(m, "eta", 1.0f, 1.0f, 1.0f);
        setSpectrumDefault(m, "k", 0.0f, 0.0f, 0.0f);
        m->floats["roughness"] = { 0.1f };
        m->floats["anisotropy"] = { 0.0f };
        m->floats["rotation"] = { 0.0f };
    }
    else if (t == "microfacetscattering") {
        m->addParam("coeff", kBoth, "Spectrum");
        m->addParam("eta ext", kBoth, "Spectrum");
        m->addParam("eta int", kBoth, "Spectrum");
        m->addParam("roughness/anisotropy/rotation", kNode, "Float", 3);
        m->addParam("roughness", kImm, "Float");
        m->addParam("anisotropy", kImm, "Float");
        m->addParam("rotation", kImm, "Float");
        setSpectrumDefault(m, "coeff", 0.8f, 0.8f, 0.8f);
        setSpectrumDefault(m, "eta ext", 1.0f, 1.0f, 1.0f);
        setSpectrumDefault(m, "eta int", 1.5f, 1.5f, 1.5f);
        m->floats["roughness"] = { 0.1f };
        m->floats["anisotropy"] = { 0.0f };
        m->floats["rotation"] = { 0.0f };
    }
    else if (t == "lambertianscattering") {
        m->addParam("coeff", kBoth, "Spectrum");
        m->addParam("f0", kBoth, "Float");
        setSpectrumDefault(m, "coeff", 0.8f, 0.8f, 0.8f);
        m->floats["f0"] = { 0.04f };
    }
    else if (t == "ue4") {
        m->addParam("base color", kBoth, "Spectrum");
        m->addParam("occlusion/roughness/metallic", kNode, "Float", 3);
        m->addParam("occlusion", kImm, "Float");
        m->addParam("roughness", kImm, "Float");
        m->addParam("metallic", kImm, "Float");
        setSpectrumDefault(m, "base color", 0.18f, 0.18f, 0.18f);
        m->floats["occlusion"] = { 0.0f };
        m->floats["roughness"] = { 0.1f };
        m->floats["metallic"] = { 0.0f };
    }
    else if (t == "diffuseemitter" || t == "environmentemitter") {
        m->addParam("emittance", kBoth, "Spectrum");
        m->addParam("scale", kImm, "Float");
        setSpectrumDefault(m, "emittance", pi, pi, pi);
        m->floats["scale"] = { 1.0f };
    }
    else if (t == "pointemitter") {
        // PointEmitterSurfaceMaterial (materials.cpp:1900-1945)
        m->addParam("intensity", kBoth, "Spectrum");
        m->addParam("scale", kImm, "Float");
        setSpectrumDefault(m, "intensity", pi, pi, pi);
        m->floats["scale"] = { 1.0f };
    }
    else if (t == "directionalemitter") {
        // DirectionalEmitterSurfaceMaterial (materials.cpp:1729-1763)
        m->addParam("emittance", kBoth, "Spectrum");
        m->addParam("scale", kImm, "Float");
        m->addParam("direction", kBoth, "Vector3D");
        setSpectrumDefault(m, "emittance", pi, pi, pi);
        m->floats["scale"] = { 1.0f };
        m->floats["direction"] = { 0.0f, 0.0f, 1.0f };
    }
    else if (t == "multi") {
        // MultiSurfaceMaterial (materials.cpp:2055-2160): up to four sub-materials "0".."3"
        for (const char* k : { "0", "1", "2", "3" }) m->addParam(k, kNode, "SurfaceMaterial");
    }
    else {
        // OldStyle: not rendered here.
        return false;
    }
    return true;
}

bool initShaderNode(ShaderNode* n, const std::string &type) {
    const std::string t = lower(type);
    if (t == "environmenttexture") {
        n->addParam("image", kNode, "Image");
        n->addParam("min filter", kImm, "TextureFilter");
        n->addParam("mag filter", kImm, "TextureFilter");
        n->enums["min filter"] = "Linear";
        n->enums["mag filter"] = "Linear";
        return true;
    }
    if (t == "image2dtexture") {
        // Image2DTextureShaderNode parameters and defaults (shader_nodes.cpp:1593-1647);
        // its Spectrum plug drives a material's colour parameters
        n->addParam("image", kNode, "Image");
        n->addParam("bump type", kImm, "BumpType");
        n->addParam("bump coeff", kImm, "Float");
        n->addParam("min filter", kImm, "TextureFilter");
        n->addParam("mag filter", kImm, "TextureFilter");
        n->addParam("wrap u", kImm, "TextureWrapMode");
        n->addParam("wrap v", kImm, "TextureWrapMode");
        n->addParam("texcoord", kNode, "TextureCoordinates");
        n->enums["bump type"] = "Normal Map (DirectX)";
        n->floats["bump coeff"] = { 1.0f };
        n->enums["min filter"] = "Linear";
        n->enums["mag filter"] = "Linear";
        n->enums["wrap u"] = "Repeat";
        n->enums["wrap v"] = "Repeat";
        return true;
    }
    if (t == "tripletspectrum") {
        n->addParam("spectrum type", kImm, "SpectrumType");
        n->addParam("color space", kImm, "ColorSpace");
        n->addParam("triplet", kImm, "Float", 3);
        n->enums["spectrum type"] = "Reflectance";
        n->enums["color space"] = "Rec709(D65)";
        n->floats["triplet"] = { 0.18f, 0.18f, 0.18f };
        return true;
    }
    return false;
}

bool initCamera(api::Camera* c, const std::string &type) {
    const std::string t = lower(type);
    if (t == "equirectangular") {
        // EquirectangularCamera parameters and defaults (scene.cpp:1680-1725)
        c->type = t;
        c->addParam("position", kImm, "Point3D");
        c->addParam("orientation", kImm, "Quaternion");
        c->addParam("sensitivity", kImm, "Float");
        c->addParam("h angle", kImm, "Float");
        c->addParam("v angle", kImm, "Float");
        c->floats["position"] = { 0, 0, 0 };
        c->floats["orientation"] = { 0, 0, 0, 1 };
        c->floats["sensitivity"] = { 1.0f };
        c->floats["h angle"] = { 2 * kPi };
        c->floats["v angle"] = { kPi };
        return true;
    }
    if (t != "perspective") return false;
    c->type = t;
    c->addParam("position", kImm, "Point3D");
    c->addParam("orientation", kImm, "Quaternion");
    c->addParam("aspect", kImm, "Float");
    c->addParam("sensitivity", kImm, "Float");
    c->addParam("fovy", kImm, "Float");
    c->addParam("lens radius", kImm, "Float");
    c->addParam("op distance", kImm, "Float");
    // PerspectiveCamera constructor defaults (scene.cpp:1515-1524).
    c->floats["position"] = { 0, 0, 0 };
    c->floats["orientation"] = { 0, 0, 0, 1 };
    c->floats["aspect"] = { 1.0f };
    c->floats["fovy"] = { 45 * kPi / 180 };
    c->floats["lens radius"] = { 1.0f };
    c->floats["sensitivity"] = { 1.0f };
    c->floats["op distance"] = { 1.0f };
    return true;
}

template <typename T>
T* checked(const void* h, VLRResult* err, bool (*kindOk)(const Object*)) {
    if (!h) { *err = VLRResult_InvalidArgument; return nullptr; }
    auto* o = reinterpret_cast<Object*>(const_cast<void*>(h));
    if (o->magic != kMagic || !kindOk(o)) { *err = VLRResult_InvalidInstance; return nullptr; }
    return static_cast<T*>(o);
}

bool kindContext(const Object* o) { return o->kind == Kind::Context; }
bool kindMaterial(const Object* o) { return o->kind == Kind::SurfaceMaterial; }
bool kindShaderNode(const Object* o) { return o->kind == Kind::ShaderNode; }
bool kindCamera(const Object* o) { return o->kind == Kind::Camera; }
bool kindTransform(const Object* o) { return o->kind == Kind::StaticTransform; }
bool kindMesh(const Object* o) { return o->kind == Kind::TriangleMeshSurfaceNode; }
bool kindPoint(const Object* o) { return o->kind == Kind::PointSurfaceNode; }
bool kindInternal(const Object* o) { return o->kind == Kind::InternalNode; }
bool kindScene(const Object* o) { return o->kind == Kind::Scene; }
bool kindParamInfo(const Object* o) { return o->kind == Kind::ParameterInfo; }
bool kindAny(const Object*) { return true; }

#define CHECK_HANDLE(var, T, pred, h)            \
    VLRResult _err = VLRResult_NoError;          \
    T* var = checked<T>(h, &_err, pred);         \
    if (!var) return _err

#define API_TRY try {
#define API_CATCH(name)                                               \
    }                                                                 \
    catch (const std::exception &ex) {                                \
        cudaGetLastError(); /* a failed call must not leak into the next */ \
        std::fprintf(stderr, "%s: %s\n", name, ex.what());            \
        return VLRResult_InternalError;                               \
    }

void touch(Object* o) {
    if (o && o->ctx) o->ctx->markDirty();
}

} // namespace

extern "C" {

const char* vlrGetErrorMessage(VLRResult code) {
    switch (code) {
    case VLRResult_NoError: return "No Error";
    case VLRResult_InvalidContext: return "Invalid Context";
    case VLRResult_InvalidInstance: return "Invalid Instance";
    case VLRResult_InvalidArgument: return "Invalid Argument";
    case VLRResult_IncompatibleNodeType: return "Incompatible Node Type";
    case VLRResult_InternalError: return "Internal Error";
    default: return "Unknown Error";
    }
}

// ---------------------------------------------------------------- context
VLRResult vlrCreateContext(CUcontext cuContext, bool logging, uint32_t maxCallableDepth, VLRContext* context) {
    (void)maxCallableDepth;
    if (!context) return VLRResult_InvalidArgument;
    API_TRY
    if (cuContext) {
        // Make the caller's context current through the driver entry point the
        // runtime exposes (no link-time libcuda dependency).
        using SetCurrentFn = CUresult (*)(CUcontext);
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxSetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
            return VLRResult_InvalidContext;
        if (reinterpret_cast<SetCurrentFn>(fn)(cuContext) != CUDA_SUCCESS) return VLRResult_InvalidContext;
    }
    *context = reinterpret_cast<VLRContext>(static_cast<Object*>(new Context(cuContext, logging)));
    return VLRResult_NoError;
    API_CATCH("vlrCreateContext")
}

VLRResult vlrDestroyContext(VLRContext context) {
    CHECK_HANDLE(c, Context, kindContext, context);
    API_TRY
    delete c;
    return VLRResult_NoError;
    API_CATCH("vlrDestroyContext")
}

VLRResult vlrContextGetCUcontext(VLRContext context, CUcontext* cuContext) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!cuContext) return VLRResult_InvalidArgument;
    *cuContext = c->cuContext;
    return VLRResult_NoError;
}

VLRResult vlrContextBindOutputBuffer(VLRContext context, uint32_t width, uint32_t height, uint32_t glTexID) {
    CHECK_HANDLE(c, Context, kindContext, context);
    // Graphics interop (glTexID > 0, context.cpp:1145-1159) does not exist
    // here: the output is a device buffer.
    if (glTexID != 0 || width == 0 || height == 0) return VLRResult_InvalidArgument;
    API_TRY
    c->bindOutput(width, height);
    return VLRResult_NoError;
    API_CATCH("vlrContextBindOutputBuffer")
}

VLRResult vlrContextGetOutputBufferSize(VLRContext context, uint32_t* width, uint32_t* height) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!width || !height) return VLRResult_InvalidArgument;
    *width = c->width;
    *height = c->height;
    return VLRResult_NoError;
}

VLRResult vlrContextGetOutputBuffer(VLRContext context, CUarray* array) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!array) return VLRResult_InvalidArgument;
    API_TRY
    *array = c->outputArray();
    return VLRResult_NoError;
    API_CATCH("vlrContextGetOutputBuffer")
}

VLRResult vlrContextReadOutputBuffer(VLRContext context, float* data) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!data || c->width == 0) return VLRResult_InvalidArgument;
    API_TRY
    c->readOutput(data);
    return VLRResult_NoError;
    API_CATCH("vlrContextReadOutputBuffer")
}

VLRResult vlrContextSetScene(VLRContext context, VLRScene scene) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    Scene* s = checked<Scene>(scene, &e2, kindScene);
    if (!s) return e2;
    c->setScene(s);
    return VLRResult_NoError;
}

VLRResult vlrContextSetRenderer(VLRContext context, enum VLRRenderer renderer) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (renderer != VLRRenderer_PathTracing && renderer != VLRRenderer_BPT && renderer != VLRRenderer_LightTracing)
        return VLRResult_InvalidArgument;
    c->renderer = renderer;
    return VLRResult_NoError;
}

VLRResult vlrContextSetDebugRenderingAttribute(VLRContext context, enum VLRDebugRenderingMode attr) {
    CHECK_HANDLE(c, Context, kindContext, context);
    (void)c;
    (void)attr;
    return VLRResult_NoError;
}

VLRResult vlrContextSetProbePixel(VLRContext context, int32_t x, int32_t y) {
    CHECK_HANDLE(c, Context, kindContext, context);
    (void)c; (void)x; (void)y;
    return VLRResult_NoError;
}

VLRResult vlrContextRender(VLRContext context, CUstream stream, VLRCameraConst camera, bool denoise,
                           uint32_t shrinkCoeff, bool firstFrame, uint32_t limitNumAccumFrames,
                           uint32_t* numAccumFrames) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    const api::Camera* cam = checked<const api::Camera>(camera, &e2, kindCamera);
    if (!cam || !numAccumFrames) return VLRResult_InvalidArgument;
    if (shrinkCoeff == 0) return VLRResult_InvalidArgument;
    API_TRY
    // denoise: the guided wavelet denoiser stands in for the OptiX one
    c->render(reinterpret_cast<cudaStream_t>(stream), cam, firstFrame, limitNumAccumFrames, 1, numAccumFrames,
              shrinkCoeff, denoise);
    return VLRResult_NoError;
    API_CATCH("vlrContextRender")
}

// ---------------------------------------------------------------- object / parameter info / enums
VLRResult vlrObjectGetType(VLRObjectConst object, const char** typeName) {
    CHECK_HANDLE(o, Object, kindAny, object);
    if (!typeName) return VLRResult_InvalidArgument;
    *typeName = o->typeName.c_str();
    return VLRResult_NoError;
}

VLRResult vlrParameterInfoGetName(VLRParameterInfoConst paramInfo, const char** name) {
    CHECK_HANDLE(p, ParameterInfoObj, kindParamInfo, paramInfo);
    if (!name) return VLRResult_InvalidArgument;
    *name = p->info.name.c_str();
    return VLRResult_NoError;
}

VLRResult vlrParameterInfoGetSocketForm(VLRParameterInfoConst paramInfo, enum VLRParameterFormFlag* form) {
    CHECK_HANDLE(p, ParameterInfoObj, kindParamInfo, paramInfo);
    if (!form) return VLRResult_InvalidArgument;
    *form = static_cast<VLRParameterFormFlag>(p->info.form);
    return VLRResult_NoError;
}

VLRResult vlrParameterInfoGetType(VLRParameterInfoConst paramInfo, const char** type) {
    CHECK_HANDLE(p, ParameterInfoObj, kindParamInfo, paramInfo);
    if (!type) return VLRResult_InvalidArgument;
    *type = p->info.type.c_str();
    return VLRResult_NoError;
}

VLRResult vlrParameterInfoGetTupleSize(VLRParameterInfoConst paramInfo, uint32_t* size) {
    CHECK_HANDLE(p, ParameterInfoObj, kindParamInfo, paramInfo);
    if (!size) return VLRResult_InvalidArgument;
    *size = p->info.tupleSize;
    return VLRResult_NoError;
}

VLRResult vlrGetNumEnumMembers(const char* typeName, uint32_t* numMembers) {
    if (!typeName || !numMembers) return VLRResult_InvalidArgument;
    const auto* m = enumMembers(typeName);
    if (!m) return VLRResult_InvalidArgument;
    *numMembers = static_cast<uint32_t>(m->size());
    return VLRResult_NoError;
}

VLRResult vlrGetEnumMember(const char* typeName, uint32_t index, const char** value) {
    if (!typeName || !value) return VLRResult_InvalidArgument;
    const auto* m = enumMembers(typeName);
    if (!m || index >= m->size()) return VLRResult_InvalidArgument;
    *value = (*m)[index];
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- queryable
VLRResult vlrQueryableGetNumParameters(VLRQueryableConst queryable, uint32_t* numParams) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!numParams) return VLRResult_InvalidArgument;
    *numParams = static_cast<uint32_t>(q->infos.size());
    return VLRResult_NoError;
}

VLRResult vlrQueryableGetParameterInfo(VLRQueryableConst queryable, uint32_t index, VLRParameterInfoConst* paramInfo) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramInfo || index >= q->infos.size()) return VLRResult_InvalidArgument;
    *paramInfo = reinterpret_cast<VLRParameterInfoConst>(static_cast<const Object*>(q->infos[index].get()));
    return VLRResult_NoError;
}

namespace {
// Looks up a parameter of the expected type; InvalidArgument otherwise.
const ParamInfo* paramOf(const Queryable* q, const char* name, const char* type) {
    if (!name) return nullptr;
    const ParamInfo* p = q->find(name);
    if (!p || p->type != type) return nullptr;
    return p;
}
VLRResult getFloats(const Queryable* q, const char* name, const char* type, float* out, uint32_t n) {
    if (!out || !paramOf(q, name, type)) return VLRResult_InvalidArgument;
    auto it = q->floats.find(lower(name));
    if (it == q->floats.end()) return VLRResult_InvalidArgument;
    for (uint32_t i = 0; i < n; ++i) out[i] = i < it->second.size() ? it->second[i] : 0.0f;
    return VLRResult_NoError;
}
VLRResult setFloats(Queryable* q, const char* name, const char* type, const float* in, uint32_t n) {
    if (!in || !paramOf(q, name, type)) return VLRResult_InvalidArgument;
    for (uint32_t i = 0; i < n; ++i) if (!std::isfinite(in[i])) return VLRResult_InvalidArgument;
    q->floats[lower(name)] = std::vector<float>(in, in + n);
    if (q->kind != Kind::Camera) touch(q);
    return VLRResult_NoError;
}
}

VLRResult vlrQueryableGetEnumValue(VLRQueryableConst queryable, const char* paramName, const char** value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !value) return VLRResult_InvalidArgument;
    auto it = q->enums.find(lower(paramName));
    if (it == q->enums.end()) return VLRResult_InvalidArgument;
    *value = it->second.c_str();
    return VLRResult_NoError;
}
VLRResult vlrQueryableGetPoint3D(VLRQueryableConst queryable, const char* paramName, struct VLRPoint3D* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return getFloats(q, paramName, "Point3D", value ? &value->x : nullptr, 3);
}
VLRResult vlrQueryableGetVector3D(VLRQueryableConst queryable, const char* paramName, struct VLRVector3D* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return getFloats(q, paramName, "Vector3D", value ? &value->x : nullptr, 3);
}
VLRResult vlrQueryableGetNormal3D(VLRQueryableConst queryable, const char* paramName, struct VLRNormal3D* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return getFloats(q, paramName, "Normal3D", value ? &value->x : nullptr, 3);
}
VLRResult vlrQueryableGetQuaternion(VLRQueryableConst queryable, const char* paramName, struct VLRQuaternion* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return getFloats(q, paramName, "Quaternion", value ? &value->x : nullptr, 4);
}
VLRResult vlrQueryableGetFloat(VLRQueryableConst queryable, const char* paramName, float* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return getFloats(q, paramName, "Float", value, 1);
}
VLRResult vlrQueryableGetFloatTuple(VLRQueryableConst queryable, const char* paramName, float* values, uint32_t length) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return getFloats(q, paramName, "Float", values, length);
}
VLRResult vlrQueryableGetFloatArray(VLRQueryableConst queryable, const char* paramName, const float** values,
                                    uint32_t* length) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !values || !length) return VLRResult_InvalidArgument;
    auto it = q->floats.find(lower(paramName));
    if (it == q->floats.end()) return VLRResult_InvalidArgument;
    *values = it->second.data();
    *length = static_cast<uint32_t>(it->second.size());
    return VLRResult_NoError;
}
VLRResult vlrQueryableGetImage2D(VLRQueryableConst queryable, const char* paramName, VLRImage2DConst* image) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !image || !paramOf(q, paramName, "Image")) return VLRResult_InvalidArgument;
    auto it = q->objects.find(lower(paramName));
    *image = it == q->objects.end() ? nullptr : reinterpret_cast<VLRImage2DConst>(it->second);
    return VLRResult_NoError;
}
VLRResult vlrQueryableGetImmediateSpectrum(VLRQueryableConst queryable, const char* paramName,
                                           struct VLRImmediateSpectrum* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !value || !paramOf(q, paramName, "Spectrum")) return VLRResult_InvalidArgument;
    auto it = q->spectra.find(lower(paramName));
    if (it == q->spectra.end()) return VLRResult_InvalidArgument;
    value->colorSpace = it->second.colorSpace.c_str();
    value->e0 = it->second.e[0]; value->e1 = it->second.e[1]; value->e2 = it->second.e[2];
    return VLRResult_NoError;
}
VLRResult vlrQueryableGetSurfaceMaterial(VLRQueryableConst queryable, const char* paramName,
                                         VLRSurfaceMaterialConst* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !value || !paramOf(q, paramName, "SurfaceMaterial")) return VLRResult_InvalidArgument;
    auto it = q->objects.find(lower(paramName));
    *value = it == q->objects.end() ? nullptr : reinterpret_cast<VLRSurfaceMaterialConst>(it->second);
    return VLRResult_NoError;
}
VLRResult vlrQueryableGetShaderNodePlug(VLRQueryableConst queryable, const char* paramName,
                                        struct VLRShaderNodePlug* plug) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !plug || !q->find(paramName)) return VLRResult_InvalidArgument;
    auto it = q->plugs.find(lower(paramName));
    *plug = it == q->plugs.end() ? VLRShaderNodePlug{ 0, 0 } : it->second;
    return VLRResult_NoError;
}

VLRResult vlrQueryableSetEnumValue(VLRQueryable queryable, const char* paramName, const char* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !value) return VLRResult_InvalidArgument;
    const ParamInfo* p = q->find(paramName);
    if (!p) return VLRResult_InvalidArgument;
    const auto* members = enumMembers(p->type);
    if (!members) return VLRResult_InvalidArgument;
    for (const char* m : *members)
        if (lower(m) == lower(value)) {
            q->enums[lower(paramName)] = m;
            touch(q);
            return VLRResult_NoError;
        }
    return VLRResult_InvalidArgument;
}
VLRResult vlrQueryableSetPoint3D(VLRQueryable queryable, const char* paramName, const struct VLRPoint3D* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return setFloats(q, paramName, "Point3D", value ? &value->x : nullptr, 3);
}
VLRResult vlrQueryableSetVector3D(VLRQueryable queryable, const char* paramName, const struct VLRVector3D* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return setFloats(q, paramName, "Vector3D", value ? &value->x : nullptr, 3);
}
VLRResult vlrQueryableSetNormal3D(VLRQueryable queryable, const char* paramName, const struct VLRNormal3D* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return setFloats(q, paramName, "Normal3D", value ? &value->x : nullptr, 3);
}
VLRResult vlrQueryableSetQuaternion(VLRQueryable queryable, const char* paramName, const struct VLRQuaternion* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return setFloats(q, paramName, "Quaternion", value ? &value->x : nullptr, 4);
}
VLRResult vlrQueryableSetFloat(VLRQueryable queryable, const char* paramName, float value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    return setFloats(q, paramName, "Float", &value, 1);
}
VLRResult vlrQueryableSetFloatTuple(VLRQueryable queryable, const char* paramName, const float* values, uint32_t length) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName) return VLRResult_InvalidArgument;
    const ParamInfo* p = q->find(paramName);
    if (!p || (p->tupleSize != 0 && length != p->tupleSize)) return VLRResult_InvalidArgument;
    return setFloats(q, paramName, "Float", values, length);
}
VLRResult vlrQueryableSetImage2D(VLRQueryable queryable, const char* paramName, VLRImage2DConst image) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !paramOf(q, paramName, "Image")) return VLRResult_InvalidArgument;
    if (image) {
        VLRResult e2 = VLRResult_NoError;
        if (!checked<const Object>(image, &e2, isImage)) return e2;
    }
    q->objects[lower(paramName)] = reinterpret_cast<const Object*>(image);
    touch(q);
    return VLRResult_NoError;
}
VLRResult vlrQueryableSetImmediateSpectrum(VLRQueryable queryable, const char* paramName,
                                           const struct VLRImmediateSpectrum* value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !value || !paramOf(q, paramName, "Spectrum")) return VLRResult_InvalidArgument;
    ImmSpectrum s;
    s.colorSpace = value->colorSpace ? value->colorSpace : "Rec709(D65)";
    const auto* cs = enumMembers("ColorSpace");
    bool known = false;
    for (const char* m : *cs) if (lower(m) == lower(s.colorSpace)) known = true;
    if (!known) return VLRResult_InvalidArgument;
    s.e[0] = value->e0; s.e[1] = value->e1; s.e[2] = value->e2;
    q->spectra[lower(paramName)] = s;
    touch(q);
    return VLRResult_NoError;
}
VLRResult vlrQueryableSetSurfaceMaterial(VLRQueryable queryable, const char* paramName, VLRSurfaceMaterialConst value) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName || !paramOf(q, paramName, "SurfaceMaterial")) return VLRResult_InvalidArgument;
    if (value) {
        VLRResult e2 = VLRResult_NoError;
        if (!checked<const Object>(value, &e2, kindMaterial)) return e2;
    }
    q->objects[lower(paramName)] = reinterpret_cast<const Object*>(value);
    touch(q);
    return VLRResult_NoError;
}
VLRResult vlrQueryableSetShaderNodePlug(VLRQueryable queryable, const char* paramName, struct VLRShaderNodePlug plug) {
    CHECK_HANDLE(q, Queryable, isQueryable, queryable);
    if (!paramName) return VLRResult_InvalidArgument;
    const ParamInfo* p = q->find(paramName);
    if (!p || !(p->form & kNode)) return VLRResult_InvalidArgument;
    if (plug.nodeRef) {
        VLRResult e2 = VLRResult_NoError;
        if (!checked<const Object>(reinterpret_cast<const void*>(plug.nodeRef), &e2, kindShaderNode)) return e2;
    }
    q->plugs[lower(paramName)] = plug;
    touch(q);
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- images
VLRResult vlrImage2DGetWidth(VLRImage2DConst image, uint32_t* width) {
    CHECK_HANDLE(im, Image2D, isImage, image);
    if (!width) return VLRResult_InvalidArgument;
    *width = im->width;
    return VLRResult_NoError;
}
VLRResult vlrImage2DGetHeight(VLRImage2DConst image, uint32_t* height) {
    CHECK_HANDLE(im, Image2D, isImage, image);
    if (!height) return VLRResult_InvalidArgument;
    *height = im->height;
    return VLRResult_NoError;
}
VLRResult vlrImage2DGetStride(VLRImage2DConst image, uint32_t* stride) {
    CHECK_HANDLE(im, Image2D, isImage, image);
    if (!stride) return VLRResult_InvalidArgument;
    *stride = 16;
    return VLRResult_NoError;
}
VLRResult vlrImage2DGetOriginalDataFormat(VLRImage2DConst image, const char** format) {
    CHECK_HANDLE(im, Image2D, isImage, image);
    if (!format) return VLRResult_InvalidArgument;
    *format = im->format.c_str();
    return VLRResult_NoError;
}
VLRResult vlrImage2DOriginalHasAlpha(VLRImage2DConst image, bool* hasAlpha) {
    CHECK_HANDLE(im, Image2D, isImage, image);
    if (!hasAlpha) return VLRResult_InvalidArgument;
    *hasAlpha = im->format == "RGBA8x4" || im->format == "RGBA16Fx4" || im->format == "RGBA32Fx4";
    return VLRResult_NoError;
}

VLRResult vlrLinearImage2DCreate(VLRContext context, uint8_t* linearData, uint32_t width, uint32_t height,
                                 const char* format, const char* spectrumType, const char* colorSpace,
                                 VLRLinearImage2D* image) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!linearData || !format || !spectrumType || !colorSpace || !image || width == 0 || height == 0)
        return VLRResult_InvalidArgument;
    API_TRY
    const std::string fmt = format;
    const bool srgb = lower(colorSpace) == "rec709(d65) srgb gamma";
    auto* im = c->adopt(new Image2D(Kind::LinearImage2D));
    im->typeName = "LinearImage2D";
    im->width = width; im->height = height;
    im->format = fmt; im->spectrumType = spectrumType; im->colorSpace = colorSpace;
    const size_t n = size_t(width) * height;
    im->rgba.resize(n * 4);
    auto lin = [&](float v) { return srgb ? sRGBDegamma(v) : v; };
    if (fmt == "RGBA32Fx4") {
        const float* src = reinterpret_cast<const float*>(linearData);
        for (size_t i = 0; i < n * 4; ++i) im->rgba[i] = src[i];
    }
    else if (fmt == "RGB8x3" || fmt == "RGBA8x4" || fmt == "RGB_8x4") {
        const size_t stride = fmt == "RGB8x3" ? 3 : 4;
        for (size_t i = 0; i < n; ++i) {
            for (int k = 0; k < 3; ++k) im->rgba[4 * i + k] = lin(linearData[stride * i + k] / 255.0f);
            im->rgba[4 * i + 3] = stride == 4 && fmt == "RGBA8x4" ? linearData[stride * i + 3] / 255.0f : 1.0f;
        }
    }
    else if (fmt == "Gray32F") {
        const float* src = reinterpret_cast<const float*>(linearData);
        for (size_t i = 0; i < n; ++i) { for (int k = 0; k < 3; ++k) im->rgba[4 * i + k] = src[i]; im->rgba[4 * i + 3] = 1.0f; }
    }
    else if (fmt == "Gray8") {
        for (size_t i = 0; i < n; ++i) { for (int k = 0; k < 3; ++k) im->rgba[4 * i + k] = lin(linearData[i] / 255.0f); im->rgba[4 * i + 3] = 1.0f; }
    }
    else {
        c->destroy(im);
        return VLRResult_InvalidArgument;
    }
    *image = reinterpret_cast<VLRLinearImage2D>(static_cast<Object*>(im));
    return VLRResult_NoError;
    API_CATCH("vlrLinearImage2DCreate")
}

VLRResult vlrLinearImage2DDestroy(VLRContext context, VLRLinearImage2D image) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    Image2D* im = checked<Image2D>(image, &e2, [](const Object* o) { return o->kind == Kind::LinearImage2D; });
    if (!im) return e2;
    c->destroy(im);
    return VLRResult_NoError;
}

VLRResult vlrBlockCompressedImage2DCreate(VLRContext context, uint8_t** data, size_t* sizes, uint32_t mipCount,
                                          uint32_t width, uint32_t height, const char* dataFormat,
                                          const char* spectrumType, const char* colorSpace,
                                          VLRBlockCompressedImage2D* image) {
    CHECK_HANDLE(c, Context, kindContext, context);
    (void)c; (void)data; (void)sizes; (void)mipCount; (void)width; (void)height;
    (void)dataFormat; (void)spectrumType; (void)colorSpace; (void)image;
    // Block-compressed textures are not part of the rendered feature set.
    return VLRResult_InvalidArgument;
}

VLRResult vlrBlockCompressedImage2DDestroy(VLRContext context, VLRBlockCompressedImage2D image) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    Object* o = checked<Object>(image, &e2, [](const Object* x) { return x->kind == Kind::BlockCompressedImage2D; });
    if (!o) return e2;
    c->destroy(o);
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- shader nodes
VLRResult vlrShaderNodeCreate(VLRContext context, const char* typeName, VLRShaderNode* node) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!typeName || !node) return VLRResult_InvalidArgument;
    API_TRY
    auto* n = new ShaderNode();
    n->ctx = c;
    if (!initShaderNode(n, typeName)) { delete n; return VLRResult_InvalidArgument; }
    n->typeName = typeName;
    c->adopt(n);
    *node = reinterpret_cast<VLRShaderNode>(static_cast<Object*>(n));
    return VLRResult_NoError;
    API_CATCH("vlrShaderNodeCreate")
}

VLRResult vlrShaderNodeDestroy(VLRContext context, VLRShaderNode node) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    ShaderNode* n = checked<ShaderNode>(node, &e2, kindShaderNode);
    if (!n) return e2;
    c->destroy(n);
    return VLRResult_NoError;
}

VLRResult vlrShaderNodeGetPlug(VLRShaderNodeConst node, enum VLRShaderNodePlugType plugType, uint32_t option,
                               struct VLRShaderNodePlug* plug) {
    CHECK_HANDLE(n, ShaderNode, kindShaderNode, node);
    if (!plug || plugType >= NumVLRShaderNodePlugTypes) return VLRResult_InvalidArgument;
    plug->nodeRef = reinterpret_cast<uintptr_t>(static_cast<const Object*>(n));
    plug->info = (static_cast<uint32_t>(plugType) & 0xFFu) | ((option & 0xFFu) << 8);
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- materials
VLRResult vlrSurfaceMaterialCreate(VLRContext context, const char* typeName, VLRSurfaceMaterial* material) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!typeName || !material) return VLRResult_InvalidArgument;
    API_TRY
    auto* m = new SurfaceMaterial();
    m->ctx = c;
    if (!initMaterial(m, typeName)) { delete m; return VLRResult_InvalidArgument; }
    m->typeName = typeName;
    c->adopt(m);
    *material = reinterpret_cast<VLRSurfaceMaterial>(static_cast<Object*>(m));
    return VLRResult_NoError;
    API_CATCH("vlrSurfaceMaterialCreate")
}

VLRResult vlrSurfaceMaterialDestroy(VLRContext context, VLRSurfaceMaterial material) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    SurfaceMaterial* m = checked<SurfaceMaterial>(material, &e2, kindMaterial);
    if (!m) return e2;
    c->destroy(m);
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- transforms
namespace {
bool invert4(const float m[16], float inv[16]) {
    double a[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    double r[16];
    r[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] + a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    r[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] - a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    r[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] + a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    r[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] - a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    r[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] - a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    r[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] + a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    r[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] - a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    r[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] + a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    r[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] + a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    r[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] - a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    r[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] + a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    r[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] - a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    r[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] - a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    r[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] + a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    r[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] - a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    r[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] + a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    double det = a[0] * r[0] + a[1] * r[4] + a[2] * r[8] + a[3] * r[12];
    if (det == 0.0 || !std::isfinite(det)) return false;
    for (int i = 0; i < 16; ++i) inv[i] = static_cast<float>(r[i] / det);
    return true;
}
}

VLRResult vlrStaticTransformCreate(VLRContext context, const float mat[16], VLRStaticTransform* transform) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!mat || !transform) return VLRResult_InvalidArgument;
    API_TRY
    auto* t = new StaticTransform();
    std::memcpy(t->m, mat, sizeof(t->m));
    if (!invert4(t->m, t->inv)) { delete t; return VLRResult_InvalidArgument; }
    t->typeName = "StaticTransform";
    c->adopt(t);
    *transform = reinterpret_cast<VLRStaticTransform>(static_cast<Object*>(t));
    return VLRResult_NoError;
    API_CATCH("vlrStaticTransformCreate")
}

VLRResult vlrStaticTransformDestroy(VLRContext context, VLRStaticTransform transform) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    StaticTransform* t = checked<StaticTransform>(transform, &e2, kindTransform);
    if (!t) return e2;
    c->destroy(t);
    return VLRResult_NoError;
}

VLRResult vlrStaticTransformGetArrays(VLRStaticTransformConst transform, float mat[16], float invMat[16]) {
    CHECK_HANDLE(t, StaticTransform, kindTransform, transform);
    if (!mat || !invMat) return VLRResult_InvalidArgument;
    std::memcpy(mat, t->m, sizeof(t->m));
    std::memcpy(invMat, t->inv, sizeof(t->inv));
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- nodes
VLRResult vlrNodeSetName(VLRNode node, const char* name) {
    CHECK_HANDLE(n, Node, isNode, node);
    if (!name) return VLRResult_InvalidArgument;
    n->name = name;
    return VLRResult_NoError;
}

VLRResult vlrNodeGetName(VLRNodeConst node, const char** name) {
    CHECK_HANDLE(n, Node, isNode, node);
    if (!name) return VLRResult_InvalidArgument;
    *name = n->name.c_str();
    return VLRResult_NoError;
}

VLRResult vlrTriangleMeshSurfaceNodeCreate(VLRContext context, const char* name, VLRTriangleMeshSurfaceNode* surfaceNode) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!name || !surfaceNode) return VLRResult_InvalidArgument;
    API_TRY
    auto* n = c->adopt(new TriangleMeshNode());
    n->name = name;
    n->typeName = "TriangleMeshSurfaceNode";
    *surfaceNode = reinterpret_cast<VLRTriangleMeshSurfaceNode>(static_cast<Object*>(n));
    return VLRResult_NoError;
    API_CATCH("vlrTriangleMeshSurfaceNodeCreate")
}

VLRResult vlrTriangleMeshSurfaceNodeDestroy(VLRContext context, VLRTriangleMeshSurfaceNode surfaceNode) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    TriangleMeshNode* n = checked<TriangleMeshNode>(surfaceNode, &e2, kindMesh);
    if (!n) return e2;
    for (Object* o : c->objects)
        if (isParentNode(o)) {
            auto &ch = static_cast<ParentNode*>(o)->children;
            ch.erase(std::remove(ch.begin(), ch.end(), n), ch.end());
        }
    c->destroy(n);
    return VLRResult_NoError;
}

VLRResult vlrTriangleMeshSurfaceNodeSetVertices(VLRTriangleMeshSurfaceNode surfaceNode, const struct VLRVertex* vertices,
                                                uint32_t numVertices) {
    CHECK_HANDLE(n, TriangleMeshNode, kindMesh, surfaceNode);
    if (!vertices && numVertices > 0) return VLRResult_InvalidArgument;
    API_TRY
    n->vertices.assign(vertices, vertices + numVertices);
    touch(n);
    return VLRResult_NoError;
    API_CATCH("vlrTriangleMeshSurfaceNodeSetVertices")
}

VLRResult vlrTriangleMeshSurfaceNodeAddMaterialGroup(VLRTriangleMeshSurfaceNode surfaceNode, const uint32_t* indices,
                                                     uint32_t numIndices, VLRSurfaceMaterialConst material,
                                                     struct VLRShaderNodePlug nodeNormal,
                                                     struct VLRShaderNodePlug nodeTangent,
                                                     struct VLRShaderNodePlug nodeAlpha) {
    CHECK_HANDLE(n, TriangleMeshNode, kindMesh, surfaceNode);
    if (!indices || numIndices % 3 != 0) return VLRResult_InvalidArgument;
    VLRResult e2 = VLRResult_NoError;
    const SurfaceMaterial* m = checked<const SurfaceMaterial>(material, &e2, kindMaterial);
    if (!m) return e2;
    for (uint32_t i = 0; i < numIndices; ++i)
        if (indices[i] >= n->vertices.size()) return VLRResult_InvalidArgument;
    API_TRY
    MaterialGroup g;
    g.indices.assign(indices, indices + numIndices);
    g.material = m;
    g.nodeNormal = nodeNormal;
    g.nodeTangent = nodeTangent;
    g.nodeAlpha = nodeAlpha;
    n->groups.push_back(std::move(g));
    touch(n);
    return VLRResult_NoError;
    API_CATCH("vlrTriangleMeshSurfaceNodeAddMaterialGroup")
}

VLRResult vlrPointSurfaceNodeCreate(VLRContext context, const char* name, VLRPointSurfaceNode* surfaceNode) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!name || !surfaceNode) return VLRResult_InvalidArgument;
    API_TRY
    auto* n = c->adopt(new PointNode());
    n->name = name;
    n->typeName = "PointSurfaceNode";
    *surfaceNode = reinterpret_cast<VLRPointSurfaceNode>(static_cast<Object*>(n));
    return VLRResult_NoError;
    API_CATCH("vlrPointSurfaceNodeCreate")
}

VLRResult vlrPointSurfaceNodeDestroy(VLRContext context, VLRPointSurfaceNode surfaceNode) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    PointNode* n = checked<PointNode>(surfaceNode, &e2, kindPoint);
    if (!n) return e2;
    c->destroy(n);
    return VLRResult_NoError;
}

VLRResult vlrPointSurfaceNodeSetVertices(VLRPointSurfaceNode surfaceNode, const struct VLRVertex* vertices,
                                         uint32_t numVertices) {
    CHECK_HANDLE(n, PointNode, kindPoint, surfaceNode);
    if (!vertices && numVertices > 0) return VLRResult_InvalidArgument;
    n->vertices.assign(vertices, vertices + numVertices);
    return VLRResult_NoError;
}

VLRResult vlrPointSurfaceNodeAddMaterialGroup(VLRPointSurfaceNode surfaceNode, const uint32_t* indices,
                                              uint32_t numIndices, VLRSurfaceMaterialConst material) {
    CHECK_HANDLE(n, PointNode, kindPoint, surfaceNode);
    if (!indices && numIndices > 0) return VLRResult_InvalidArgument;
    VLRResult e2 = VLRResult_NoError;
    const SurfaceMaterial* m = checked<const SurfaceMaterial>(material, &e2, kindMaterial);
    if (!m) return e2;
    API_TRY
    MaterialGroup g;
    g.indices.assign(indices, indices + numIndices);
    g.material = m;
    n->groups.push_back(std::move(g));
    touch(n);
    return VLRResult_NoError;
    API_CATCH("vlrPointSurfaceNodeAddMaterialGroup")
}

VLRResult vlrParentNodeSetTransform(VLRParentNode node, VLRTransformConst localToWorld) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    VLRResult e2 = VLRResult_NoError;
    const StaticTransform* t = checked<const StaticTransform>(localToWorld, &e2, kindTransform);
    if (!t) return e2;
    n->transform = t;
    touch(n);
    return VLRResult_NoError;
}

VLRResult vlrParentNodeGetTransform(VLRParentNodeConst node, VLRTransformConst* localToWorld) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    if (!localToWorld) return VLRResult_InvalidArgument;
    *localToWorld = reinterpret_cast<VLRTransformConst>(static_cast<const Object*>(n->transform));
    return VLRResult_NoError;
}

VLRResult vlrParentNodeAddChild(VLRParentNode node, VLRNode child) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    VLRResult e2 = VLRResult_NoError;
    Node* ch = checked<Node>(child, &e2, isNode);
    if (!ch) return e2;
    if (ch->kind == Kind::Scene || ch == n) return VLRResult_InvalidArgument;
    if (std::find(n->children.begin(), n->children.end(), ch) == n->children.end()) n->children.push_back(ch);
    touch(n);
    return VLRResult_NoError;
}

VLRResult vlrParentNodeRemoveChild(VLRParentNode node, VLRNode child) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    VLRResult e2 = VLRResult_NoError;
    Node* ch = checked<Node>(child, &e2, isNode);
    if (!ch) return e2;
    auto it = std::find(n->children.begin(), n->children.end(), ch);
    if (it == n->children.end()) return VLRResult_InvalidArgument;
    n->children.erase(it);
    touch(n);
    return VLRResult_NoError;
}

VLRResult vlrParentNodeGetNumChildren(VLRParentNodeConst node, uint32_t* numChildren) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    if (!numChildren) return VLRResult_InvalidArgument;
    *numChildren = static_cast<uint32_t>(n->children.size());
    return VLRResult_NoError;
}

VLRResult vlrParentNodeGetChildren(VLRParentNodeConst node, VLRNode* children) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    if (!children) return VLRResult_InvalidArgument;
    for (size_t i = 0; i < n->children.size(); ++i)
        children[i] = reinterpret_cast<VLRNode>(static_cast<Object*>(n->children[i]));
    return VLRResult_NoError;
}

VLRResult vlrParentNodeGetChildAt(VLRParentNodeConst node, uint32_t index, VLRNode* child) {
    CHECK_HANDLE(n, ParentNode, isParentNode, node);
    if (!child || index >= n->children.size()) return VLRResult_InvalidArgument;
    *child = reinterpret_cast<VLRNode>(static_cast<Object*>(n->children[index]));
    return VLRResult_NoError;
}

VLRResult vlrInternalNodeCreate(VLRContext context, const char* name, VLRTransformConst transform, VLRInternalNode* node) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!name || !node) return VLRResult_InvalidArgument;
    VLRResult e2 = VLRResult_NoError;
    const StaticTransform* t = checked<const StaticTransform>(transform, &e2, kindTransform);
    if (!t) return e2;
    API_TRY
    auto* n = c->adopt(new ParentNode(Kind::InternalNode));
    n->name = name;
    n->typeName = "InternalNode";
    n->transform = t;
    *node = reinterpret_cast<VLRInternalNode>(static_cast<Object*>(n));
    return VLRResult_NoError;
    API_CATCH("vlrInternalNodeCreate")
}

VLRResult vlrInternalNodeDestroy(VLRContext context, VLRInternalNode node) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    ParentNode* n = checked<ParentNode>(node, &e2, kindInternal);
    if (!n) return e2;
    for (Object* o : c->objects)
        if (isParentNode(o) && o != n) {
            auto &ch = static_cast<ParentNode*>(o)->children;
            ch.erase(std::remove(ch.begin(), ch.end(), n), ch.end());
        }
    c->destroy(n);
    return VLRResult_NoError;
}

VLRResult vlrSceneCreate(VLRContext context, VLRTransformConst transform, VLRScene* scene) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!scene) return VLRResult_InvalidArgument;
    VLRResult e2 = VLRResult_NoError;
    const StaticTransform* t = checked<const StaticTransform>(transform, &e2, kindTransform);
    if (!t) return e2;
    API_TRY
    auto* s = c->adopt(new Scene());
    s->typeName = "Scene";
    s->name = "Scene";
    s->transform = t;
    *scene = reinterpret_cast<VLRScene>(static_cast<Object*>(s));
    return VLRResult_NoError;
    API_CATCH("vlrSceneCreate")
}

VLRResult vlrSceneDestroy(VLRContext context, VLRScene scene) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    Scene* s = checked<Scene>(scene, &e2, kindScene);
    if (!s) return e2;
    c->destroy(s);
    return VLRResult_NoError;
}

VLRResult vlrSceneSetEnvironment(VLRScene scene, VLRSurfaceMaterial material) {
    CHECK_HANDLE(s, Scene, kindScene, scene);
    VLRResult e2 = VLRResult_NoError;
    SurfaceMaterial* m = checked<SurfaceMaterial>(material, &e2, kindMaterial);
    if (!m) return e2;
    if (lower(m->typeName) != "environmentemitter") return VLRResult_InvalidArgument;
    s->envMaterial = m;
    touch(s);
    return VLRResult_NoError;
}

VLRResult vlrSceneSetEnvironmentRotation(VLRScene scene, float rotationPhi) {
    CHECK_HANDLE(s, Scene, kindScene, scene);
    if (!std::isfinite(rotationPhi)) return VLRResult_InvalidArgument;
    s->envRotation = rotationPhi;
    touch(s);
    return VLRResult_NoError;
}

VLRResult vlrCameraCreate(VLRContext context, const char* typeName, VLRCamera* camera) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!typeName || !camera) return VLRResult_InvalidArgument;
    API_TRY
    auto* cam = new api::Camera();
    cam->ctx = c;
    if (!initCamera(cam, typeName)) { delete cam; return VLRResult_InvalidArgument; }
    cam->typeName = typeName;
    c->adopt(cam);
    *camera = reinterpret_cast<VLRCamera>(static_cast<Object*>(cam));
    return VLRResult_NoError;
    API_CATCH("vlrCameraCreate")
}

VLRResult vlrCameraDestroy(VLRContext context, VLRCamera camera) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    api::Camera* cam = checked<api::Camera>(camera, &e2, kindCamera);
    if (!cam) return e2;
    c->destroy(cam);
    return VLRResult_NoError;
}

// ---------------------------------------------------------------- extensions (include/vlrb.h)
VLRResult vlrbContextRenderSamples(VLRContext context, CUstream stream, VLRCameraConst camera, bool firstFrame,
                                   uint32_t samples, uint32_t limitNumAccumFrames, uint32_t* numAccumFrames) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    const api::Camera* cam = checked<const api::Camera>(camera, &e2, kindCamera);
    if (!cam || !numAccumFrames) return VLRResult_InvalidArgument;
    API_TRY
    c->render(reinterpret_cast<cudaStream_t>(stream), cam, firstFrame, limitNumAccumFrames, samples, numAccumFrames);
    return VLRResult_NoError;
    API_CATCH("vlrbContextRenderSamples")
}

VLRResult vlrbContextSetRenderOptions(VLRContext context, const VLRBRenderOptions* options) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!options || options->maxPathLength == 0 || options->maxPathLength > kMaxBounces ||
        options->maxPathsInFlight == 0 || options->blocksPerSM > 64 || options->bvhTreeletRounds > 8)
        return VLRResult_InvalidArgument;
    c->options.blocksPerSM = options->blocksPerSM ? options->blocksPerSM : 8;
    c->options.auxBuffers = options->auxBuffers != 0;
    c->options.maxPathLength = options->maxPathLength;
    c->options.maxPathsInFlight = options->maxPathsInFlight;
    c->options.lightPathsPerFrame = options->lightPathsPerFrame;
    c->options.rngSeed = options->rngSeed;
    if (c->options.consistentDielectricPdf != (options->consistentDielectricPdf != 0)) {
        c->options.consistentDielectricPdf = options->consistentDielectricPdf != 0;
        c->markDirty();
    }
    if (c->options.bvhTreeletRounds != options->bvhTreeletRounds) {
        c->options.bvhTreeletRounds = options->bvhTreeletRounds;
        c->markDirty();
    }
    return VLRResult_NoError;
}

VLRResult vlrbContextGetRenderOptions(VLRContext context, VLRBRenderOptions* options) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!options) return VLRResult_InvalidArgument;
    options->maxPathLength = c->options.maxPathLength;
    options->maxPathsInFlight = c->options.maxPathsInFlight;
    options->lightPathsPerFrame = c->options.lightPathsPerFrame;
    options->rngSeed = c->options.rngSeed;
    options->consistentDielectricPdf = c->options.consistentDielectricPdf ? 1u : 0u;
    options->blocksPerSM = c->options.blocksPerSM;
    options->bvhTreeletRounds = c->options.bvhTreeletRounds;
    options->auxBuffers = c->options.auxBuffers ? 1u : 0u;
    return VLRResult_NoError;
}

VLRResult vlrbContextAutotune(VLRContext context, CUstream stream, VLRCameraConst camera, uint32_t samplesPerTrial,
                              VLRBAutotuneTrial* trials, uint32_t maxTrials, uint32_t* numTrials) {
    CHECK_HANDLE(c, Context, kindContext, context);
    VLRResult e2 = VLRResult_NoError;
    const api::Camera* cam = checked<const api::Camera>(camera, &e2, kindCamera);
    if (!cam || samplesPerTrial == 0 || (maxTrials > 0 && !trials)) return VLRResult_InvalidArgument;
    API_TRY
    std::vector<AutotuneTrial> t = c->autotune(reinterpret_cast<cudaStream_t>(stream), cam, samplesPerTrial);
    for (uint32_t i = 0; i < maxTrials && i < t.size(); ++i)
        trials[i] = VLRBAutotuneTrial{ t[i].maxPathsInFlight, t[i].blocksPerSM, t[i].segmentsPerSecond };
    if (numTrials) *numTrials = static_cast<uint32_t>(t.size());
    return VLRResult_NoError;
    API_CATCH("vlrbContextAutotune")
}

struct VLRBRenderBatch_API {
    std::unique_ptr<api::RenderBatch> impl;
};

VLRResult vlrbRenderBatchCreate(const VLRBBatchItem* items, uint32_t numItems, CUstream stream,
                                VLRBRenderBatch* batch) {
    return vlrbRenderBatchCreateEx(items, numItems, stream, 0u, batch);
}

VLRResult vlrbRenderBatchCreateEx(const VLRBBatchItem* items, uint32_t numItems, CUstream stream, uint32_t flags,
                                  VLRBRenderBatch* batch) {
    if (!items || numItems == 0 || !batch || (flags & ~VLRB_BATCH_PERSISTENT)) return VLRResult_InvalidArgument;
    std::vector<api::BatchItem> its;
    for (uint32_t i = 0; i < numItems; ++i) {
        CHECK_HANDLE(c, Context, kindContext, items[i].context);
        VLRResult e2 = VLRResult_NoError;
        const api::Camera* cam = checked<const api::Camera>(items[i].camera, &e2, kindCamera);
        if (!cam || items[i].samples == 0) return VLRResult_InvalidArgument;
        if (c->renderer != VLRRenderer_PathTracing) return VLRResult_InvalidArgument;
        its.push_back(api::BatchItem{ c, cam, items[i].samples, items[i].firstFrame });
    }
    API_TRY
    auto* b = new VLRBRenderBatch_API;
    b->impl.reset(new api::RenderBatch(std::move(its), reinterpret_cast<cudaStream_t>(stream),
                                       (flags & VLRB_BATCH_PERSISTENT) != 0));
    *batch = b;
    return VLRResult_NoError;
    API_CATCH("vlrbRenderBatchCreateEx")
}

VLRResult vlrbRenderBatchLaunch(VLRBRenderBatch batch, CUstream stream) {
    if (!batch) return VLRResult_InvalidInstance;
    API_TRY
    batch->impl->launch(reinterpret_cast<cudaStream_t>(stream));
    return VLRResult_NoError;
    API_CATCH("vlrbRenderBatchLaunch")
}

VLRResult vlrbRenderBatchItemTimes(VLRBRenderBatch batch, float* itemMs) {
    if (!batch) return VLRResult_InvalidInstance;
    if (!itemMs) return VLRResult_InvalidArgument;
    API_TRY
    std::vector<float> ms;
    batch->impl->itemTimes(&ms);
    for (size_t i = 0; i < ms.size(); ++i) itemMs[i] = ms[i];
    return VLRResult_NoError;
    API_CATCH("vlrbRenderBatchItemTimes")
}

VLRResult vlrbRenderBatchDestroy(VLRBRenderBatch batch) {
    if (!batch) return VLRResult_InvalidInstance;
    delete batch;
    return VLRResult_NoError;
}

VLRResult vlrbContextSetGuiding(VLRContext context, const VLRBGuidingOptions* o) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!o || o->log2TableSize < 8 || o->log2TableSize > 24 || !(o->learningRate > 0.0f) ||
        o->samplesPerStep == 0 || o->samplesPerStep > (1u << 24) || o->recordBounces == 0 ||
        o->recordBounces > kMaxRecBounces)
        return VLRResult_InvalidArgument;
    GuidingOptions &g = c->guiding;
    g.enabled = o->enabled;
    g.train = o->train;
    g.log2TableSize = o->log2TableSize;
    g.learningRate = o->learningRate;
    g.samplesPerStep = o->samplesPerStep;
    g.stepsPerLaunch = o->stepsPerLaunch;
    g.recordBounces = o->recordBounces;
    g.warmupLaunches = o->warmupLaunches;
    g.weightClamp = o->weightClamp;
    g.trainInterval = o->trainInterval;
    return VLRResult_NoError;
}

VLRResult vlrbContextGetGuiding(VLRContext context, VLRBGuidingOptions* o) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!o) return VLRResult_InvalidArgument;
    const GuidingOptions &g = c->guiding;
    *o = VLRBGuidingOptions{ g.enabled, g.train, g.log2TableSize, g.learningRate, g.samplesPerStep,
                             g.stepsPerLaunch, g.recordBounces, g.warmupLaunches, g.weightClamp,
                             g.trainInterval };
    return VLRResult_NoError;
}

VLRResult vlrbContextGetGuideNet(VLRContext context, VLRBGuideNet* net) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!net || !c->guideNet) return VLRResult_InvalidArgument;
    *net = new VLRBGuideNet_API{ c->guideNet.get(), false };
    return VLRResult_NoError;
}

VLRResult vlrbContextGetGuidingStats(VLRContext context, VLRBGuidingStats* st) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!st) return VLRResult_InvalidArgument;
    API_TRY
    st->lastLoss = c->guideNet ? c->guideNet->lastLoss() : 0.0f;
    st->trainingSteps = c->guidingStats.trainingSteps;
    st->guidedLaunches = c->guidingStats.guidedLaunches;
    st->lastSamples = c->guideSamplesRecorded();
    if (c->guideNet && c->guideNet->errorBits())
        throw std::runtime_error("guiding network: tensor-core wait timed out");
    return VLRResult_NoError;
    API_CATCH("vlrbContextGetGuidingStats")
}

VLRResult vlrbContextGetStats(VLRContext context, VLRBRenderStats* stats) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!stats) return VLRResult_InvalidArgument;
    API_TRY
    RenderStats s;
    c->readStats(&s);
    stats->pathSegments = s.segments;
    stats->shadowRays = s.shadowRays;
    stats->frames = s.frames;
    stats->lightVertexOverflow = s.lightVertexOverflow;
    stats->numTriangles = c->numTriangles();
    stats->bvhMaxDepth = c->bvhDepth();
    return VLRResult_NoError;
    API_CATCH("vlrbContextGetStats")
}

VLRResult vlrbContextReadPixelRngStates(VLRContext context, uint64_t* states, uint32_t count) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!states && count > 0) return VLRResult_InvalidArgument;
    API_TRY
    return c->readPixelRngStates(states, count) ? VLRResult_NoError : VLRResult_InvalidArgument;
    API_CATCH("vlrbContextReadPixelRngStates")
}

VLRResult vlrbContextReadBounceCounters(VLRContext context, uint32_t* counters, uint32_t bounces) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!counters || bounces == 0) return VLRResult_InvalidArgument;
    API_TRY
    return c->readBounceCounters(counters, bounces) ? VLRResult_NoError : VLRResult_InvalidArgument;
    API_CATCH("vlrbContextReadBounceCounters")
}

VLRResult vlrbContextSaveOutputImages(VLRContext context, const char* pathWithoutExtension, float brightnessCoeff) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!pathWithoutExtension || c->width == 0 || c->height == 0) return VLRResult_InvalidArgument;
    API_TRY
    std::vector<float> rgba(size_t(c->width) * c->height * 4);
    c->readOutput(rgba.data());
    return vlrbWriteOutputImages(rgba.data(), c->width, c->height, pathWithoutExtension, brightnessCoeff);
    API_CATCH("vlrbContextSaveOutputImages")
}

VLRResult vlrbContextReadAuxBuffers(VLRContext context, float* albedo, float* normal) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!albedo && !normal) return VLRResult_InvalidArgument;
    API_TRY
    return c->readAux(albedo, normal) ? VLRResult_NoError : VLRResult_InvalidArgument;
    API_CATCH("vlrbContextReadAuxBuffers")
}

VLRResult vlrbContextReadFilm(VLRContext context, double* strata) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!strata || c->width == 0) return VLRResult_InvalidArgument;
    API_TRY
    c->readFilm(strata);
    return VLRResult_NoError;
    API_CATCH("vlrbContextReadFilm")
}

VLRResult vlrbContextGetOutputDevicePointer(VLRContext context, void** devicePtr) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!devicePtr || c->width == 0) return VLRResult_InvalidArgument;
    *devicePtr = c->outputDevicePtr();
    return VLRResult_NoError;
}

VLRResult vlrbContextSetProfiling(VLRContext context, bool enabled) {
    CHECK_HANDLE(c, Context, kindContext, context);
    c->timer.enabled = enabled;
    return VLRResult_NoError;
}

VLRResult vlrbContextGetKernelTimes(VLRContext context, double stageMs[6], uint64_t stageLaunches[6],
                                    uint64_t* launchCount) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!stageMs || !stageLaunches || !launchCount) return VLRResult_InvalidArgument;
    for (int i = 0; i < 6; ++i) { stageMs[i] = c->timer.ms[i]; stageLaunches[i] = c->timer.launches[i]; }
    *launchCount = c->timer.totalLaunches;
    return VLRResult_NoError;
}

VLRResult vlrbContextResetKernelTimes(VLRContext context) {
    CHECK_HANDLE(c, Context, kindContext, context);
    for (int i = 0; i < 5; ++i) { c->timer.ms[i] = 0; c->timer.launches[i] = 0; }
    c->timer.totalLaunches = 0;
    c->timer.paramBytes = 0;
    return VLRResult_NoError;
}

VLRResult vlrbContextGetLaunchParamBytes(VLRContext context, uint64_t* bytes) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!bytes) return VLRResult_InvalidArgument;
    *bytes = c->timer.paramBytes;
    return VLRResult_NoError;
}

VLRResult vlrbContextGetFilmDevicePointer(VLRContext context, void** devicePtr) {
    CHECK_HANDLE(c, Context, kindContext, context);
    if (!devicePtr || c->width == 0) return VLRResult_InvalidArgument;
    *devicePtr = c->filmDevicePtr();
    return VLRResult_NoError;
}

} // extern "C"
