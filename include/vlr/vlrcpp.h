/* C++ surface of the VLR API over libvlr_b200's C ABI (namespace vlr).
 *
 * The classes and methods a program written against the reference's
 * libVLR/include/vlr/vlrcpp.h calls, with the same names, arguments and
 * ownership: a Context created by Context::create (vlrcpp.h:684-691) makes
 * every other object; objects are shared_ptr-held ("...Ref"), a holder keeps
 * the holders it references (a node its children and transform, a
 * material's parameters their images, materials and shader nodes) alive, and
 * destroys its C object when the last reference goes.  Errors: every C call's
 * VLRResult is checked; the codes the context enables (by default
 * InvalidContext, InvalidInstance and InternalError, vlrcpp.h:697-701) throw
 * std::runtime_error with vlrGetErrorMessage's text, the others are returned
 * (the boolean get/set forms report them as false).  Header only.
 */
#pragma once

#include <algorithm>
#include <cctype>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "vlr.h"
#include "basic_types.h"

namespace vlr {

class Context;
using ContextRef = std::shared_ptr<Context>;
using ContextConstRef = std::shared_ptr<const Context>;

#define VLR_PROCESS_CLASS(Name) \
    class Name##Holder; \
    using Name##Ref = std::shared_ptr<Name##Holder>
VLR_PROCESS_CLASS_LIST();
#undef VLR_PROCESS_CLASS

inline VLRContext getRawContext(const ContextConstRef &context);
inline VLRResult checkResult(const ContextConstRef &context, VLRResult code);

class ObjectHolder : public std::enable_shared_from_this<ObjectHolder> {
protected:
    ContextConstRef m_context;
    VLRObject m_raw = nullptr;

    VLRResult errorCheck(VLRResult code) const { return checkResult(m_context, code); }

public:
    explicit ObjectHolder(const ContextConstRef &context) : m_context(context) {}
    virtual ~ObjectHolder() = default;
    ObjectHolder(const ObjectHolder &) = delete;
    ObjectHolder &operator=(const ObjectHolder &) = delete;

    std::string getType() const {
        const char* name = nullptr;
        errorCheck(vlrObjectGetType(reinterpret_cast<VLRObjectConst>(m_raw), &name));
        return name ? name : "";
    }

    template <typename VLRType>
    VLRType getRaw() const { return reinterpret_cast<VLRType>(m_raw); }
};

// A shader node's output plug, keeping the node alive.
struct ShaderNodePlug {
    ShaderNodeRef node;
    VLRShaderNodePlug plug = { 0, 0 };
    ShaderNodePlug() = default;
    ShaderNodePlug(const ShaderNodeRef &n, const VLRShaderNodePlug &p) : node(n), plug(p) {}
};

class ParameterInfoHolder {
    ContextConstRef m_context;
    VLRParameterInfoConst m_raw;

public:
    ParameterInfoHolder(const ContextConstRef &context, VLRParameterInfoConst raw) : m_context(context), m_raw(raw) {}
    const char* getName() const {
        const char* s = nullptr;
        checkResult(m_context, vlrParameterInfoGetName(m_raw, &s));
        return s;
    }
    VLRParameterFormFlag getSocketForm() const {
        VLRParameterFormFlag f = VLRParameterFormFlag_ImmediateValue;
        checkResult(m_context, vlrParameterInfoGetSocketForm(m_raw, &f));
        return f;
    }
    const char* getType() const {
        const char* s = nullptr;
        checkResult(m_context, vlrParameterInfoGetType(m_raw, &s));
        return s;
    }
    uint32_t getTupleSize(VLRResult* error = nullptr) const {
        uint32_t n = 0;
        const VLRResult e = checkResult(m_context, vlrParameterInfoGetTupleSize(m_raw, &n));
        if (error) *error = e;
        return n;
    }
};

class QueryableHolder : public ObjectHolder {
    // what this object references through set(): kept alive while set
    std::unordered_map<std::string, Image2DRef> m_images;
    std::unordered_map<std::string, SurfaceMaterialRef> m_materials;
    std::unordered_map<std::string, ShaderNodePlug> m_plugs;

    VLRQueryable q() const { return getRaw<VLRQueryable>(); }
    VLRQueryableConst qc() const { return getRaw<VLRQueryableConst>(); }
    bool ok(VLRResult e) const { return errorCheck(e) == VLRResult_NoError; }
    static std::string key(const char* paramName) {
        std::string s(paramName ? paramName : "");
        std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
        return s;
    }

public:
    explicit QueryableHolder(const ContextConstRef &context) : ObjectHolder(context) {}

    bool get(const char* paramName, const char** enumValue) const { return ok(vlrQueryableGetEnumValue(qc(), paramName, enumValue)); }
    bool get(const char* paramName, Point3D* value) const {
        VLRPoint3D v;
        if (!ok(vlrQueryableGetPoint3D(qc(), paramName, &v))) return false;
        *value = Point3D(v.x, v.y, v.z);
        return true;
    }
    bool get(const char* paramName, Vector3D* value) const {
        VLRVector3D v;
        if (!ok(vlrQueryableGetVector3D(qc(), paramName, &v))) return false;
        *value = Vector3D(v.x, v.y, v.z);
        return true;
    }
    bool get(const char* paramName, Normal3D* value) const {
        VLRNormal3D v;
        if (!ok(vlrQueryableGetNormal3D(qc(), paramName, &v))) return false;
        *value = Normal3D(v.x, v.y, v.z);
        return true;
    }
    bool get(const char* paramName, Quaternion* value) const {
        VLRQuaternion v;
        if (!ok(vlrQueryableGetQuaternion(qc(), paramName, &v))) return false;
        *value = Quaternion(v.x, v.y, v.z, v.w);
        return true;
    }
    bool get(const char* paramName, float* value) const { return ok(vlrQueryableGetFloat(qc(), paramName, value)); }
    bool get(const char* paramName, float* values, uint32_t length) const {
        return ok(vlrQueryableGetFloatTuple(qc(), paramName, values, length));
    }
    bool get(const char* paramName, const float** values, uint32_t* length) const {
        return ok(vlrQueryableGetFloatArray(qc(), paramName, values, length));
    }
    bool get(const char* paramName, VLRImmediateSpectrum* spectrum) const {
        return ok(vlrQueryableGetImmediateSpectrum(qc(), paramName, spectrum));
    }
    bool get(const char* paramName, Image2DRef* image) const;
    bool get(const char* paramName, SurfaceMaterialRef* material) const;
    bool get(const char* paramName, ShaderNodePlug* plug) const;

    bool set(const char* paramName, const char* enumValue) const {
        return ok(vlrQueryableSetEnumValue(q(), paramName, enumValue));
    }
    bool set(const char* paramName, const Point3D &value) const {
        const VLRPoint3D v = { value.x, value.y, value.z };
        return ok(vlrQueryableSetPoint3D(q(), paramName, &v));
    }
    bool set(const char* paramName, const Vector3D &value) const {
        const VLRVector3D v = { value.x, value.y, value.z };
        return ok(vlrQueryableSetVector3D(q(), paramName, &v));
    }
    bool set(const char* paramName, const Normal3D &value) const {
        const VLRNormal3D v = { value.x, value.y, value.z };
        return ok(vlrQueryableSetNormal3D(q(), paramName, &v));
    }
    bool set(const char* paramName, const Quaternion &value) const {
        const VLRQuaternion v = { value.x, value.y, value.z, value.w };
        return ok(vlrQueryableSetQuaternion(q(), paramName, &v));
    }
    bool set(const char* paramName, float value) const { return ok(vlrQueryableSetFloat(q(), paramName, value)); }
    bool set(const char* paramName, const float* values, uint32_t length) const {
        return ok(vlrQueryableSetFloatTuple(q(), paramName, values, length));
    }
    bool set(const char* paramName, const VLRImmediateSpectrum &spectrum) const {
        return ok(vlrQueryableSetImmediateSpectrum(q(), paramName, &spectrum));
    }
    bool set(const char* paramName, const Image2DRef &image);
    bool set(const char* paramName, const SurfaceMaterialRef &material);
    bool set(const char* paramName, const ShaderNodePlug &plug);

    uint32_t getNumParameters() const {
        uint32_t n = 0;
        errorCheck(vlrQueryableGetNumParameters(qc(), &n));
        return n;
    }
    ParameterInfoHolder getParameterInfo(uint32_t index) const {
        VLRParameterInfoConst info = nullptr;
        errorCheck(vlrQueryableGetParameterInfo(qc(), index, &info));
        return ParameterInfoHolder(m_context, info);
    }
};

class Image2DHolder : public QueryableHolder {
public:
    explicit Image2DHolder(const ContextConstRef &context) : QueryableHolder(context) {}
    uint32_t getWidth() const { uint32_t v = 0; errorCheck(vlrImage2DGetWidth(getRaw<VLRImage2DConst>(), &v)); return v; }
    uint32_t getHeight() const { uint32_t v = 0; errorCheck(vlrImage2DGetHeight(getRaw<VLRImage2DConst>(), &v)); return v; }
    uint32_t getStride() const { uint32_t v = 0; errorCheck(vlrImage2DGetStride(getRaw<VLRImage2DConst>(), &v)); return v; }
    const char* getOriginalDataFormat() const {
        const char* f = nullptr;
        errorCheck(vlrImage2DGetOriginalDataFormat(getRaw<VLRImage2DConst>(), &f));
        return f;
    }
    bool originalHasAlpha() const {
        bool a = false;
        errorCheck(vlrImage2DOriginalHasAlpha(getRaw<VLRImage2DConst>(), &a));
        return a;
    }
};

class LinearImage2DHolder : public Image2DHolder {
public:
    LinearImage2DHolder(const ContextConstRef &context, const uint8_t* linearData, uint32_t width, uint32_t height,
                        const char* format, const char* spectrumType, const char* colorSpace)
        : Image2DHolder(context) {
        errorCheck(vlrLinearImage2DCreate(getRawContext(m_context), const_cast<uint8_t*>(linearData), width, height,
                                          format, spectrumType, colorSpace,
                                          reinterpret_cast<VLRLinearImage2D*>(&m_raw)));
    }
    ~LinearImage2DHolder() override {
        if (m_raw) errorCheck(vlrLinearImage2DDestroy(getRawContext(m_context), getRaw<VLRLinearImage2D>()));
    }
};

class BlockCompressedImage2DHolder : public Image2DHolder {
public:
    BlockCompressedImage2DHolder(const ContextConstRef &context, const uint8_t* const* data, const size_t* sizes,
                                 uint32_t mipCount, uint32_t width, uint32_t height, const char* dataFormat,
                                 const char* spectrumType, const char* colorSpace)
        : Image2DHolder(context) {
        errorCheck(vlrBlockCompressedImage2DCreate(getRawContext(m_context), const_cast<uint8_t**>(data),
                                                   const_cast<size_t*>(sizes), mipCount, width, height, dataFormat,
                                                   spectrumType, colorSpace,
                                                   reinterpret_cast<VLRBlockCompressedImage2D*>(&m_raw)));
    }
    ~BlockCompressedImage2DHolder() override {
        if (m_raw)
            errorCheck(vlrBlockCompressedImage2DDestroy(getRawContext(m_context), getRaw<VLRBlockCompressedImage2D>()));
    }
};

class ShaderNodeHolder : public QueryableHolder {
public:
    ShaderNodeHolder(const ContextConstRef &context, const char* typeName) : QueryableHolder(context) {
        errorCheck(vlrShaderNodeCreate(getRawContext(m_context), typeName, reinterpret_cast<VLRShaderNode*>(&m_raw)));
    }
    ~ShaderNodeHolder() override {
        if (m_raw) errorCheck(vlrShaderNodeDestroy(getRawContext(m_context), getRaw<VLRShaderNode>()));
    }
    ShaderNodePlug getPlug(VLRShaderNodePlugType plugType, uint32_t option) {
        VLRShaderNodePlug p = { 0, 0 };
        errorCheck(vlrShaderNodeGetPlug(getRaw<VLRShaderNodeConst>(), plugType, option, &p));
        return ShaderNodePlug(std::static_pointer_cast<ShaderNodeHolder>(shared_from_this()), p);
    }
};

class SurfaceMaterialHolder : public QueryableHolder {
public:
    SurfaceMaterialHolder(const ContextConstRef &context, const char* typeName) : QueryableHolder(context) {
        errorCheck(vlrSurfaceMaterialCreate(getRawContext(m_context), typeName,
                                            reinterpret_cast<VLRSurfaceMaterial*>(&m_raw)));
    }
    ~SurfaceMaterialHolder() override {
        if (m_raw) errorCheck(vlrSurfaceMaterialDestroy(getRawContext(m_context), getRaw<VLRSurfaceMaterial>()));
    }
};

inline bool QueryableHolder::set(const char* paramName, const Image2DRef &image) {
    if (!ok(vlrQueryableSetImage2D(q(), paramName, image ? image->getRaw<VLRImage2DConst>() : nullptr))) return false;
    if (image) m_images[key(paramName)] = image;
    else m_images.erase(key(paramName));
    return true;
}
inline bool QueryableHolder::set(const char* paramName, const SurfaceMaterialRef &material) {
    if (!ok(vlrQueryableSetSurfaceMaterial(q(), paramName,
                                           material ? material->getRaw<VLRSurfaceMaterialConst>() : nullptr)))
        return false;
    if (material) m_materials[key(paramName)] = material;
    else m_materials.erase(key(paramName));
    return true;
}
inline bool QueryableHolder::set(const char* paramName, const ShaderNodePlug &plug) {
    if (!ok(vlrQueryableSetShaderNodePlug(q(), paramName, plug.plug))) return false;
    if (plug.node) m_plugs[key(paramName)] = plug;
    else m_plugs.erase(key(paramName));
    return true;
}
inline bool QueryableHolder::get(const char* paramName, Image2DRef* image) const {
    VLRImage2DConst raw = nullptr;
    if (!ok(vlrQueryableGetImage2D(qc(), paramName, &raw))) return false;
    auto it = m_images.find(key(paramName));
    *image = (raw && it != m_images.end() && it->second->getRaw<VLRImage2DConst>() == raw) ? it->second : nullptr;
    return true;
}
inline bool QueryableHolder::get(const char* paramName, SurfaceMaterialRef* material) const {
    VLRSurfaceMaterialConst raw = nullptr;
    if (!ok(vlrQueryableGetSurfaceMaterial(qc(), paramName, &raw))) return false;
    auto it = m_materials.find(key(paramName));
    *material = (raw && it != m_materials.end() && it->second->getRaw<VLRSurfaceMaterialConst>() == raw) ? it->second
                                                                                                        : nullptr;
    return true;
}
inline bool QueryableHolder::get(const char* paramName, ShaderNodePlug* plug) const {
    VLRShaderNodePlug raw = { 0, 0 };
    if (!ok(vlrQueryableGetShaderNodePlug(qc(), paramName, &raw))) return false;
    auto it = m_plugs.find(key(paramName));
    ShaderNodeRef node = (raw.nodeRef && it != m_plugs.end()) ? it->second.node : nullptr;
    *plug = ShaderNodePlug(node, raw);
    return true;
}

class TransformHolder : public ObjectHolder {
public:
    explicit TransformHolder(const ContextConstRef &context) : ObjectHolder(context) {}
};

class StaticTransformHolder : public TransformHolder {
public:
    StaticTransformHolder(const ContextConstRef &context, const float mat[16]) : TransformHolder(context) {
        errorCheck(vlrStaticTransformCreate(getRawContext(m_context), mat,
                                            reinterpret_cast<VLRStaticTransform*>(&m_raw)));
    }
    StaticTransformHolder(const ContextConstRef &context, const Matrix4x4 &mat) : TransformHolder(context) {
        float a[16];
        mat.getArray(a);
        errorCheck(vlrStaticTransformCreate(getRawContext(m_context), a, reinterpret_cast<VLRStaticTransform*>(&m_raw)));
    }
    ~StaticTransformHolder() override {
        if (m_raw) errorCheck(vlrStaticTransformDestroy(getRawContext(m_context), getRaw<VLRStaticTransform>()));
    }
    void getArrays(float mat[16], float invMat[16]) const {
        errorCheck(vlrStaticTransformGetArrays(getRaw<VLRStaticTransformConst>(), mat, invMat));
    }
    void getMatrices(Matrix4x4* mat, Matrix4x4* invMat) const {
        float a[16], b[16];
        getArrays(a, b);
        *mat = Matrix4x4(a);
        *invMat = Matrix4x4(b);
    }
};

class NodeHolder : public ObjectHolder {
public:
    explicit NodeHolder(const ContextConstRef &context) : ObjectHolder(context) {}
    void setName(const std::string &name) const { errorCheck(vlrNodeSetName(getRaw<VLRNode>(), name.c_str())); }
    const char* getName() const {
        const char* n = nullptr;
        errorCheck(vlrNodeGetName(getRaw<VLRNodeConst>(), &n));
        return n;
    }
};

class SurfaceNodeHolder : public NodeHolder {
public:
    explicit SurfaceNodeHolder(const ContextConstRef &context) : NodeHolder(context) {}
};

class TriangleMeshSurfaceNodeHolder : public SurfaceNodeHolder {
    std::vector<SurfaceMaterialRef> m_materials;
    std::vector<ShaderNodePlug> m_plugs;

public:
    TriangleMeshSurfaceNodeHolder(const ContextConstRef &context, const char* name) : SurfaceNodeHolder(context) {
        errorCheck(vlrTriangleMeshSurfaceNodeCreate(getRawContext(m_context), name,
                                                    reinterpret_cast<VLRTriangleMeshSurfaceNode*>(&m_raw)));
    }
    ~TriangleMeshSurfaceNodeHolder() override {
        if (m_raw)
            errorCheck(vlrTriangleMeshSurfaceNodeDestroy(getRawContext(m_context), getRaw<VLRTriangleMeshSurfaceNode>()));
    }
    void setVertices(Vertex* vertices, uint32_t numVertices) {
        errorCheck(vlrTriangleMeshSurfaceNodeSetVertices(getRaw<VLRTriangleMeshSurfaceNode>(),
                                                         reinterpret_cast<const VLRVertex*>(vertices), numVertices));
    }
    void addMaterialGroup(uint32_t* indices, uint32_t numIndices, const SurfaceMaterialRef &material,
                          const ShaderNodePlug &nodeNormal, const ShaderNodePlug &nodeTangent,
                          const ShaderNodePlug &nodeAlpha) {
        errorCheck(vlrTriangleMeshSurfaceNodeAddMaterialGroup(
            getRaw<VLRTriangleMeshSurfaceNode>(), indices, numIndices,
            material ? material->getRaw<VLRSurfaceMaterialConst>() : nullptr, nodeNormal.plug, nodeTangent.plug,
            nodeAlpha.plug));
        m_materials.push_back(material);
        m_plugs.push_back(nodeNormal);
        m_plugs.push_back(nodeTangent);
        m_plugs.push_back(nodeAlpha);
    }
};

class PointSurfaceNodeHolder : public SurfaceNodeHolder {
    std::vector<SurfaceMaterialRef> m_materials;

public:
    PointSurfaceNodeHolder(const ContextConstRef &context, const char* name) : SurfaceNodeHolder(context) {
        errorCheck(vlrPointSurfaceNodeCreate(getRawContext(m_context), name,
                                             reinterpret_cast<VLRPointSurfaceNode*>(&m_raw)));
    }
    ~PointSurfaceNodeHolder() override {
        if (m_raw) errorCheck(vlrPointSurfaceNodeDestroy(getRawContext(m_context), getRaw<VLRPointSurfaceNode>()));
    }
    void setVertices(Vertex* vertices, uint32_t numVertices) {
        errorCheck(vlrPointSurfaceNodeSetVertices(getRaw<VLRPointSurfaceNode>(),
                                                  reinterpret_cast<const VLRVertex*>(vertices), numVertices));
    }
    void addMaterialGroup(uint32_t* indices, uint32_t numIndices, const SurfaceMaterialRef &material) {
        errorCheck(vlrPointSurfaceNodeAddMaterialGroup(getRaw<VLRPointSurfaceNode>(), indices, numIndices,
                                                       material ? material->getRaw<VLRSurfaceMaterialConst>()
                                                                : nullptr));
        m_materials.push_back(material);
    }
};

class ParentNodeHolder : public NodeHolder {
    StaticTransformRef m_transform;
    std::unordered_map<VLRNode, NodeRef> m_children;   // raw handle -> holder

    void add(const NodeRef &child) {
        errorCheck(vlrParentNodeAddChild(getRaw<VLRParentNode>(), child->getRaw<VLRNode>()));
        m_children[child->getRaw<VLRNode>()] = child;
    }
    void remove(const NodeRef &child) {
        errorCheck(vlrParentNodeRemoveChild(getRaw<VLRParentNode>(), child->getRaw<VLRNode>()));
        m_children.erase(child->getRaw<VLRNode>());
    }
    NodeRef holderOf(VLRNode raw) const {
        auto it = m_children.find(raw);
        return it != m_children.end() ? it->second : nullptr;
    }

public:
    ParentNodeHolder(const ContextConstRef &context, const StaticTransformRef &transform)
        : NodeHolder(context), m_transform(transform) {}
    void setTransform(const StaticTransformRef &transform) {
        errorCheck(vlrParentNodeSetTransform(getRaw<VLRParentNode>(),
                                             transform ? transform->getRaw<VLRTransformConst>() : nullptr));
        m_transform = transform;
    }
    TransformRef getTransform() const { return m_transform; }
    void addChild(const ParentNodeRef &child) { add(child); }
    void removeChild(const ParentNodeRef &child) { remove(child); }
    void addChild(const SurfaceNodeRef &child) { add(child); }
    void removeChild(const SurfaceNodeRef &child) { remove(child); }
    uint32_t getNumChildren() const {
        uint32_t n = 0;
        errorCheck(vlrParentNodeGetNumChildren(getRaw<VLRParentNodeConst>(), &n));
        return n;
    }
    void getChildren(uint32_t numChildren, NodeRef* children) const {
        std::vector<VLRNode> raw(getNumChildren());
        errorCheck(vlrParentNodeGetChildren(getRaw<VLRParentNodeConst>(), raw.data()));
        for (uint32_t i = 0; i < numChildren && i < raw.size(); ++i) children[i] = holderOf(raw[i]);
    }
    NodeRef getChildAt(uint32_t index) const {
        VLRNode raw = nullptr;
        errorCheck(vlrParentNodeGetChildAt(getRaw<VLRParentNodeConst>(), index, &raw));
        return holderOf(raw);
    }
};

class InternalNodeHolder : public ParentNodeHolder {
public:
    InternalNodeHolder(const ContextConstRef &context, const char* name, const StaticTransformRef &transform)
        : ParentNodeHolder(context, transform) {
        errorCheck(vlrInternalNodeCreate(getRawContext(m_context), name,
                                         transform ? transform->getRaw<VLRTransformConst>() : nullptr,
                                         reinterpret_cast<VLRInternalNode*>(&m_raw)));
    }
    ~InternalNodeHolder() override {
        if (m_raw) errorCheck(vlrInternalNodeDestroy(getRawContext(m_context), getRaw<VLRInternalNode>()));
    }
};

class SceneHolder : public ParentNodeHolder {
    SurfaceMaterialRef m_environment;

public:
    SceneHolder(const ContextConstRef &context, const StaticTransformRef &transform)
        : ParentNodeHolder(context, transform) {
        errorCheck(vlrSceneCreate(getRawContext(m_context),
                                  transform ? transform->getRaw<VLRTransformConst>() : nullptr,
                                  reinterpret_cast<VLRScene*>(&m_raw)));
    }
    ~SceneHolder() override {
        if (m_raw) errorCheck(vlrSceneDestroy(getRawContext(m_context), getRaw<VLRScene>()));
    }
    void setEnvironment(const SurfaceMaterialRef &matEnv, float rotationPhi) {
        errorCheck(vlrSceneSetEnvironment(getRaw<VLRScene>(), matEnv ? matEnv->getRaw<VLRSurfaceMaterial>() : nullptr));
        errorCheck(vlrSceneSetEnvironmentRotation(getRaw<VLRScene>(), rotationPhi));
        m_environment = matEnv;
    }
    void setEnvironmentRotation(float rotationPhi) {
        errorCheck(vlrSceneSetEnvironmentRotation(getRaw<VLRScene>(), rotationPhi));
    }
};

class CameraHolder : public QueryableHolder {
public:
    CameraHolder(const ContextConstRef &context, const char* typeName) : QueryableHolder(context) {
        errorCheck(vlrCameraCreate(getRawContext(m_context), typeName, reinterpret_cast<VLRCamera*>(&m_raw)));
    }
    ~CameraHolder() override {
        if (m_raw) errorCheck(vlrCameraDestroy(getRawContext(m_context), getRaw<VLRCamera>()));
    }
};

class Context : public std::enable_shared_from_this<Context> {
    VLRContext m_raw = nullptr;
    bool m_throw[VLRResult_NumErrors] = {};
    StaticTransformRef m_identityTransform;
    mutable SceneRef m_scene;      // the bound scene, kept alive while bound

    struct Token {};

public:
    explicit Context(Token) {}
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    ~Context() {
        m_scene.reset();
        m_identityTransform.reset();
        if (m_raw) vlrDestroyContext(m_raw);
    }

    // Error codes that throw std::runtime_error from every call of this context.
    void enableException(VLRResult code) { if (code < VLRResult_NumErrors) m_throw[code] = true; }
    void disableException(VLRResult code) { if (code < VLRResult_NumErrors) m_throw[code] = false; }
    void enableAllExceptions() { for (bool &t : m_throw) t = true; m_throw[VLRResult_NoError] = false; }
    void disableAllExceptions() { for (bool &t : m_throw) t = false; }
    bool throws(VLRResult code) const { return code < VLRResult_NumErrors && m_throw[code]; }

    static ContextRef create(CUcontext cuContext, bool logging, uint32_t maxCallableDepth = 8) {
        ContextRef c = std::make_shared<Context>(Token{});
        c->enableException(VLRResult_InvalidContext);
        c->enableException(VLRResult_InvalidInstance);
        c->enableException(VLRResult_InternalError);
        checkResult(c, vlrCreateContext(cuContext, logging, maxCallableDepth, &c->m_raw));
        const float identity[16] = { 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1 };
        c->m_identityTransform = std::make_shared<StaticTransformHolder>(c, identity);
        return c;
    }

    VLRContext get() const { return m_raw; }
    CUcontext getCUcontext() const {
        CUcontext cu = nullptr;
        checkResult(shared_from_this(), vlrContextGetCUcontext(m_raw, &cu));
        return cu;
    }

    void bindOutputBuffer(uint32_t width, uint32_t height, uint32_t glTexID) const {
        checkResult(shared_from_this(), vlrContextBindOutputBuffer(m_raw, width, height, glTexID));
    }
    void getOutputBufferSize(uint32_t* width, uint32_t* height) const {
        checkResult(shared_from_this(), vlrContextGetOutputBufferSize(m_raw, width, height));
    }
    void getOutputBuffer(CUarray* array) const {
        checkResult(shared_from_this(), vlrContextGetOutputBuffer(m_raw, array));
    }
    void readOutputBuffer(float* data) const {
        checkResult(shared_from_this(), vlrContextReadOutputBuffer(m_raw, data));
    }
    void setScene(const SceneRef &scene) const {
        checkResult(shared_from_this(), vlrContextSetScene(m_raw, scene ? scene->getRaw<VLRScene>() : nullptr));
        m_scene = scene;
    }
    void setRenderer(VLRRenderer renderer) const {
        checkResult(shared_from_this(), vlrContextSetRenderer(m_raw, renderer));
    }
    void setDebugRenderingAttribute(VLRDebugRenderingMode attr) const {
        checkResult(shared_from_this(), vlrContextSetDebugRenderingAttribute(m_raw, attr));
    }
    void setProbePixel(int32_t x, int32_t y) const {
        checkResult(shared_from_this(), vlrContextSetProbePixel(m_raw, x, y));
    }
    void render(CUstream stream, const CameraRef &camera, bool denoise, uint32_t shrinkCoeff, bool firstFrame,
                uint32_t limitNumAccumFrames, uint32_t* numAccumFrames) const {
        checkResult(shared_from_this(),
                    vlrContextRender(m_raw, stream, camera ? camera->getRaw<VLRCameraConst>() : nullptr, denoise,
                                     shrinkCoeff, firstFrame, limitNumAccumFrames, numAccumFrames));
    }

    LinearImage2DRef createLinearImage2D(uint8_t* linearData, uint32_t width, uint32_t height, const char* format,
                                         const char* spectrumType, const char* colorSpace) const {
        return std::make_shared<LinearImage2DHolder>(shared_from_this(), linearData, width, height, format,
                                                     spectrumType, colorSpace);
    }
    BlockCompressedImage2DRef createBlockCompressedImage2D(uint8_t** data, size_t* sizes, uint32_t mipCount,
                                                           uint32_t width, uint32_t height, const char* dataFormat,
                                                           const char* spectrumType, const char* colorSpace) const {
        return std::make_shared<BlockCompressedImage2DHolder>(shared_from_this(), data, sizes, mipCount, width,
                                                              height, dataFormat, spectrumType, colorSpace);
    }
    ShaderNodeRef createShaderNode(const char* typeName) const {
        return std::make_shared<ShaderNodeHolder>(shared_from_this(), typeName);
    }
    SurfaceMaterialRef createSurfaceMaterial(const char* typeName) const {
        return std::make_shared<SurfaceMaterialHolder>(shared_from_this(), typeName);
    }
    StaticTransformRef createStaticTransform(const float mat[16]) const {
        return std::make_shared<StaticTransformHolder>(shared_from_this(), mat);
    }
    StaticTransformRef createStaticTransform(const Matrix4x4 &mat) const {
        return std::make_shared<StaticTransformHolder>(shared_from_this(), mat);
    }
    const StaticTransformRef &getIdentityTransform() const { return m_identityTransform; }
    TriangleMeshSurfaceNodeRef createTriangleMeshSurfaceNode(const char* name) const {
        return std::make_shared<TriangleMeshSurfaceNodeHolder>(shared_from_this(), name);
    }
    PointSurfaceNodeRef createPointSurfaceNode(const char* name) const {
        return std::make_shared<PointSurfaceNodeHolder>(shared_from_this(), name);
    }
    InternalNodeRef createInternalNode(const char* name, const StaticTransformRef &transform = nullptr) const {
        return std::make_shared<InternalNodeHolder>(shared_from_this(), name,
                                                    transform ? transform : m_identityTransform);
    }
    SceneRef createScene(const StaticTransformRef &transform = nullptr) const {
        return std::make_shared<SceneHolder>(shared_from_this(), transform ? transform : m_identityTransform);
    }
    CameraRef createCamera(const char* typeName) const {
        return std::make_shared<CameraHolder>(shared_from_this(), typeName);
    }
};

inline VLRContext getRawContext(const ContextConstRef &context) { return context ? context->get() : nullptr; }

inline VLRResult checkResult(const ContextConstRef &context, VLRResult code) {
    if (code != VLRResult_NoError && context && context->throws(code))
        throw std::runtime_error(vlrGetErrorMessage(code));
    return code;
}

} // namespace vlr
