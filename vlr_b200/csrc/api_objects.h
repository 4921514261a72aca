// Host object model behind the VLR C API handles: queryable parameter
// stores for materials, shader nodes, images and cameras; the scene graph;
// the rendering context.  Handles are pointers to these objects; every entry
// point checks the object's kind before use, returning VLRResult codes the
// way the reference's C layer does (libVLR/vlr.cpp:13-34).
#pragma once

#include "../../include/vlrb.h"
#include "core.cuh"

#include <cstdint>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

namespace vlrb {
namespace api {

class Context;

enum class Kind : uint32_t {
    Context, ParameterInfo, LinearImage2D, BlockCompressedImage2D, ShaderNode, SurfaceMaterial,
    StaticTransform, TriangleMeshSurfaceNode, PointSurfaceNode, InternalNode, Scene, Camera
};

constexpr uint32_t kMagic = 0x56524C42u;

// Case-insensitive parameter-name comparison (queryable.cpp:4-6).
std::string lower(const std::string &s);

struct ParamInfo {
    std::string name;
    uint32_t form;            // VLRParameterFormFlag
    std::string type;         // "Float", "Spectrum", "Point3D", ..., or an enum type name
    uint32_t tupleSize;
};

struct Object {
    uint32_t magic = kMagic;
    Kind kind;
    Context* ctx = nullptr;
    std::string typeName;
    explicit Object(Kind k) : kind(k) {}
    virtual ~Object() { magic = 0; }
};

struct ParameterInfoObj : Object {
    ParamInfo info;
    ParameterInfoObj() : Object(Kind::ParameterInfo) {}
};

struct ImmSpectrum {
    std::string colorSpace = "Rec709(D65)";
    float e[3] = { 0, 0, 0 };
};

// Generic parameter store used by every queryable object.
struct Queryable : Object {
    std::vector<std::unique_ptr<ParameterInfoObj>> infos;
    std::map<std::string, std::vector<float>> floats;        // Float / FloatTuple / Point / Vector / Normal / Quaternion
    std::map<std::string, ImmSpectrum> spectra;
    std::map<std::string, std::string> enums;
    std::map<std::string, const Object*> objects;            // Image2D, SurfaceMaterial
    std::map<std::string, VLRShaderNodePlug> plugs;
    explicit Queryable(Kind k) : Object(k) {}
    void addParam(const char* name, uint32_t form, const char* type, uint32_t tuple = 1);
    const ParamInfo* find(const std::string &name) const;
    float getFloat(const char* name, float def) const;
};

struct Image2D : Queryable {
    uint32_t width = 0, height = 0;
    std::string format, spectrumType, colorSpace;
    std::vector<float> rgba;   // linear float RGBA, row-major, top row first
    explicit Image2D(Kind k) : Queryable(k) {}
};

struct ShaderNode : Queryable {
    ShaderNode() : Queryable(Kind::ShaderNode) {}
};

struct SurfaceMaterial : Queryable {
    SurfaceMaterial() : Queryable(Kind::SurfaceMaterial) {}
    bool isEmitting() const;
};

struct Camera : Queryable {
    std::string type;    // "perspective" or "equirectangular"
    Camera() : Queryable(Kind::Camera) {}
};

struct StaticTransform : Object {
    float m[16], inv[16];       // column-major
    StaticTransform() : Object(Kind::StaticTransform) {}
};

struct Node : Object {
    std::string name;
    explicit Node(Kind k) : Object(k) {}
};

struct MaterialGroup {
    std::vector<uint32_t> indices;
    const SurfaceMaterial* material = nullptr;
    VLRShaderNodePlug nodeNormal{}, nodeTangent{}, nodeAlpha{};
};

struct TriangleMeshNode : Node {
    std::vector<VLRVertex> vertices;
    std::vector<MaterialGroup> groups;
    TriangleMeshNode() : Node(Kind::TriangleMeshSurfaceNode) {}
};

struct PointNode : Node {
    std::vector<VLRVertex> vertices;
    std::vector<MaterialGroup> groups;   // indices are point (vertex) indices
    PointNode() : Node(Kind::PointSurfaceNode) {}
};

struct ParentNode : Node {
    const StaticTransform* transform = nullptr;
    std::vector<Node*> children;
    explicit ParentNode(Kind k) : Node(k) {}
};

struct Scene : ParentNode {
    const SurfaceMaterial* envMaterial = nullptr;
    float envRotation = 0.0f;
    Scene() : ParentNode(Kind::Scene) {}
};

bool isQueryable(const Object* o);
bool isNode(const Object* o);
bool isParentNode(const Object* o);
bool isImage(const Object* o);

template <typename T>
inline T* as(void* h) { return static_cast<T*>(reinterpret_cast<Object*>(h)); }

} // namespace api
} // namespace vlrb
