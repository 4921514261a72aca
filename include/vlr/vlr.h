/* The VLR C API as exported by libvlr_b200.so.
 *
 * Every function here replaces the reference entry point of the same name in
 * libVLR/include/vlr/vlr.h (line numbers given per block) with the same
 * signature, argument meaning and VLRResult error codes, at the same path
 * (include/vlr/vlr.h, beside public_types.h, basic_types.h and vlrcpp.h), so
 * code written against the reference, C or its vlrcpp.h C++ wrapper,
 * compiles and links against this library unchanged.
 * Implementation: vlr_b200/csrc/vlr_api.cu.
 *
 * Supported surface (everything else validates its arguments and returns
 * VLRResult_InvalidArgument for features this library does not render):
 *   context, output buffer (glTexID must be 0: no graphics interop),
 *   scenes, internal nodes, static transforms, triangle meshes, point
 *   nodes, materials Matte, SpecularReflection, SpecularScattering,
 *   MicrofacetReflection, MicrofacetScattering, LambertianScattering, UE4,
 *   Multi, DiffuseEmitter, DirectionalEmitter, PointEmitter,
 *   EnvironmentEmitter; shader nodes Image2DTexture, EnvironmentTexture and
 *   immediate spectra; the Perspective and Equirectangular cameras;
 *   renderers PathTracing, LightTracing and BPT.
 */
#ifndef VLRB_VLR_H
#define VLRB_VLR_H

#include "public_types.h"
#include <cuda.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* vlr.h:32-40 */
enum VLRResult {
    VLRResult_NoError = 0,
    VLRResult_InvalidContext,
    VLRResult_InvalidInstance,
    VLRResult_InvalidArgument,
    VLRResult_IncompatibleNodeType,
    VLRResult_InternalError,
    VLRResult_NumErrors
};
#if !defined(__cplusplus)
typedef enum VLRResult VLRResult;
#endif

/* Opaque handles (vlr.h:46-58): the context and every class of the list in
 * public_types.h (VLR_PROCESS_CLASS_LIST). */
#define VLR_PROCESS_CLASS(name) \
    typedef struct VLR##name##_API* VLR##name; \
    typedef const struct VLR##name##_API* VLR##name##Const
VLR_PROCESS_CLASS(Context);
VLR_PROCESS_CLASS_LIST();
#undef VLR_PROCESS_CLASS
#define VLR_TYPEDEF_DONE

/* vlr.h:64 */
const char* vlrGetErrorMessage(VLRResult code);

/* Context: vlr.h:70-106 */
VLRResult vlrCreateContext(CUcontext cuContext, bool logging, uint32_t maxCallableDepth, VLRContext* context);
VLRResult vlrDestroyContext(VLRContext context);
VLRResult vlrContextGetCUcontext(VLRContext context, CUcontext* cuContext);
VLRResult vlrContextBindOutputBuffer(VLRContext context, uint32_t width, uint32_t height, uint32_t glTexID);
VLRResult vlrContextGetOutputBufferSize(VLRContext context, uint32_t* width, uint32_t* height);
VLRResult vlrContextGetOutputBuffer(VLRContext context, CUarray* array);
VLRResult vlrContextReadOutputBuffer(VLRContext context, float* data);
VLRResult vlrContextSetScene(VLRContext context, VLRScene scene);
VLRResult vlrContextSetRenderer(VLRContext context, enum VLRRenderer renderer);
VLRResult vlrContextSetDebugRenderingAttribute(VLRContext context, enum VLRDebugRenderingMode attr);
VLRResult vlrContextSetProbePixel(VLRContext context, int32_t x, int32_t y);
VLRResult vlrContextRender(VLRContext context, CUstream stream, VLRCameraConst camera, bool denoise,
                           uint32_t shrinkCoeff, bool firstFrame, uint32_t limitNumAccumFrames,
                           uint32_t* numAccumFrames);

/* Object / parameter info / enums: vlr.h:110-136 */
VLRResult vlrObjectGetType(VLRObjectConst object, const char** typeName);
VLRResult vlrParameterInfoGetName(VLRParameterInfoConst paramInfo, const char** name);
VLRResult vlrParameterInfoGetSocketForm(VLRParameterInfoConst paramInfo, enum VLRParameterFormFlag* form);
VLRResult vlrParameterInfoGetType(VLRParameterInfoConst paramInfo, const char** type);
VLRResult vlrParameterInfoGetTupleSize(VLRParameterInfoConst paramInfo, uint32_t* size);
VLRResult vlrGetNumEnumMembers(const char* typeName, uint32_t* numMembers);
VLRResult vlrGetEnumMember(const char* typeName, uint32_t index, const char** value);

/* Queryable getters: vlr.h:143-196 */
VLRResult vlrQueryableGetNumParameters(VLRQueryableConst queryable, uint32_t* numParams);
VLRResult vlrQueryableGetParameterInfo(VLRQueryableConst queryable, uint32_t index, VLRParameterInfoConst* paramInfo);
VLRResult vlrQueryableGetEnumValue(VLRQueryableConst queryable, const char* paramName, const char** value);
VLRResult vlrQueryableGetPoint3D(VLRQueryableConst queryable, const char* paramName, struct VLRPoint3D* value);
VLRResult vlrQueryableGetVector3D(VLRQueryableConst queryable, const char* paramName, struct VLRVector3D* value);
VLRResult vlrQueryableGetNormal3D(VLRQueryableConst queryable, const char* paramName, struct VLRNormal3D* value);
VLRResult vlrQueryableGetQuaternion(VLRQueryableConst queryable, const char* paramName, struct VLRQuaternion* value);
VLRResult vlrQueryableGetFloat(VLRQueryableConst queryable, const char* paramName, float* value);
VLRResult vlrQueryableGetFloatTuple(VLRQueryableConst queryable, const char* paramName, float* values, uint32_t length);
VLRResult vlrQueryableGetFloatArray(VLRQueryableConst queryable, const char* paramName, const float** values, uint32_t* length);
VLRResult vlrQueryableGetImage2D(VLRQueryableConst queryable, const char* paramName, VLRImage2DConst* image);
VLRResult vlrQueryableGetImmediateSpectrum(VLRQueryableConst queryable, const char* paramName, struct VLRImmediateSpectrum* value);
VLRResult vlrQueryableGetSurfaceMaterial(VLRQueryableConst queryable, const char* paramName, VLRSurfaceMaterialConst* value);
VLRResult vlrQueryableGetShaderNodePlug(VLRQueryableConst queryable, const char* paramName, struct VLRShaderNodePlug* plug);

/* Queryable setters: vlr.h:199-231 */
VLRResult vlrQueryableSetEnumValue(VLRQueryable queryable, const char* paramName, const char* value);
VLRResult vlrQueryableSetPoint3D(VLRQueryable queryable, const char* paramName, const struct VLRPoint3D* value);
VLRResult vlrQueryableSetVector3D(VLRQueryable queryable, const char* paramName, const struct VLRVector3D* value);
VLRResult vlrQueryableSetNormal3D(VLRQueryable queryable, const char* paramName, const struct VLRNormal3D* value);
VLRResult vlrQueryableSetQuaternion(VLRQueryable queryable, const char* paramName, const struct VLRQuaternion* value);
VLRResult vlrQueryableSetFloat(VLRQueryable queryable, const char* paramName, float value);
VLRResult vlrQueryableSetFloatTuple(VLRQueryable queryable, const char* paramName, const float* values, uint32_t length);
VLRResult vlrQueryableSetImage2D(VLRQueryable queryable, const char* paramName, VLRImage2DConst image);
VLRResult vlrQueryableSetImmediateSpectrum(VLRQueryable queryable, const char* paramName, const struct VLRImmediateSpectrum* value);
VLRResult vlrQueryableSetSurfaceMaterial(VLRQueryable queryable, const char* paramName, VLRSurfaceMaterialConst value);
VLRResult vlrQueryableSetShaderNodePlug(VLRQueryable queryable, const char* paramName, struct VLRShaderNodePlug plug);

/* Images: vlr.h:238-277 */
VLRResult vlrImage2DGetWidth(VLRImage2DConst image, uint32_t* width);
VLRResult vlrImage2DGetHeight(VLRImage2DConst image, uint32_t* height);
VLRResult vlrImage2DGetStride(VLRImage2DConst image, uint32_t* stride);
VLRResult vlrImage2DGetOriginalDataFormat(VLRImage2DConst image, const char** format);
VLRResult vlrImage2DOriginalHasAlpha(VLRImage2DConst image, bool* hasAlpha);
VLRResult vlrLinearImage2DCreate(VLRContext context, uint8_t* linearData, uint32_t width, uint32_t height,
                                 const char* format, const char* spectrumType, const char* colorSpace,
                                 VLRLinearImage2D* image);
VLRResult vlrLinearImage2DDestroy(VLRContext context, VLRLinearImage2D image);
VLRResult vlrBlockCompressedImage2DCreate(VLRContext context, uint8_t** data, size_t* sizes, uint32_t mipCount,
                                          uint32_t width, uint32_t height, const char* dataFormat,
                                          const char* spectrumType, const char* colorSpace,
                                          VLRBlockCompressedImage2D* image);
VLRResult vlrBlockCompressedImage2DDestroy(VLRContext context, VLRBlockCompressedImage2D image);

/* Shader nodes: vlr.h:284-295 */
VLRResult vlrShaderNodeCreate(VLRContext context, const char* typeName, VLRShaderNode* node);
VLRResult vlrShaderNodeDestroy(VLRContext context, VLRShaderNode node);
VLRResult vlrShaderNodeGetPlug(VLRShaderNodeConst node, enum VLRShaderNodePlugType plugType, uint32_t option,
                               struct VLRShaderNodePlug* plug);

/* Surface materials: vlr.h:301-307 */
VLRResult vlrSurfaceMaterialCreate(VLRContext context, const char* typeName, VLRSurfaceMaterial* material);
VLRResult vlrSurfaceMaterialDestroy(VLRContext context, VLRSurfaceMaterial material);

/* Transforms: vlr.h:313-322 (mat is column-major 4x4) */
VLRResult vlrStaticTransformCreate(VLRContext context, const float mat[16], VLRStaticTransform* transform);
VLRResult vlrStaticTransformDestroy(VLRContext context, VLRStaticTransform transform);
VLRResult vlrStaticTransformGetArrays(VLRStaticTransformConst transform, float mat[16], float invMat[16]);

/* Nodes: vlr.h:330-335 */
VLRResult vlrNodeSetName(VLRNode node, const char* name);
VLRResult vlrNodeGetName(VLRNodeConst node, const char** name);

/* Triangle meshes: vlr.h:341-356 */
VLRResult vlrTriangleMeshSurfaceNodeCreate(VLRContext context, const char* name, VLRTriangleMeshSurfaceNode* surfaceNode);
VLRResult vlrTriangleMeshSurfaceNodeDestroy(VLRContext context, VLRTriangleMeshSurfaceNode surfaceNode);
VLRResult vlrTriangleMeshSurfaceNodeSetVertices(VLRTriangleMeshSurfaceNode surfaceNode, const struct VLRVertex* vertices,
                                                uint32_t numVertices);
VLRResult vlrTriangleMeshSurfaceNodeAddMaterialGroup(VLRTriangleMeshSurfaceNode surfaceNode, const uint32_t* indices,
                                                     uint32_t numIndices, VLRSurfaceMaterialConst material,
                                                     struct VLRShaderNodePlug nodeNormal,
                                                     struct VLRShaderNodePlug nodeTangent,
                                                     struct VLRShaderNodePlug nodeAlpha);

/* Point surfaces: vlr.h:361-374 (not rendered by this library) */
VLRResult vlrPointSurfaceNodeCreate(VLRContext context, const char* name, VLRPointSurfaceNode* surfaceNode);
VLRResult vlrPointSurfaceNodeDestroy(VLRContext context, VLRPointSurfaceNode surfaceNode);
VLRResult vlrPointSurfaceNodeSetVertices(VLRPointSurfaceNode surfaceNode, const struct VLRVertex* vertices,
                                         uint32_t numVertices);
VLRResult vlrPointSurfaceNodeAddMaterialGroup(VLRPointSurfaceNode surfaceNode, const uint32_t* indices,
                                              uint32_t numIndices, VLRSurfaceMaterialConst material);

/* Parent nodes: vlr.h:381-401 */
VLRResult vlrParentNodeSetTransform(VLRParentNode node, VLRTransformConst localToWorld);
VLRResult vlrParentNodeGetTransform(VLRParentNodeConst node, VLRTransformConst* localToWorld);
VLRResult vlrParentNodeAddChild(VLRParentNode node, VLRNode child);
VLRResult vlrParentNodeRemoveChild(VLRParentNode node, VLRNode child);
VLRResult vlrParentNodeGetNumChildren(VLRParentNodeConst node, uint32_t* numChildren);
VLRResult vlrParentNodeGetChildren(VLRParentNodeConst node, VLRNode* children);
VLRResult vlrParentNodeGetChildAt(VLRParentNodeConst node, uint32_t index, VLRNode* child);

/* Internal nodes: vlr.h:408-414 */
VLRResult vlrInternalNodeCreate(VLRContext context, const char* name, VLRTransformConst transform, VLRInternalNode* node);
VLRResult vlrInternalNodeDestroy(VLRContext context, VLRInternalNode node);

/* Scenes: vlr.h:420-432 */
VLRResult vlrSceneCreate(VLRContext context, VLRTransformConst transform, VLRScene* scene);
VLRResult vlrSceneDestroy(VLRContext context, VLRScene scene);
VLRResult vlrSceneSetEnvironment(VLRScene scene, VLRSurfaceMaterial material);
VLRResult vlrSceneSetEnvironmentRotation(VLRScene scene, float rotationPhi);

/* Cameras: vlr.h:438-444 */
VLRResult vlrCameraCreate(VLRContext context, const char* typeName, VLRCamera* camera);
VLRResult vlrCameraDestroy(VLRContext context, VLRCamera camera);

#if defined(__cplusplus)
}
#endif

#endif /* VLRB_VLR_H */
