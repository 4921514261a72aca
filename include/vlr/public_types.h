/* Plain-old-data types of the VLR C API, as libvlr_b200 exports it.
 *
 * Layouts and enumerator values are identical to the reference's
 * libVLR/include/vlr/public_types.h so that existing callers (and the
 * vlrcpp C++ wrapper) compile and run unchanged against this library:
 *   VLRParameterFormFlag      public_types.h:10-14
 *   VLRShaderNodePlugType     public_types.h:16-28
 *   VLRShaderNodePlug         public_types.h:30-33
 *   VLRRenderer               public_types.h:37-42
 *   VLRDebugRenderingMode     public_types.h:44-57
 *   VLRImmediateSpectrum      public_types.h:69-74
 *   VLRPoint3D ... Quaternion public_types.h:76-94
 *   VLRVertex (44 bytes)      public_types.h:107-112
 *   VLR_PROCESS_CLASS_LIST    public_types.h:120-146 (the API's classes, in the
 *                             order vlr.h and vlrcpp.h expand them)
 */
#ifndef VLRB_PUBLIC_TYPES_H
#define VLRB_PUBLIC_TYPES_H

#if defined(__cplusplus)
#include <cstdint>
#else
#include <stdbool.h>
#include <stdint.h>
#endif

enum VLRParameterFormFlag {
    VLRParameterFormFlag_ImmediateValue = 1 << 0,
    VLRParameterFormFlag_Node = 1 << 1,
    VLRParameterFormFlag_Both = (1 << 0) | (1 << 1)
};

enum VLRShaderNodePlugType {
    VLRShaderNodePlugType_float1 = 0,
    VLRShaderNodePlugType_float2,
    VLRShaderNodePlugType_float3,
    VLRShaderNodePlugType_float4,
    VLRShaderNodePlugType_Point3D,
    VLRShaderNodePlugType_Vector3D,
    VLRShaderNodePlugType_Normal3D,
    VLRShaderNodePlugType_Spectrum,
    VLRShaderNodePlugType_Alpha,
    VLRShaderNodePlugType_TextureCoordinates,
    NumVLRShaderNodePlugTypes
};

/* nodeRef == 0 means "no node": the immediate value is used. */
struct VLRShaderNodePlug {
    uintptr_t nodeRef;
    uint32_t info;
};

enum VLRRenderer {
    VLRRenderer_PathTracing = 0,
    VLRRenderer_LightTracing,
    VLRRenderer_BPT,
    VLRRenderer_DebugRendering
};

enum VLRDebugRenderingMode {
    VLRDebugRenderingMode_BaseColor = 0,
    VLRDebugRenderingMode_GeometricNormal,
    VLRDebugRenderingMode_ShadingTangent,
    VLRDebugRenderingMode_ShadingBitangent,
    VLRDebugRenderingMode_ShadingNormal,
    VLRDebugRenderingMode_TextureCoordinates,
    VLRDebugRenderingMode_ShadingNormalViewCos,
    VLRDebugRenderingMode_GeometricVsShadingNormal,
    VLRDebugRenderingMode_ShadingFrameLengths,
    VLRDebugRenderingMode_ShadingFrameOrthogonality,
    VLRDebugRenderingMode_DenoiserAlbedo,
    VLRDebugRenderingMode_DenoiserNormal
};

#if !defined(__cplusplus)
typedef enum VLRParameterFormFlag VLRParameterFormFlag;
typedef enum VLRShaderNodePlugType VLRShaderNodePlugType;
typedef struct VLRShaderNodePlug VLRShaderNodePlug;
typedef enum VLRDebugRenderingMode VLRDebugRenderingMode;
typedef enum VLRRenderer VLRRenderer;
#endif

/* colorSpace: "Rec709(D65) sRGB Gamma", "Rec709(D65)", "XYZ" or "xyY". */
struct VLRImmediateSpectrum {
    const char* colorSpace;
    float e0;
    float e1;
    float e2;
};

struct VLRPoint3D { float x, y, z; };
struct VLRNormal3D { float x, y, z; };
struct VLRVector3D { float x, y, z; };
struct VLRTexCoord2D { float u, v; };
struct VLRQuaternion { float x, y, z, w; };

#if !defined(__cplusplus)
typedef struct VLRImmediateSpectrum VLRImmediateSpectrum;
typedef struct VLRPoint3D VLRPoint3D;
typedef struct VLRNormal3D VLRNormal3D;
typedef struct VLRVector3D VLRVector3D;
typedef struct VLRTexCoord2D VLRTexCoord2D;
typedef struct VLRQuaternion VLRQuaternion;
#endif

struct VLRVertex {
    struct VLRPoint3D position;
    struct VLRNormal3D normal;
    struct VLRVector3D tc0Direction;
    struct VLRTexCoord2D texCoord;
};

#if !defined(__cplusplus)
typedef struct VLRVertex VLRVertex;
#endif

/* The classes of the API.  A user defines VLR_PROCESS_CLASS(Name) and expands
 * the list (vlr.h declares a handle type per class, vlrcpp.h a holder). */
#define VLR_PROCESS_CLASS_LIST() \
    VLR_PROCESS_CLASS(Object); \
    VLR_PROCESS_CLASS(ParameterInfo); \
    VLR_PROCESS_CLASS(Queryable); \
    VLR_PROCESS_CLASS(Image2D); \
    VLR_PROCESS_CLASS(LinearImage2D); \
    VLR_PROCESS_CLASS(BlockCompressedImage2D); \
    VLR_PROCESS_CLASS(ShaderNode); \
    VLR_PROCESS_CLASS(SurfaceMaterial); \
    VLR_PROCESS_CLASS(Transform); \
    VLR_PROCESS_CLASS(StaticTransform); \
    VLR_PROCESS_CLASS(Node); \
    VLR_PROCESS_CLASS(SurfaceNode); \
    VLR_PROCESS_CLASS(TriangleMeshSurfaceNode); \
    VLR_PROCESS_CLASS(PointSurfaceNode); \
    VLR_PROCESS_CLASS(ParentNode); \
    VLR_PROCESS_CLASS(InternalNode); \
    VLR_PROCESS_CLASS(Scene); \
    VLR_PROCESS_CLASS(Camera)

#endif /* VLRB_PUBLIC_TYPES_H */
