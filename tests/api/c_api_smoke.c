/* A C program written against include/vlr/vlr.h (C99, no C++): creates a
 * context, a material, a shader node, an image and a mesh through the C API
 * and checks each VLRResult.  Compiled (and linked) by the CPU tests; it runs
 * only where a GPU is present. */
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>

#include <vlr/vlr.h>

#define CHECK(call) \
    do { \
        VLRResult res_ = (call); \
        if (res_ != VLRResult_NoError) { \
            fprintf(stderr, "%s failed: %s\n", #call, vlrGetErrorMessage(res_)); \
            return 1; \
        } \
    } while (0)

int main(void) {
    CUcontext cu;
    CUdevice dev;
    if (cuInit(0) != CUDA_SUCCESS) return 3;
    cuDeviceGet(&dev, 0);
    cuDevicePrimaryCtxRetain(&cu, dev);
    cuCtxSetCurrent(cu);
    VLRContext ctx;
    CHECK(vlrCreateContext(cu, false, 8, &ctx));
    uint8_t texels[4 * 4 * 4] = { 0 };
    VLRLinearImage2D image;
    CHECK(vlrLinearImage2DCreate(ctx, texels, 4, 4, "RGBA8x4", "Reflectance", "Rec709(D65) sRGB Gamma", &image));
    uint32_t width = 0;
    CHECK(vlrImage2DGetWidth((VLRImage2DConst)image, &width));
    VLRShaderNode node;
    CHECK(vlrShaderNodeCreate(ctx, "Image2DTexture", &node));
    CHECK(vlrQueryableSetImage2D((VLRQueryable)node, "image", (VLRImage2DConst)image));
    VLRSurfaceMaterial mat;
    CHECK(vlrSurfaceMaterialCreate(ctx, "UE4", &mat));
    VLRShaderNodePlug plug;
    CHECK(vlrShaderNodeGetPlug((VLRShaderNodeConst)node, VLRShaderNodePlugType_Spectrum, 0, &plug));
    CHECK(vlrQueryableSetShaderNodePlug((VLRQueryable)mat, "base color", plug));
    VLRTriangleMeshSurfaceNode mesh;
    CHECK(vlrTriangleMeshSurfaceNodeCreate(ctx, "mesh", &mesh));
    VLRVertex v[3] = { { { 0, 0, 0 }, { 0, 1, 0 }, { 1, 0, 0 }, { 0, 0 } },
                       { { 1, 0, 0 }, { 0, 1, 0 }, { 1, 0, 0 }, { 1, 0 } },
                       { { 0, 0, 1 }, { 0, 1, 0 }, { 1, 0, 0 }, { 0, 1 } } };
    CHECK(vlrTriangleMeshSurfaceNodeSetVertices(mesh, v, 3));
    CHECK(vlrTriangleMeshSurfaceNodeDestroy(ctx, mesh));
    CHECK(vlrSurfaceMaterialDestroy(ctx, mat));
    CHECK(vlrShaderNodeDestroy(ctx, node));
    CHECK(vlrLinearImage2DDestroy(ctx, image));
    CHECK(vlrDestroyContext(ctx));
    printf("c api ok (width %u)\n", width);
    cuDevicePrimaryCtxRelease(dev);
    return width == 4 ? 0 : 1;
}
