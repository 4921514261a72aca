// A program written against the VLR C++ surface (include/vlr/vlrcpp.h): it
// creates a context, a small closed room with a ceiling light and a glossy
// block through vlr::Context::create / createScene / createTriangleMeshSurfaceNode
// / createSurfaceMaterial / createCamera, renders `frames` frames with
// Context::render and writes the RGBA32F output buffer to `out`.
//     vlrcpp_scene <frames> <out.bin> [width height]
// Exit code 0 on success; any VLR error throws and exits 1.
#include <vlr/vlrcpp.h>
#include <cuda.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

namespace {

void quad(std::vector<vlr::Vertex> &v, std::vector<uint32_t> &idx, vlr::Point3D o, vlr::Vector3D a, vlr::Vector3D b,
          vlr::Normal3D n) {
    const uint32_t base = static_cast<uint32_t>(v.size());
    const vlr::Vector3D t = a.normalize();
    v.push_back(vlr::Vertex{ o, n, t, vlr::TexCoord2D(0, 0) });
    v.push_back(vlr::Vertex{ o + a, n, t, vlr::TexCoord2D(1, 0) });
    v.push_back(vlr::Vertex{ o + a + b, n, t, vlr::TexCoord2D(1, 1) });
    v.push_back(vlr::Vertex{ o + b, n, t, vlr::TexCoord2D(0, 1) });
    const uint32_t q[6] = { base, base + 1, base + 2, base, base + 2, base + 3 };
    idx.insert(idx.end(), q, q + 6);
}

} // namespace

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const uint32_t frames = static_cast<uint32_t>(std::atoi(argv[1]));
    const uint32_t W = argc > 4 ? static_cast<uint32_t>(std::atoi(argv[3])) : 64;
    const uint32_t H = argc > 4 ? static_cast<uint32_t>(std::atoi(argv[4])) : 64;
    try {
        if (cuInit(0) != CUDA_SUCCESS) return 3;
        CUdevice dev;
        CUcontext cu;
        cuDeviceGet(&dev, 0);
        cuDevicePrimaryCtxRetain(&cu, dev);
        cuCtxSetCurrent(cu);
        using namespace vlr;
        ContextRef context = Context::create(cu, false);
        SceneRef scene = context->createScene();

        SurfaceMaterialRef white = context->createSurfaceMaterial("Matte");
        white->set("albedo", VLRImmediateSpectrum{ "Rec709(D65)", 0.75f, 0.75f, 0.75f });
        SurfaceMaterialRef red = context->createSurfaceMaterial("Matte");
        red->set("albedo", VLRImmediateSpectrum{ "Rec709(D65)", 0.75f, 0.1f, 0.1f });
        SurfaceMaterialRef metal = context->createSurfaceMaterial("MicrofacetReflection");
        metal->set("roughness", 0.3f);
        SurfaceMaterialRef light = context->createSurfaceMaterial("DiffuseEmitter");
        light->set("emittance", VLRImmediateSpectrum{ "Rec709(D65)", 10.0f, 10.0f, 10.0f });

        std::vector<Vertex> v;
        std::vector<uint32_t> floor, walls, left, lamp, block;
        quad(v, floor, Point3D(-1.5f, 0, 1.5f), Vector3D(3, 0, 0), Vector3D(0, 0, -3), Normal3D(0, 1, 0));
        quad(v, walls, Point3D(-1.5f, 3, -1.5f), Vector3D(3, 0, 0), Vector3D(0, 0, 3), Normal3D(0, -1, 0));
        quad(v, walls, Point3D(-1.5f, 0, -1.5f), Vector3D(3, 0, 0), Vector3D(0, 3, 0), Normal3D(0, 0, 1));
        quad(v, walls, Point3D(1.5f, 0, -1.5f), Vector3D(0, 0, 3), Vector3D(0, 3, 0), Normal3D(-1, 0, 0));
        quad(v, left, Point3D(-1.5f, 0, 1.5f), Vector3D(0, 0, -3), Vector3D(0, 3, 0), Normal3D(1, 0, 0));
        quad(v, lamp, Point3D(-0.5f, 2.999f, -0.5f), Vector3D(1, 0, 0), Vector3D(0, 0, 1), Normal3D(0, -1, 0));
        quad(v, block, Point3D(-0.4f, 0.8f, 0.4f), Vector3D(0.8f, 0, 0), Vector3D(0, 0, -0.8f), Normal3D(0, 1, 0));
        TriangleMeshSurfaceNodeRef mesh = context->createTriangleMeshSurfaceNode("room");
        mesh->setVertices(v.data(), static_cast<uint32_t>(v.size()));
        const ShaderNodePlug none;
        mesh->addMaterialGroup(floor.data(), static_cast<uint32_t>(floor.size()), white, none, none, none);
        mesh->addMaterialGroup(walls.data(), static_cast<uint32_t>(walls.size()), white, none, none, none);
        mesh->addMaterialGroup(left.data(), static_cast<uint32_t>(left.size()), red, none, none, none);
        mesh->addMaterialGroup(lamp.data(), static_cast<uint32_t>(lamp.size()), light, none, none, none);
        mesh->addMaterialGroup(block.data(), static_cast<uint32_t>(block.size()), metal, none, none, none);
        InternalNodeRef node = context->createInternalNode("room xf", context->createStaticTransform(scale(1.0f)));
        node->addChild(mesh);
        scene->addChild(node);
        if (scene->getNumChildren() != 1 || scene->getChildAt(0) != node) return 4;

        CameraRef camera = context->createCamera("Perspective");
        camera->set("position", Point3D(0, 1.5f, 5.5f));
        camera->set("orientation", Quaternion(0.0f, 1.0f, 0.0f, 0.0f));   // half a turn about y
        camera->set("aspect", static_cast<float>(W) / H);
        camera->set("sensitivity", 1.0f);
        camera->set("fovy", 0.6981317f);   // 40 degrees
        camera->set("lens radius", 0.0f);

        context->bindOutputBuffer(W, H, 0);
        context->setScene(scene);
        uint32_t accumulated = 0;
        for (uint32_t f = 0; f < frames; ++f)
            context->render(nullptr, camera, false, 1, f == 0, 1u << 30, &accumulated);
        if (accumulated != frames) return 5;
        std::vector<float> rgba(size_t(W) * H * 4);
        context->readOutputBuffer(rgba.data());
        FILE* fp = std::fopen(argv[2], "wb");
        if (!fp) return 6;
        std::fwrite(rgba.data(), sizeof(float), rgba.size(), fp);
        std::fclose(fp);
        cuDevicePrimaryCtxRelease(dev);
    }
    catch (const std::exception &e) {
        std::fprintf(stderr, "vlrcpp_scene: %s\n", e.what());
        return 1;
    }
    return 0;
}
