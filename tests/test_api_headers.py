"""The drop-in boundary as callers compile against it: C and C++ programs
built with include/ (vlr/vlr.h, vlr/public_types.h, vlr/basic_types.h,
vlr/vlrcpp.h, vlrb.h) and linked with libvlr_b200.so.

CPU tests compile and link; where the reference tree is present they also
compile the reference's own unmodified vlrcpp.h and compile tests
(HostProgram/c_compile_test.c, cpp_compile_test.cpp) against these headers
(a temporary copy next to our headers, outside the repository).  The GPU
test runs the C++ program and checks its image against the same scene built
through the C API from Python."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

import vlr_b200 as V

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
API = os.path.join(ROOT, "tests", "api")
CUDA_INC = "/usr/local/cuda/include"
CUDA_STUBS = "/usr/local/cuda/lib64/stubs"
REFERENCE = os.environ.get("VLR_REFERENCE", "/root/reference")
LIBDIR = os.path.dirname(V.LIB) if hasattr(V, "LIB") else os.path.join(ROOT, "vlr_b200")


def _link_flags():
    return ["-L", LIBDIR, "-lvlr_b200", "-L", CUDA_STUBS, "-lcuda", "-Wl,-rpath," + LIBDIR]


def _build(tmp_path, src, cxx):
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    cmd = ([cxx, "-std=c++17" if cxx.endswith("++") else "-std=c99", "-O1", "-Wall", "-Werror", "-I", INC,
            "-I", CUDA_INC, src, "-o", exe] + _link_flags())
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    return exe


def test_c_program_compiles_and_links(tmp_path):
    V.lib()
    _build(tmp_path, os.path.join(API, "c_api_smoke.c"), "gcc")


def test_vlrcpp_program_compiles_and_links(tmp_path):
    V.lib()
    _build(tmp_path, os.path.join(API, "vlrcpp_scene.cpp"), "g++")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "libVLR", "include", "vlr")),
                    reason="reference tree not present")
def test_reference_headers_callers_compile_against_include(tmp_path):
    """The reference's own vlrcpp.h, unmodified, beside our vlr.h,
    public_types.h, basic_types.h and common.h; the body of the reference's
    cpp_compile_test.cpp (its MSVC-only token-pasting error macro and the
    host program's lengthof replaced by standard C++) compiled with it; and
    the reference's c_compile_test.c compiled against include/vlr/vlr.h."""
    hdr = tmp_path / "hdr" / "vlr"
    hdr.mkdir(parents=True)
    for h in ("vlr.h", "public_types.h", "basic_types.h", "common.h"):
        shutil.copy(os.path.join(INC, "vlr", h), hdr / h)
    shutil.copy(os.path.join(REFERENCE, "libVLR", "include", "vlr", "vlrcpp.h"), hdr / "vlrcpp.h")
    os.symlink("vlr", tmp_path / "hdr" / "VLR")
    body = open(os.path.join(REFERENCE, "HostProgram", "cpp_compile_test.cpp")).read()
    body = body[body.index("static vlr::Image2DRef loadImage2D"):]
    import re
    body = re.sub(r"lengthof\((\w+)\)", r"(sizeof(\1) / sizeof(\1[0]))", body)
    tu = tmp_path / "cpp_compile_test.cpp"
    tu.write_text("#include <cstdio>\n#include <VLR/vlrcpp.h>\n#define CUDADRV_CHECK(call) (void)(call)\n" + body)
    p = subprocess.run(["g++", "-std=c++17", "-c", "-I", str(tmp_path / "hdr"), "-I", CUDA_INC, str(tu), "-o",
                        str(tmp_path / "cpp.o")], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    p = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-I", INC, "-I", CUDA_INC,
                        os.path.join(REFERENCE, "HostProgram", "c_compile_test.c")], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr


def _python_scene(ctx, W, H):
    """The scene of tests/api/vlrcpp_scene.cpp, built through the C API."""
    from vlr_b200 import vlr as VV
    verts, groups = [], {}

    def quad(name, o, a, b, n):
        base = len(verts)
        o, a, b = np.array(o, np.float32), np.array(a, np.float32), np.array(b, np.float32)
        t = a / np.float32(np.sqrt(np.float32(a @ a)))
        for p, uv in ((o, (0, 0)), (o + a, (1, 0)), (o + a + b, (1, 1)), (o + b, (0, 1))):
            verts.append(np.concatenate([p, n, t, uv]).astype(np.float32))
        groups.setdefault(name, []).extend([base, base + 1, base + 2, base, base + 2, base + 3])

    quad("floor", (-1.5, 0, 1.5), (3, 0, 0), (0, 0, -3), (0, 1, 0))
    quad("walls", (-1.5, 3, -1.5), (3, 0, 0), (0, 0, 3), (0, -1, 0))
    quad("walls", (-1.5, 0, -1.5), (3, 0, 0), (0, 3, 0), (0, 0, 1))
    quad("walls", (1.5, 0, -1.5), (0, 0, 3), (0, 3, 0), (-1, 0, 0))
    quad("left", (-1.5, 0, 1.5), (0, 0, -3), (0, 3, 0), (1, 0, 0))
    quad("lamp", (-0.5, 2.999, -0.5), (1, 0, 0), (0, 0, 1), (0, -1, 0))
    quad("block", (-0.4, 0.8, 0.4), (0.8, 0, 0), (0, 0, -0.8), (0, 1, 0))
    mats = {}
    mats["white"] = ctx.createSurfaceMaterial("Matte")
    mats["white"].set("albedo", VV.Spectrum("Rec709(D65)", 0.75, 0.75, 0.75))
    mats["red"] = ctx.createSurfaceMaterial("Matte")
    mats["red"].set("albedo", VV.Spectrum("Rec709(D65)", 0.75, 0.1, 0.1))
    mats["metal"] = ctx.createSurfaceMaterial("MicrofacetReflection")
    mats["metal"].set("roughness", 0.3)
    mats["light"] = ctx.createSurfaceMaterial("DiffuseEmitter")
    mats["light"].set("emittance", VV.Spectrum("Rec709(D65)", 10.0, 10.0, 10.0))
    scene = ctx.createScene()
    mesh = ctx.createTriangleMeshSurfaceNode("room")
    mesh.set_vertices(np.stack(verts))
    for g, m in (("floor", "white"), ("walls", "white"), ("left", "red"), ("lamp", "light"), ("block", "metal")):
        mesh.add_material_group(np.array(groups[g], np.uint32), mats[m])
    node = ctx.createInternalNode("room xf", ctx.transform([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]))
    node.add_child(mesh)
    scene.add_child(node)
    cam = ctx.createCamera("Perspective")
    cam.set_point("position", (0.0, 1.5, 5.5))
    cam.set_quaternion("orientation", (0.0, 1.0, 0.0, 0.0))
    cam.set("aspect", W / H)
    cam.set("sensitivity", 1.0)
    cam.set("fovy", float(np.float32(0.6981317)))
    cam.set("lens radius", 0.0)
    return scene, cam, (mats, mesh, node)


@pytest.mark.gpu
def test_vlrcpp_program_renders_like_the_c_api(tmp_path):
    """A program built on vlr::Context::create ... Context::render renders
    the image the same scene gives through the C API (16 frames of one
    sample, same seeds): every pixel within 1e-5 relative."""
    from vlr_b200 import vlr as VV
    exe = _build(tmp_path, os.path.join(API, "vlrcpp_scene.cpp"), "g++")
    W = H = 64
    out = tmp_path / "out.bin"
    p = subprocess.run([exe, "16", str(out), str(W), str(H)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, (p.returncode, p.stderr)
    cpp = np.fromfile(out, np.float32).reshape(H, W, 4)
    ctx = VV.Context()
    ctx.bindOutputBuffer(W, H)
    scene, cam, keep = _python_scene(ctx, W, H)
    ctx.setScene(scene)
    for f in range(16):
        ctx.render(cam, f == 0)
    py = ctx.read_output()
    ctx.close()
    assert np.isfinite(cpp).all() and cpp[..., :3].mean() > 0
    rel = np.abs(cpp[..., :3] - py[..., :3]) / np.maximum(np.abs(py[..., :3]), 1e-3 * py[..., :3].mean())
    assert rel.max() <= 1e-5, rel.max()
