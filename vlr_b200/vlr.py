"""Python mirror of the reference's vlrcpp.h wrapper over the C API.

Names follow libVLR/include/vlr/vlrcpp.h (Context::create, createScene,
createTriangleMeshSurfaceNode, createSurfaceMaterial, createCamera, render);
errors raise VLRError the way vlrcpp's errorCheck throws
(vlrcpp.h:697-701).  Every call goes through libvlr_b200.so's C ABI.
"""
import ctypes
import math

import numpy as np

from . import lib, check, VLRError

c_void_p = ctypes.c_void_p


class VLRVertex(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("normal", ctypes.c_float * 3),
                ("tc0Direction", ctypes.c_float * 3), ("texCoord", ctypes.c_float * 2)]


class VLRImmediateSpectrum(ctypes.Structure):
    _fields_ = [("colorSpace", ctypes.c_char_p), ("e0", ctypes.c_float), ("e1", ctypes.c_float),
                ("e2", ctypes.c_float)]


class VLRShaderNodePlug(ctypes.Structure):
    _fields_ = [("nodeRef", ctypes.c_size_t), ("info", ctypes.c_uint32)]


class VLRBRenderOptions(ctypes.Structure):
    _fields_ = [("maxPathLength", ctypes.c_uint32), ("maxPathsInFlight", ctypes.c_uint32),
                ("lightPathsPerFrame", ctypes.c_uint32), ("rngSeed", ctypes.c_uint64),
                ("consistentDielectricPdf", ctypes.c_uint32), ("blocksPerSM", ctypes.c_uint32),
                ("bvhTreeletRounds", ctypes.c_uint32),
                ("auxBuffers", ctypes.c_uint32)]


class VLRBAutotuneTrial(ctypes.Structure):
    _fields_ = [("maxPathsInFlight", ctypes.c_uint32), ("blocksPerSM", ctypes.c_uint32),
                ("segmentsPerSecond", ctypes.c_double)]


class VLRBRenderStats(ctypes.Structure):
    _fields_ = [("pathSegments", ctypes.c_uint64), ("shadowRays", ctypes.c_uint64), ("frames", ctypes.c_uint64),
                ("lightVertexOverflow", ctypes.c_uint32), ("numTriangles", ctypes.c_uint32),
                ("bvhMaxDepth", ctypes.c_uint32)]


class VLRBGuidingOptions(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_bool), ("train", ctypes.c_bool), ("log2TableSize", ctypes.c_uint32),
                ("learningRate", ctypes.c_float), ("samplesPerStep", ctypes.c_uint32),
                ("stepsPerLaunch", ctypes.c_uint32), ("recordBounces", ctypes.c_uint32),
                ("warmupLaunches", ctypes.c_uint32), ("weightClamp", ctypes.c_float),
                ("trainInterval", ctypes.c_uint32)]


class VLRBGuidingStats(ctypes.Structure):
    _fields_ = [("lastLoss", ctypes.c_float), ("trainingSteps", ctypes.c_uint64),
                ("guidedLaunches", ctypes.c_uint64), ("lastSamples", ctypes.c_uint32)]


class VLRBBatchItem(ctypes.Structure):
    _fields_ = [("context", ctypes.c_void_p), ("camera", ctypes.c_void_p), ("samples", ctypes.c_uint32),
                ("firstFrame", ctypes.c_bool)]


RENDERER_PATH_TRACING = 0
RENDERER_LIGHT_TRACING = 1
RENDERER_BPT = 2
PLUG_FLOAT1 = 0
PLUG_FLOAT3 = 2
PLUG_NORMAL3D = 6
PLUG_SPECTRUM = 7
PLUG_ALPHA = 8


def _api():
    L = lib()
    if getattr(L, "_vlr_sigs", False):
        return L
    v = c_void_p
    sigs = {
        "vlrCreateContext": [v, ctypes.c_bool, ctypes.c_uint32, ctypes.POINTER(v)],
        "vlrDestroyContext": [v],
        "vlrContextBindOutputBuffer": [v, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32],
        "vlrContextGetOutputBufferSize": [v, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)],
        "vlrContextReadOutputBuffer": [v, v],
        "vlrbContextReadAuxBuffers": [v, v, v],
        "vlrbContextReadPixelRngStates": [v, v, ctypes.c_uint32],
        "vlrbContextReadBounceCounters": [v, v, ctypes.c_uint32],
        "vlrbWriteOutputImages": [v, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_float],
        "vlrbContextSaveOutputImages": [v, ctypes.c_char_p, ctypes.c_float],
        "vlrContextSetScene": [v, v],
        "vlrContextSetRenderer": [v, ctypes.c_int],
        "vlrContextRender": [v, v, v, ctypes.c_bool, ctypes.c_uint32, ctypes.c_bool, ctypes.c_uint32,
                             ctypes.POINTER(ctypes.c_uint32)],
        "vlrSurfaceMaterialCreate": [v, ctypes.c_char_p, ctypes.POINTER(v)],
        "vlrShaderNodeCreate": [v, ctypes.c_char_p, ctypes.POINTER(v)],
        "vlrShaderNodeGetPlug": [v, ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(VLRShaderNodePlug)],
        "vlrQueryableSetImmediateSpectrum": [v, ctypes.c_char_p, ctypes.POINTER(VLRImmediateSpectrum)],
        "vlrQueryableSetFloat": [v, ctypes.c_char_p, ctypes.c_float],
        "vlrQueryableSetEnumValue": [v, ctypes.c_char_p, ctypes.c_char_p],
        "vlrQueryableSetFloatTuple": [v, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float), ctypes.c_uint32],
        "vlrQueryableSetPoint3D": [v, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float * 3)],
        "vlrQueryableSetQuaternion": [v, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float * 4)],
        "vlrQueryableSetImage2D": [v, ctypes.c_char_p, v],
        "vlrQueryableSetSurfaceMaterial": [v, ctypes.c_char_p, v],
        "vlrQueryableSetShaderNodePlug": [v, ctypes.c_char_p, VLRShaderNodePlug],
        "vlrQueryableGetFloat": [v, ctypes.c_char_p, ctypes.POINTER(ctypes.c_float)],
        "vlrQueryableGetNumParameters": [v, ctypes.POINTER(ctypes.c_uint32)],
        "vlrLinearImage2DCreate": [v, v, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p,
                                   ctypes.c_char_p, ctypes.POINTER(v)],
        "vlrStaticTransformCreate": [v, ctypes.POINTER(ctypes.c_float * 16), ctypes.POINTER(v)],
        "vlrTriangleMeshSurfaceNodeCreate": [v, ctypes.c_char_p, ctypes.POINTER(v)],
        "vlrTriangleMeshSurfaceNodeSetVertices": [v, v, ctypes.c_uint32],
        "vlrTriangleMeshSurfaceNodeAddMaterialGroup": [v, v, ctypes.c_uint32, v, VLRShaderNodePlug,
                                                       VLRShaderNodePlug, VLRShaderNodePlug],
        "vlrPointSurfaceNodeCreate": [v, ctypes.c_char_p, ctypes.POINTER(v)],
        "vlrPointSurfaceNodeSetVertices": [v, v, ctypes.c_uint32],
        "vlrPointSurfaceNodeAddMaterialGroup": [v, v, ctypes.c_uint32, v],
        "vlrInternalNodeCreate": [v, ctypes.c_char_p, v, ctypes.POINTER(v)],
        "vlrParentNodeAddChild": [v, v],
        "vlrSceneCreate": [v, v, ctypes.POINTER(v)],
        "vlrSceneSetEnvironment": [v, v],
        "vlrSceneSetEnvironmentRotation": [v, ctypes.c_float],
        "vlrCameraCreate": [v, ctypes.c_char_p, ctypes.POINTER(v)],
        "vlrbContextRenderSamples": [v, v, v, ctypes.c_bool, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.POINTER(ctypes.c_uint32)],
        "vlrbContextSetRenderOptions": [v, ctypes.POINTER(VLRBRenderOptions)],
        "vlrbContextGetRenderOptions": [v, ctypes.POINTER(VLRBRenderOptions)],
        "vlrbContextGetStats": [v, ctypes.POINTER(VLRBRenderStats)],
        "vlrbContextSetGuiding": [v, ctypes.POINTER(VLRBGuidingOptions)],
        "vlrbRenderBatchCreate": [ctypes.POINTER(VLRBBatchItem), ctypes.c_uint32, v, ctypes.POINTER(c_void_p)],
        "vlrbRenderBatchCreateEx": [ctypes.POINTER(VLRBBatchItem), ctypes.c_uint32, v, ctypes.c_uint32,
                                    ctypes.POINTER(c_void_p)],
        "vlrbRenderBatchLaunch": [v, v],
        "vlrbRenderBatchItemTimes": [v, ctypes.POINTER(ctypes.c_float)],
        "vlrbRenderBatchDestroy": [v],
        "vlrbContextAutotune": [v, v, v, ctypes.c_uint32, ctypes.POINTER(VLRBAutotuneTrial), ctypes.c_uint32,
                                ctypes.POINTER(ctypes.c_uint32)],
        "vlrbContextGetGuiding": [v, ctypes.POINTER(VLRBGuidingOptions)],
        "vlrbContextGetGuidingStats": [v, ctypes.POINTER(VLRBGuidingStats)],
        "vlrbContextGetGuideNet": [v, ctypes.POINTER(c_void_p)],
        "vlrbContextReadFilm": [v, v],
        "vlrbContextGetOutputDevicePointer": [v, ctypes.POINTER(v)],
        "vlrbContextSetProfiling": [v, ctypes.c_bool],
        "vlrbContextGetKernelTimes": [v, ctypes.POINTER(ctypes.c_double * 6), ctypes.POINTER(ctypes.c_uint64 * 6),
                                      ctypes.POINTER(ctypes.c_uint64)],
        "vlrbContextResetKernelTimes": [v],
        "vlrbContextGetLaunchParamBytes": [v, ctypes.POINTER(ctypes.c_uint64)],
        "vlrbContextGetFilmDevicePointer": [v, ctypes.POINTER(v)],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    L._vlr_sigs = True
    return L


NULL_PLUG = VLRShaderNodePlug(0, 0)


class Queryable:
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    def set(self, name, value):
        L = _api()
        n = name.encode()
        if isinstance(value, Spectrum):
            check(L.vlrQueryableSetImmediateSpectrum(self.h, n, ctypes.byref(value.c())), f"set {name}")
        elif isinstance(value, Plug):
            check(L.vlrQueryableSetShaderNodePlug(self.h, n, value.plug), f"set {name}")
        elif isinstance(value, Image):
            check(L.vlrQueryableSetImage2D(self.h, n, value.h), f"set {name}")
        elif isinstance(value, SurfaceMaterial):
            check(L.vlrQueryableSetSurfaceMaterial(self.h, n, value.h), f"set {name}")
        elif isinstance(value, (int, float)):
            check(L.vlrQueryableSetFloat(self.h, n, float(value)), f"set {name}")
        else:
            raise TypeError(value)

    def set_point(self, name, p):
        check(_api().vlrQueryableSetPoint3D(self.h, name.encode(), ctypes.byref((ctypes.c_float * 3)(*p))), name)

    def set_quaternion(self, name, q):
        check(_api().vlrQueryableSetQuaternion(self.h, name.encode(), ctypes.byref((ctypes.c_float * 4)(*q))), name)

    def set_enum(self, name, value):
        check(_api().vlrQueryableSetEnumValue(self.h, name.encode(), value.encode()), name)

    def get_float(self, name):
        v = ctypes.c_float()
        check(_api().vlrQueryableGetFloat(self.h, name.encode(), ctypes.byref(v)), name)
        return v.value


class Spectrum:
    def __init__(self, color_space, e0, e1, e2):
        self.cs = color_space.encode()
        self.e = (e0, e1, e2)

    def c(self):
        return VLRImmediateSpectrum(self.cs, *self.e)


def rgb(r, g, b):
    return Spectrum("Rec709(D65)", r, g, b)


class Plug:
    def __init__(self, plug):
        self.plug = plug


class Image:
    def __init__(self, handle, keep):
        self.h = handle
        self._keep = keep


class SurfaceMaterial(Queryable):
    """A surface material; also the value of a Multi material's "0".."3"."""


class ShaderNode(Queryable):
    def plug(self, plug_type=PLUG_SPECTRUM, option=0):
        p = VLRShaderNodePlug()
        check(_api().vlrShaderNodeGetPlug(self.h, plug_type, option, ctypes.byref(p)), "getPlug")
        return Plug(p)


class TriangleMesh:
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    def set_vertices(self, verts):
        """verts: float32 array (n, 11): position, normal, tc0Direction, texCoord."""
        a = np.ascontiguousarray(verts, dtype=np.float32)
        assert a.ndim == 2 and a.shape[1] == 11
        self._verts = a
        check(_api().vlrTriangleMeshSurfaceNodeSetVertices(self.h, a.ctypes.data_as(c_void_p), a.shape[0]),
              "setVertices")

    def add_material_group(self, indices, material, normal=None, tangent=None, alpha=None):
        """normal / tangent / alpha: Plug objects (the group's nodeNormal,
        nodeTangent and nodeAlpha), None for none."""
        idx = np.ascontiguousarray(indices, dtype=np.uint32)
        P = lambda pl: pl.plug if pl is not None else NULL_PLUG
        check(_api().vlrTriangleMeshSurfaceNodeAddMaterialGroup(
            self.h, idx.ctypes.data_as(c_void_p), idx.size, material.h, P(normal), P(tangent), P(alpha)),
            "addMaterialGroup")


class PointSet:
    """A PointSurfaceNode: points that emit with a point-emitter material."""
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    def set_vertices(self, verts):
        """verts: float32 array (n, 11): position, normal, tc0Direction, texCoord."""
        a = np.ascontiguousarray(verts, dtype=np.float32)
        assert a.ndim == 2 and a.shape[1] == 11
        self._verts = a
        check(_api().vlrPointSurfaceNodeSetVertices(self.h, a.ctypes.data_as(c_void_p), a.shape[0]), "setVertices")

    def add_material_group(self, indices, material):
        idx = np.ascontiguousarray(indices, dtype=np.uint32)
        check(_api().vlrPointSurfaceNodeAddMaterialGroup(self.h, idx.ctypes.data_as(c_void_p), idx.size, material.h),
              "addMaterialGroup")


class ParentNode:
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle
        self.children = []

    def add_child(self, node):
        self.children.append(node)
        check(_api().vlrParentNodeAddChild(self.h, node.h), "addChild")


class SceneNode(ParentNode):
    def set_environment(self, material, rotation=0.0):
        self.env = material
        check(_api().vlrSceneSetEnvironment(self.h, material.h), "setEnvironment")
        check(_api().vlrSceneSetEnvironmentRotation(self.h, rotation), "setEnvironmentRotation")


class Context:
    """vlr::Context (vlrcpp.h:652-835)."""

    def __init__(self, logging=False):
        import torch  # initialises the CUDA primary context used by the library
        torch.cuda.init()
        L = _api()
        h = c_void_p()
        check(L.vlrCreateContext(None, logging, 8, ctypes.byref(h)), "vlrCreateContext")
        self.h = h
        self._objects = []
        self.width = self.height = 0

    @classmethod
    def create(cls, logging=False):
        return cls(logging)

    def close(self):
        if self.h:
            _api().vlrDestroyContext(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _new(self, fn, *args):
        h = c_void_p()
        check(getattr(_api(), fn)(self.h, *args, ctypes.byref(h)), fn)
        return h

    def identity(self):
        m = (ctypes.c_float * 16)(*[1.0 if i % 5 == 0 else 0.0 for i in range(16)])
        return self._new("vlrStaticTransformCreate", ctypes.byref(m))

    def transform(self, mat4_colmajor):
        m = (ctypes.c_float * 16)(*[float(x) for x in mat4_colmajor])
        return self._new("vlrStaticTransformCreate", ctypes.byref(m))

    def createScene(self):
        return SceneNode(self, self._new("vlrSceneCreate", self.identity()))

    def createInternalNode(self, name, transform=None):
        t = transform if transform is not None else self.identity()
        return ParentNode(self, self._new("vlrInternalNodeCreate", name.encode(), t))

    def createTriangleMeshSurfaceNode(self, name):
        return TriangleMesh(self, self._new("vlrTriangleMeshSurfaceNodeCreate", name.encode()))

    def createPointSurfaceNode(self, name):
        return PointSet(self, self._new("vlrPointSurfaceNodeCreate", name.encode()))

    def createSurfaceMaterial(self, type_name):
        return SurfaceMaterial(self, self._new("vlrSurfaceMaterialCreate", type_name.encode()))

    def createShaderNode(self, type_name):
        return ShaderNode(self, self._new("vlrShaderNodeCreate", type_name.encode()))

    def createLinearImage2D(self, rgba_f32, spectrum_type="Light Source", color_space="Rec709(D65)"):
        a = np.ascontiguousarray(rgba_f32, dtype=np.float32)
        h, w = a.shape[:2]
        handle = self._new("vlrLinearImage2DCreate", a.ctypes.data_as(c_void_p), w, h, b"RGBA32Fx4",
                           spectrum_type.encode(), color_space.encode())
        return Image(handle, a)

    def createCamera(self, type_name="Perspective"):
        return Queryable(self, self._new("vlrCameraCreate", type_name.encode()))

    def bindOutputBuffer(self, width, height):
        check(_api().vlrContextBindOutputBuffer(self.h, width, height, 0), "bindOutputBuffer")
        self.width, self.height = width, height

    def setScene(self, scene):
        self.scene = scene
        check(_api().vlrContextSetScene(self.h, scene.h), "setScene")

    def setRenderer(self, renderer):
        check(_api().vlrContextSetRenderer(self.h, renderer), "setRenderer")

    def setOptions(self, max_path_length=None, max_paths_in_flight=None, light_paths_per_frame=None, rng_seed=None,
                   consistent_dielectric_pdf=None, blocks_per_sm=None, bvh_treelet_rounds=None, aux_buffers=None):
        o = VLRBRenderOptions()
        check(_api().vlrbContextGetRenderOptions(self.h, ctypes.byref(o)), "getOptions")
        if max_path_length is not None:
            o.maxPathLength = max_path_length
        if max_paths_in_flight is not None:
            o.maxPathsInFlight = max_paths_in_flight
        if light_paths_per_frame is not None:
            o.lightPathsPerFrame = light_paths_per_frame
        if rng_seed is not None:
            o.rngSeed = rng_seed
        if consistent_dielectric_pdf is not None:
            o.consistentDielectricPdf = int(bool(consistent_dielectric_pdf))
        if blocks_per_sm is not None:
            o.blocksPerSM = blocks_per_sm
        if bvh_treelet_rounds is not None:
            o.bvhTreeletRounds = bvh_treelet_rounds
        if aux_buffers is not None:
            o.auxBuffers = int(bool(aux_buffers))
        check(_api().vlrbContextSetRenderOptions(self.h, ctypes.byref(o)), "setOptions")

    def autotune(self, camera, samples_per_trial=4, stream=0):
        """vlrbContextAutotune: returns the trials; the fastest configuration
        is kept in the render options."""
        trials = (VLRBAutotuneTrial * 32)()
        n = ctypes.c_uint32()
        check(_api().vlrbContextAutotune(self.h, c_void_p(stream), camera.h, samples_per_trial, trials, 32,
                                         ctypes.byref(n)), "vlrbContextAutotune")
        return [(t.maxPathsInFlight, t.blocksPerSM, t.segmentsPerSecond) for t in trials[:n.value]]

    def options(self):
        o = VLRBRenderOptions()
        check(_api().vlrbContextGetRenderOptions(self.h, ctypes.byref(o)), "getOptions")
        return {k: getattr(o, k) for k, _ in VLRBRenderOptions._fields_}

    def setGuiding(self, enabled=None, train=None, **kw):
        """vlrbContextSetGuiding; keyword names are the C struct's fields
        (log2TableSize, learningRate, samplesPerStep, stepsPerLaunch,
        recordBounces, warmupLaunches, weightClamp, trainInterval)."""
        o = VLRBGuidingOptions()
        check(_api().vlrbContextGetGuiding(self.h, ctypes.byref(o)), "getGuiding")
        if enabled is not None:
            o.enabled = enabled
        if train is not None:
            o.train = train
        for k, val in kw.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown guiding option {k}")
            setattr(o, k, val)
        check(_api().vlrbContextSetGuiding(self.h, ctypes.byref(o)), "setGuiding")

    def guide_net(self):
        """The context's guiding network as a vlr_b200.guide.GuideNet (borrowed)."""
        from .guide import GuideNet
        h = c_void_p()
        check(_api().vlrbContextGetGuideNet(self.h, ctypes.byref(h)), "getGuideNet")
        o = VLRBGuidingOptions()
        check(_api().vlrbContextGetGuiding(self.h, ctypes.byref(o)), "getGuiding")
        return GuideNet.from_handle(h, o.log2TableSize)

    def guiding_stats(self):
        st = VLRBGuidingStats()
        check(_api().vlrbContextGetGuidingStats(self.h, ctypes.byref(st)), "getGuidingStats")
        return {k: getattr(st, k) for k, _ in VLRBGuidingStats._fields_}

    def render(self, camera, first_frame, limit=1 << 30, stream=0, shrink=1, denoise=False):
        """One sample per pixel, exactly like vlrContextRender (shrink: the
        shrinkCoeff preview, fixed at a first frame; denoise: the output is
        the denoised image)."""
        n = ctypes.c_uint32()
        check(_api().vlrContextRender(self.h, c_void_p(stream), camera.h, bool(denoise), shrink, first_frame, limit,
                                      ctypes.byref(n)), "vlrContextRender")
        return n.value

    def read_aux(self):
        """(albedo, normal): the denoiser's guide images, height x width x 4 each."""
        a = np.empty((self.height, self.width, 4), np.float32)
        nrm = np.empty((self.height, self.width, 4), np.float32)
        check(_api().vlrbContextReadAuxBuffers(self.h, a.ctypes.data_as(c_void_p), nrm.ctypes.data_as(c_void_p)),
              "readAuxBuffers")
        return a, nrm

    def save_images(self, path_without_extension, brightness=1.0):
        """<path>.png (tone-mapped) and <path>.exr (linear half) of the output."""
        check(_api().vlrbContextSaveOutputImages(self.h, str(path_without_extension).encode(),
                                                 ctypes.c_float(brightness)), "saveOutputImages")

    def render_samples(self, camera, first_frame, samples, limit=1 << 30, stream=0):
        n = ctypes.c_uint32()
        check(_api().vlrbContextRenderSamples(self.h, c_void_p(stream), camera.h, first_frame, samples, limit,
                                              ctypes.byref(n)), "vlrbContextRenderSamples")
        return n.value

    def read_output(self, out=None):
        if out is None:
            out = np.empty((self.height, self.width, 4), np.float32)
        check(_api().vlrContextReadOutputBuffer(self.h, out.ctypes.data_as(c_void_p)), "readOutputBuffer")
        return out

    def read_film(self):
        f = np.empty((self.height, self.width, 16), np.float64)
        check(_api().vlrbContextReadFilm(self.h, f.ctypes.data_as(c_void_p)), "readFilm")
        return f

    def output_device_ptr(self):
        p = c_void_p()
        check(_api().vlrbContextGetOutputDevicePointer(self.h, ctypes.byref(p)), "outputPtr")
        return p.value

    def set_profiling(self, on):
        check(_api().vlrbContextSetProfiling(self.h, bool(on)), "setProfiling")

    def kernel_times(self, reset=False):
        ms = (ctypes.c_double * 6)()
        ln = (ctypes.c_uint64 * 6)()
        total = ctypes.c_uint64()
        check(_api().vlrbContextGetKernelTimes(self.h, ctypes.byref(ms), ctypes.byref(ln), ctypes.byref(total)),
              "getKernelTimes")
        if reset:
            check(_api().vlrbContextResetKernelTimes(self.h), "resetKernelTimes")
        names = ("camera", "trace", "shade", "shadow", "film", "guide")
        return {n: {"ms": ms[i], "launches": ln[i]} for i, n in enumerate(names)}, total.value

    def launch_param_bytes(self):
        b = ctypes.c_uint64()
        check(_api().vlrbContextGetLaunchParamBytes(self.h, ctypes.byref(b)), "launchParamBytes")
        return b.value

    def film_device_ptr(self):
        p = c_void_p()
        check(_api().vlrbContextGetFilmDevicePointer(self.h, ctypes.byref(p)), "filmPtr")
        return p.value

    def read_pixel_rng_states(self, count=None):
        """Per-pixel PCG32 states of the path tracer, in pixel order."""
        n = self.width * self.height if count is None else count
        out = np.zeros(n, np.uint64)
        check(_api().vlrbContextReadPixelRngStates(self.h, out.ctypes.data_as(c_void_p), ctypes.c_uint32(n)),
              "readPixelRngStates")
        return out

    def read_bounce_counters(self, bounces=16):
        """Queue lengths of the path tracer's last launch, [bounces, 16]
        (vlrbContextReadBounceCounters)."""
        out = np.zeros((bounces, 16), np.uint32)
        check(_api().vlrbContextReadBounceCounters(self.h, out.ctypes.data_as(c_void_p), ctypes.c_uint32(bounces)),
              "readBounceCounters")
        return out

    def stats(self):
        s = VLRBRenderStats()
        check(_api().vlrbContextGetStats(self.h, ctypes.byref(s)), "getStats")
        return {k: getattr(s, k) for k, _ in VLRBRenderStats._fields_}


class RenderBatch:
    """vlrbRenderBatch*: items = [(context, camera, samples, first_frame)];
    persistent: the plain items in one persistent kernel launch
    (VLRB_BATCH_PERSISTENT)."""

    def __init__(self, items, stream=0, persistent=False):
        self.n = len(items)
        arr = (VLRBBatchItem * self.n)()
        for i, (ctx, cam, spp, first) in enumerate(items):
            arr[i] = VLRBBatchItem(ctx.h.value if hasattr(ctx.h, "value") else ctx.h, cam.h.value
                                   if hasattr(cam.h, "value") else cam.h, spp, first)
        self.h = c_void_p()
        check(_api().vlrbRenderBatchCreateEx(arr, self.n, c_void_p(stream), ctypes.c_uint32(1 if persistent else 0),
                                             ctypes.byref(self.h)), "batchCreate")

    def launch(self, stream=0):
        check(_api().vlrbRenderBatchLaunch(self.h, c_void_p(stream)), "batchLaunch")

    def item_times(self):
        ms = (ctypes.c_float * self.n)()
        check(_api().vlrbRenderBatchItemTimes(self.h, ms), "batchItemTimes")
        return list(ms)

    def close(self):
        if self.h:
            _api().vlrbRenderBatchDestroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_images(rgba, path_without_extension, brightness=1.0):
    """vlrbWriteOutputImages: <path>.png and <path>.exr from an H x W x 4 float image."""
    a = np.ascontiguousarray(rgba, np.float32)
    h, w = a.shape[:2]
    check(_api().vlrbWriteOutputImages(a.ctypes.data_as(c_void_p), w, h, str(path_without_extension).encode(),
                                       ctypes.c_float(brightness)), "writeOutputImages")


def quat_rotate_y(angle):
    return (0.0, math.sin(angle / 2), 0.0, math.cos(angle / 2))


__all__ = ["Context", "RenderBatch", "rgb", "Spectrum", "VLRError", "quat_rotate_y", "RENDERER_PATH_TRACING",
           "RENDERER_LIGHT_TRACING", "RENDERER_BPT"]
