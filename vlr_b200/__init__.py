"""Python host bindings for libvlr_b200.so (ctypes over the C ABI).

The library is the product; this module only loads it and converts numpy /
torch buffers into the pointers the C entry points take.  Importing never
falls back to anything: if the shared library is missing, `lib()` raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvlr_b200.so")
_lib = None

# VLRResult codes (include/vlr/vlr.h)
NO_ERROR = 0
INVALID_CONTEXT = 1
INVALID_INSTANCE = 2
INVALID_ARGUMENT = 3
INCOMPATIBLE_NODE_TYPE = 4
INTERNAL_ERROR = 5

MATERIALS = ("Matte", "SpecularReflection", "MicrofacetReflection",
             "MicrofacetScattering", "LambertianScattering", "UE4")


class VLRError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed with VLRResult {code}")
        self.code = code


class _BsdfBatch(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int64)] + [
        (name, ctypes.c_void_p) for name in (
            "wo", "material", "roughness", "ior", "albedo", "metallic", "u", "wavelengthU",
            "value", "pdf", "wi", "evalValue", "evalPdf")]


def lib():
    """Load libvlr_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m vlr_b200.build`")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.vlrbVersion.restype = ctypes.c_char_p
        _lib.vlrbBsdfBatch.argtypes = [ctypes.POINTER(_BsdfBatch), ctypes.c_void_p]
        _lib.vlrbBsdfBatchHost.argtypes = [ctypes.POINTER(_BsdfBatch), ctypes.POINTER(ctypes.c_float)]
        _lib.vlrbBsdfBatchHostEx.argtypes = [ctypes.POINTER(_BsdfBatch), ctypes.c_uint32,
                                             ctypes.POINTER(ctypes.c_float)]
    return _lib


def check(code, what):
    if code != NO_ERROR:
        raise VLRError(code, what)


BATCH_INPUTS = ("wo", "material", "roughness", "ior", "albedo", "metallic", "u", "wavelengthU")
BATCH_OUTPUTS = {"value": 4, "pdf": 1, "wi": 3, "evalValue": 4, "evalPdf": 1}


def make_bsdf_batch_inputs(n, seed=0, materials=6):
    """Seeded synthetic BSDF-batch queries: material uniform over the first
    `materials` ids (6: the six BSDFs of the shading-batch workload; 7 adds
    SpecularScattering), wo uniform on the sphere, roughness log-uniform in [0.01, 1] per
    axis, IOR uniform in [1.3, 1.8], albedo and metallic uniform in [0, 1],
    three uniform numbers for (uComponent, uDir0, uDir1) and two for the
    wavelength offset and hero selection."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    wo = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1).astype(np.float32)
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    return {
        "wo": np.ascontiguousarray(wo, dtype=np.float32),
        "material": rng.integers(0, materials, n).astype(np.uint32),
        "roughness": np.exp(rng.uniform(np.log(0.01), 0.0, (n, 2))).astype(np.float32),
        "ior": rng.uniform(1.3, 1.8, n).astype(np.float32),
        "albedo": rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32),
        "metallic": rng.uniform(0.0, 1.0, n).astype(np.float32),
        "u": rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32),
        "wavelengthU": rng.uniform(0.0, 1.0, (n, 2)).astype(np.float32),
    }


def _ptr(a):
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def bsdf_batch_host(inputs, contracted=False, outputs=None):
    """Run the BSDF batch from host numpy arrays (copies in and out).
    contracted: run the copy of the kernel compiled with FMA contraction (the
    renderers' arithmetic) instead of the exactly rounded one.  outputs: host
    arrays to write (e.g. pinned), else new ones.
    Returns (outputs dict, kernel milliseconds)."""
    n = len(inputs["material"])
    outs = outputs if outputs is not None else \
        {k: np.zeros((n, c) if c > 1 else n, np.float32) for k, c in BATCH_OUTPUTS.items()}
    ins = {k: np.ascontiguousarray(inputs[k]) for k in BATCH_INPUTS}
    b = _BsdfBatch(n, *[_ptr(ins[k]).value for k in BATCH_INPUTS],
                   *[_ptr(outs[k]).value for k in BATCH_OUTPUTS])
    ms = ctypes.c_float(0.0)
    check(lib().vlrbBsdfBatchHostEx(ctypes.byref(b), ctypes.c_uint32(1 if contracted else 0), ctypes.byref(ms)),
          "vlrbBsdfBatchHostEx")
    return outs, ms.value


def bsdf_batch_device(ins, outs, stream=0):
    """Run the BSDF batch on device tensors (torch CUDA tensors or raw
    integer device addresses) on `stream` (a CUstream handle)."""
    n = len(ins["material"])
    b = _BsdfBatch(n, *[_ptr(ins[k]).value for k in BATCH_INPUTS],
                   *[_ptr(outs[k]).value for k in BATCH_OUTPUTS])
    check(lib().vlrbBsdfBatch(ctypes.byref(b), ctypes.c_void_p(stream)), "vlrbBsdfBatch")
