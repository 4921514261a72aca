"""ctypes access to the reference's own host-compiled BSDF/spectral code
(oracle/_ref/libvlrref.so, built by oracle/build_ref.sh).
TEST INFRASTRUCTURE ONLY."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libvlrref.so")
_lib = None

BATCH_INPUTS = ("wo", "material", "roughness", "ior", "albedo", "metallic", "u", "wavelengthU")
BATCH_OUTPUTS = {"value": 4, "pdf": 1, "wi": 3, "evalValue": 4, "evalPdf": 1}


def available():
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(REF_LIB)
        _lib.vlrref_init()
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def bsdf_batch(inputs, threads=0):
    """Run the reference BSDF classes over a batch (see vlrref_bsdf_batch)."""
    n = len(inputs["material"])
    ins = [np.ascontiguousarray(inputs[k]) for k in BATCH_INPUTS]
    outs = {k: np.zeros((n, c) if c > 1 else n, np.float32) for k, c in BATCH_OUTPUTS.items()}
    lib().vlrref_bsdf_batch(ctypes.c_int64(n), ctypes.c_int(threads), *[_p(a) for a in ins],
                            *[_p(outs[k]) for k in BATCH_OUTPUTS])
    return outs


def upsample(sp_type, color_space, e0, e1, e2):
    out = (ctypes.c_uint32 * 3)()
    lib().vlrref_upsample(sp_type, color_space, ctypes.c_float(e0), ctypes.c_float(e1),
                          ctypes.c_float(e2), out)
    return tuple(out)


def tables():
    """(grid bytes [168*8], points float32 [186*99], cmf16 [3,16], integralCMF)."""
    g = ctypes.c_void_p()
    p = ctypes.c_void_p()
    c = ctypes.POINTER(ctypes.c_float)()
    integ = ctypes.c_float()
    lib().vlrref_tables(ctypes.byref(g), ctypes.byref(p), ctypes.byref(c), ctypes.byref(integ))
    grid = np.ctypeslib.as_array(ctypes.cast(g, ctypes.POINTER(ctypes.c_uint8)), (168 * 8,)).copy()
    pts = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_float)), (186 * 99,)).copy()
    cmf = np.ctypeslib.as_array(c, (48,)).copy().reshape(3, 16)
    return grid, pts, cmf, integ.value
