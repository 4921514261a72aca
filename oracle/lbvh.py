"""ctypes access to the host LBVH oracle (oracle/lbvh_host.c).
TEST INFRASTRUCTURE ONLY."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build():
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-o", LIB, os.path.join(HERE, "lbvh_host.c")])


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "lbvh_host.c")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            build()
        _lib = ctypes.CDLL(LIB)
    return _lib


def build_lbvh(tri_verts):
    v = np.ascontiguousarray(tri_verts, np.float32).reshape(-1, 9)
    n = v.shape[0]
    codes = np.zeros(n, np.uint32)
    prims = np.zeros(n, np.uint32)
    ch = np.zeros(max(n - 1, 1) * 2, np.int32)
    boxes = np.zeros(max(n - 1, 1) * 6, np.float32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib().oracle_lbvh_build(P(v), ctypes.c_uint32(n), P(codes), P(prims), P(ch), P(boxes))
    assert rc == 0
    return codes, prims, ch[: 2 * (n - 1)], boxes[: 6 * (n - 1)]


def optimize_lbvh(tri_verts, prims, children, boxes, rounds=3):
    """Treelet restructuring of an LBVH from build_lbvh (copies modified);
    returns (children, boxes, number of treelets rebuilt)."""
    v = np.ascontiguousarray(tri_verts, np.float32).reshape(-1, 9)
    n = v.shape[0]
    ch = np.ascontiguousarray(children, np.int32).copy()
    bx = np.ascontiguousarray(boxes, np.float32).copy()
    pr = np.ascontiguousarray(prims, np.uint32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = lib().oracle_lbvh_optimize(P(v), ctypes.c_uint32(n), P(pr), P(ch), P(bx), ctypes.c_uint32(rounds))
    assert rc >= 0
    return ch, bx, rc
