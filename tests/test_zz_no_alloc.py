"""The allocation-free LBVH build (vlrbBvhBuildNoAlloc) against the regular
entry point (vlrbBvhBuildHost): same codes, permutation, hierarchy and boxes,
bit for bit, on two calls in a row.  Collected last so it also runs after the
rest of the GPU suite has used the device."""
import ctypes

import numpy as np
import pytest

import vlr_b200 as V

pytestmark = pytest.mark.gpu

MAX_TRIS = 65536
INVALID_ARGUMENT = 3


def _lib():
    L = V.lib()
    L.vlrbBvhBuildHost.argtypes = [ctypes.c_void_p, ctypes.c_uint32] + [ctypes.c_void_p] * 5
    L.vlrbBvhBuildHost.restype = ctypes.c_int
    L.vlrbBvhBuildNoAlloc.argtypes = [ctypes.c_void_p, ctypes.c_uint32] + [ctypes.c_void_p] * 7
    L.vlrbBvhBuildNoAlloc.restype = ctypes.c_int
    return L


def _triangles(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-10, 10, (n, 1, 3)).astype(np.float32)
    v = (c + rng.normal(0, 0.05, (n, 3, 3))).astype(np.float32).reshape(n, 9)
    v[: n // 50] = v[0]          # duplicates: equal Morton codes
    return v


def _host_build(L, v):
    n = v.shape[0]
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    codes = np.zeros(n, np.uint32)
    prims = np.zeros(n, np.uint32)
    ch = np.zeros(2 * (n - 1), np.int32)
    bx = np.zeros(6 * (n - 1), np.float32)
    assert L.vlrbBvhBuildHost(P(v), n, P(codes), P(prims), P(ch), P(bx), None) == 0
    return codes, prims, ch, bx


def _no_alloc_build(L, v):
    import torch
    n = v.shape[0]
    dev = torch.device("cuda")
    dv = torch.from_numpy(v).to(dev)
    codes = torch.empty(n, dtype=torch.int32, device=dev)
    prims = torch.empty(n, dtype=torch.int32, device=dev)
    ch = torch.empty(2 * (n - 1), dtype=torch.int32, device=dev)
    bx = torch.empty(6 * (n - 1), dtype=torch.float32, device=dev)
    nodes = torch.empty((n - 1) * 64, dtype=torch.uint8, device=dev)
    tris = torch.empty(n * 48, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    rc = L.vlrbBvhBuildNoAlloc(dv.data_ptr(), n, codes.data_ptr(), prims.data_ptr(), ch.data_ptr(),
                               bx.data_ptr(), nodes.data_ptr(), tris.data_ptr(), stream.cuda_stream)
    assert rc == 0
    stream.synchronize()
    tri = tris.view(torch.float32).view(n, 12).cpu().numpy()
    return (codes.cpu().numpy().view(np.uint32), prims.cpu().numpy().view(np.uint32),
            ch.cpu().numpy(), bx.cpu().numpy(), tri)


def test_no_alloc_build_matches_regular_entry_twice():
    L = _lib()
    for n, seed in ((MAX_TRIS, 11), (5003, 12)):
        v = _triangles(n, seed)
        ref = _host_build(L, v)
        got = _no_alloc_build(L, v)
        for name, a, b in zip(("codes", "prims", "children", "boxes"), got[:4], ref):
            assert np.array_equal(a, b), (n, name)
        # the sorted triangles carry the original primitive index and vertex 0
        tri = got[4]
        assert np.array_equal(tri[:, 3].view(np.uint32), ref[1])
        assert np.array_equal(tri[:, 0:3], v[ref[1], 0:3])


def test_no_alloc_build_rejects_more_than_its_limit():
    L = _lib()
    rc = L.vlrbBvhBuildNoAlloc(None, MAX_TRIS + 1, None, None, None, None, None, None, None)
    assert rc == INVALID_ARGUMENT
