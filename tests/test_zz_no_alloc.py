"""The allocation-free LBVH build (vlrbBvhBuildNoAlloc) against the regular
entry point (vlrbBvhBuildHost): same codes, permutation, hierarchy, boxes and
traversal nodes, bit for bit, on two calls in a row.  Collected last so it
also runs after the rest of the GPU suite has used the device.

The entry point exists for callers that may not allocate device memory while
they run (an application whose device memory belongs to its own pool, or a
per-frame rebuild inside a fixed budget); its scratch is a static device
array, so it is limited to 65,536 triangles per call."""
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
    ch = np.zeros(max(2 * (n - 1), 1), np.int32)
    bx = np.zeros(max(6 * (n - 1), 1), np.float32)
    assert L.vlrbBvhBuildHost(P(v), n, P(codes), P(prims), P(ch), P(bx), None) == 0
    return codes, prims, ch[: 2 * (n - 1)], bx[: 6 * (n - 1)]


def _no_alloc_build(L, v):
    import torch
    n = v.shape[0]
    dev = torch.device("cuda")
    dv = torch.from_numpy(v).to(dev)
    codes = torch.empty(n, dtype=torch.int32, device=dev)
    prims = torch.empty(n, dtype=torch.int32, device=dev)
    tris = torch.empty(n * 48, dtype=torch.uint8, device=dev)
    if n > 1:
        ch = torch.empty(2 * (n - 1), dtype=torch.int32, device=dev)
        bx = torch.empty(6 * (n - 1), dtype=torch.float32, device=dev)
        nodes = torch.empty((n - 1) * 64, dtype=torch.uint8, device=dev)
        ptrs = (ch.data_ptr(), bx.data_ptr(), nodes.data_ptr())
    else:   # a single triangle has no internal node: those outputs may be NULL
        ptrs = (None, None, None)
    stream = torch.cuda.current_stream()
    rc = L.vlrbBvhBuildNoAlloc(dv.data_ptr(), n, codes.data_ptr(), prims.data_ptr(), *ptrs,
                               tris.data_ptr(), stream.cuda_stream)
    assert rc == 0
    stream.synchronize()
    tri = tris.view(torch.float32).view(n, 12).cpu().numpy()
    if n > 1:
        got = (ch.cpu().numpy(), bx.cpu().numpy(), nodes.view(torch.float32).view(n - 1, 16).cpu().numpy())
    else:
        got = (np.zeros(0, np.int32), np.zeros(0, np.float32), np.zeros((0, 16), np.float32))
    return (codes.cpu().numpy().view(np.uint32), prims.cpu().numpy().view(np.uint32)) + got + (tri,)


def _check_nodes(nodes, children, boxes, prims, v):
    """Each traversal node holds its two children's references and boxes: an
    internal child's box from nodeBoxes, a leaf's from its triangle."""
    n1 = nodes.shape[0]
    if n1 == 0:
        return
    assert np.array_equal(nodes[:, 3].view(np.int32), children[0::2])
    assert np.array_equal(nodes[:, 11].view(np.int32), children[1::2])
    tv = v.reshape(-1, 3, 3)
    tlo, thi = tv.min(axis=1), tv.max(axis=1)
    bx = boxes.reshape(-1, 6)
    for k, (lo_off, hi_off) in enumerate(((0, 4), (8, 12))):
        c = children[k::2]
        internal = c >= 0
        exp_lo = np.where(internal[:, None], bx[np.where(internal, c, 0), 0:3], tlo[prims[np.where(internal, 0, ~c)]])
        exp_hi = np.where(internal[:, None], bx[np.where(internal, c, 0), 3:6], thi[prims[np.where(internal, 0, ~c)]])
        assert np.array_equal(nodes[:, lo_off:lo_off + 3], exp_lo), k
        assert np.array_equal(nodes[:, hi_off:hi_off + 3], exp_hi), k


def test_no_alloc_build_matches_regular_entry_twice():
    L = _lib()
    for n, seed in ((MAX_TRIS, 11), (5003, 12), (2, 13), (1, 14)):
        v = _triangles(n, seed)
        ref = _host_build(L, v)
        for _ in range(2):          # two calls in a row share the static scratch
            got = _no_alloc_build(L, v)
            for name, a, b in zip(("codes", "prims", "children", "boxes"), got[:4], ref):
                assert np.array_equal(a, b), (n, name)
            _check_nodes(got[4], ref[2], ref[3], ref[1], v)
            # the sorted triangles carry the original primitive index and vertex 0
            tri = got[5]
            assert np.array_equal(tri[:, 3].view(np.uint32), ref[1])
            assert np.array_equal(tri[:, 0:3], v[ref[1], 0:3])


def test_no_alloc_build_rejects_more_than_its_limit():
    L = _lib()
    rc = L.vlrbBvhBuildNoAlloc(None, MAX_TRIS + 1, None, None, None, None, None, None, None)
    assert rc == INVALID_ARGUMENT
