"""ctypes binding of the learned path-guiding network (include/vlrb.h,
vlrbGuideNet*).  All compute runs in libvlr_b200.so on the GPU."""
import ctypes
from ctypes import c_void_p, c_uint32, c_uint64, c_float

import numpy as np

from . import lib, check

N_WEIGHTS = 15360
N_RAW = 40
SAMPLE_FLOATS = 16


def _api():
    L = lib()
    if not getattr(L, "_guide_bound", False):
        L.vlrbGuideNetCreate.argtypes = [c_uint32, c_uint64, ctypes.POINTER(c_void_p)]
        L.vlrbGuideNetDestroy.argtypes = [c_void_p]
        L.vlrbGuideNetSetBounds.argtypes = [c_void_p, c_void_p, c_void_p]
        L.vlrbGuideNetGetSizes.argtypes = [c_void_p, ctypes.POINTER(c_uint32), ctypes.POINTER(c_uint64)]
        L.vlrbGuideNetGetParams.argtypes = [c_void_p, c_void_p, c_void_p]
        L.vlrbGuideNetSetParams.argtypes = [c_void_p, c_void_p, c_void_p]
        L.vlrbGuideNetInferHost.argtypes = [c_void_p, c_uint32, c_void_p, c_void_p, c_void_p, c_void_p]
        L.vlrbGuideNetGradientsHost.argtypes = [c_void_p, c_uint32, c_void_p, c_void_p, c_void_p,
                                                ctypes.POINTER(c_float)]
        L.vlrbGuideNetTrainHost.argtypes = [c_void_p, c_uint32, c_void_p, c_float, c_uint32, c_void_p]
        L._guide_bound = True
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


class GuideNet:
    """vlrbGuideNet: hash-grid + MLP -> 8-lobe vMF mixture."""

    def __init__(self, log2_table=19, seed=1):
        self.h = c_void_p()
        self.log2_table = log2_table
        check(_api().vlrbGuideNetCreate(log2_table, seed, ctypes.byref(self.h)), "vlrbGuideNetCreate")
        nw, ng = c_uint32(), c_uint64()
        check(_api().vlrbGuideNetGetSizes(self.h, ctypes.byref(nw), ctypes.byref(ng)), "getSizes")
        self.n_weights, self.n_grid = nw.value, ng.value

    @classmethod
    def from_handle(cls, h, log2_table):
        """Wrap an existing handle (e.g. vlrbContextGetGuideNet's)."""
        self = cls.__new__(cls)
        self.h = h
        self.log2_table = log2_table
        nw, ng = c_uint32(), c_uint64()
        check(_api().vlrbGuideNetGetSizes(self.h, ctypes.byref(nw), ctypes.byref(ng)), "getSizes")
        self.n_weights, self.n_grid = nw.value, ng.value
        return self

    def close(self):
        if self.h:
            _api().vlrbGuideNetDestroy(self.h)
            self.h = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_bounds(self, lo, hi):
        lo = np.asarray(lo, np.float32)
        hi = np.asarray(hi, np.float32)
        check(_api().vlrbGuideNetSetBounds(self.h, _p(lo), _p(hi)), "setBounds")

    def params(self):
        w = np.zeros(self.n_weights, np.float32)
        g = np.zeros(self.n_grid, np.float32)
        check(_api().vlrbGuideNetGetParams(self.h, _p(w), _p(g)), "getParams")
        return w, g

    def set_params(self, weights=None, grid=None):
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        g = None if grid is None else np.ascontiguousarray(grid, np.float32)
        check(_api().vlrbGuideNetSetParams(self.h, _p(w), _p(g)), "setParams")

    def infer(self, pos, wo, nrm):
        pos, wo, nrm = (np.ascontiguousarray(a, np.float32) for a in (pos, wo, nrm))
        n = pos.shape[0]
        raw = np.zeros((n, N_RAW), np.float32)
        check(_api().vlrbGuideNetInferHost(self.h, n, _p(pos), _p(wo), _p(nrm), _p(raw)), "infer")
        return raw

    def gradients(self, samples):
        s = np.ascontiguousarray(samples, np.float32)
        wg = np.zeros(self.n_weights, np.float32)
        gg = np.zeros(self.n_grid, np.float32)
        loss = c_float()
        check(_api().vlrbGuideNetGradientsHost(self.h, s.shape[0], _p(s), _p(wg), _p(gg), ctypes.byref(loss)),
              "gradients")
        return loss.value, wg, gg

    def train(self, samples, lr=1e-2, steps=1):
        s = np.ascontiguousarray(samples, np.float32)
        losses = np.zeros(steps, np.float32)
        check(_api().vlrbGuideNetTrainHost(self.h, s.shape[0], _p(s), lr, steps, _p(losses)), "train")
        return losses
