"""CPU restatement of the guiding network (TEST INFRASTRUCTURE ONLY: the
oracle for the tensor-core kernels in vlr_b200/csrc/guide_*.cuh).

The reference renderer has no learned guiding, so there is no reference code
to follow; this module restates the network the library documents (header
include/vlrb.h, "Learned path-guiding network") in numpy, float64:

  encoding   multi-resolution hash grid over the normalised position (16
             levels x 2 features, trilinear, dense indexing while
             (res+1)^3 fits the table, else the spatial hash of Mueller et al.
             2022), real spherical harmonics of degree <= 3 of the outgoing
             direction and of the shading normal;
  MLP        64-64-64-64-48, ReLU, no biases; the kernels round every layer
             input (features, activations, weights) to BF16 and accumulate
             in FP32 -- the oracle rounds the same tensors to BF16 and
             accumulates in float64;
  output     8 von Mises-Fisher lobes (direction, log concentration clamped
             to [-4, 8], softmax logit);
  loss       sum_j (w_j / sum w) * -log q(wi_j) and its gradient, backward
             through the MLP (gradients of BF16-rounded upstream values) to
             the weights and the hash-grid entries.

`finite_difference_check` validates the analytic backward pass of this
oracle against central differences on the unrounded float64 network."""
import math

import numpy as np

LEVELS = 16
FEAT = 2
N_IN = 64
N_HID = 64
N_OUT = 48
N_RAW = 40
LOBES = 8
LAYER_OUT = (64, 64, 64, 48)
W_OFF = (0, 4096, 8192, 12288, 15360)
LOG_KAPPA_MIN, LOG_KAPPA_MAX = -4.0, 8.0


def bf16(x):
    """Round float64/float32 values to BF16 (round to nearest even) and back."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def level_scales():
    g = math.exp(math.log(2048.0 / 16.0) / (LEVELS - 1))
    return [float(np.float32(math.floor(16.0 * math.pow(g, l)))) for l in range(LEVELS)]


def corners(p, res, log2t):
    """Table indices [n,8] and trilinear weights [n,8] of one level
    (FP32 position arithmetic, as on the device)."""
    T = 1 << log2t
    ires = int(res)
    dense = (ires + 1) ** 3 <= T
    p = p.astype(np.float32)
    x = p * np.float32(res)
    c = np.minimum(np.floor(x).astype(np.int64), ires - 1)
    t = (x - c.astype(np.float32)).astype(np.float32)
    idx = np.zeros((p.shape[0], 8), np.int64)
    w = np.zeros((p.shape[0], 8), np.float64)
    for k in range(8):
        d = np.array([k & 1, (k >> 1) & 1, k >> 2])
        cc = c + d
        wk = np.where(d[None, :] == 1, t, np.float32(1) - t).astype(np.float64)
        w[:, k] = wk[:, 0] * wk[:, 1] * wk[:, 2]
        if dense:
            idx[:, k] = cc[:, 0] + (ires + 1) * (cc[:, 1] + (ires + 1) * cc[:, 2])
        else:
            h = (cc[:, 0].astype(np.uint64) * np.uint64(1)) ^ (cc[:, 1].astype(np.uint64) * np.uint64(2654435761)) \
                ^ (cc[:, 2].astype(np.uint64) * np.uint64(805459861))
            idx[:, k] = (h & np.uint64(0xFFFFFFFF) & np.uint64(T - 1)).astype(np.int64)
    return idx, w


def sh16(d):
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([
        np.full_like(x, 0.28209479177), 0.48860251190 * y, 0.48860251190 * z, 0.48860251190 * x,
        1.09254843059 * x * y, 1.09254843059 * y * z, 0.31539156525 * (3 * zz - 1), 1.09254843059 * x * z,
        0.54627421529 * (xx - yy), 0.59004358992 * y * (3 * xx - yy), 2.89061144264 * x * y * z,
        0.45704579946 * y * (5 * zz - 1), 0.37317633259 * z * (5 * zz - 3), 0.45704579946 * x * (5 * zz - 1),
        1.44530572132 * z * (xx - yy), 0.59004358992 * x * (xx - 3 * yy)], axis=1)


def normalise(pos, lo, hi):
    lo = np.asarray(lo, np.float32)
    inv = np.where(np.asarray(hi, np.float32) > lo, np.float32(1) / (np.asarray(hi, np.float32) - lo), np.float32(1))
    return np.clip((pos.astype(np.float32) - lo) * inv.astype(np.float32), 0, 1).astype(np.float32)


def encode(grid, log2t, p01, wo, nrm):
    """Features [n,64] plus the per-level corner data for the backward pass."""
    n = p01.shape[0]
    feats = np.zeros((n, N_IN))
    cache = []
    scales = level_scales()
    g = grid.reshape(LEVELS, 1 << log2t, FEAT).astype(np.float64)
    for l in range(LEVELS):
        idx, w = corners(p01, scales[l], log2t)
        feats[:, 2 * l:2 * l + 2] = np.einsum("nk,nkf->nf", w, g[l][idx])
        cache.append((idx, w))
    feats[:, 32:48] = sh16(wo.astype(np.float64))
    feats[:, 48:64] = sh16(nrm.astype(np.float64))
    return feats, cache


def layers(weights):
    w = np.asarray(weights, np.float64)
    return [w[W_OFF[l]:W_OFF[l + 1]].reshape(LAYER_OUT[l], N_IN) for l in range(4)]


def forward(weights, feats, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    Ws = [r(W) for W in layers(weights)]
    acts = [r(feats)]
    for l in range(3):
        acts.append(r(np.maximum(acts[-1] @ Ws[l].T, 0.0)))
    y = acts[-1] @ Ws[3].T
    return y, acts, Ws


def decode(raw):
    """Mixture parameters from raw outputs [n,40]: mu [n,8,3], kappa, weights."""
    r = raw[:, :N_RAW].reshape(-1, LOBES, 5)
    v = r[:, :, 0:3]
    ln = np.linalg.norm(v, axis=2, keepdims=True)
    mu = np.where(ln > 1e-12, v / np.maximum(ln, 1e-300), np.array([0.0, 0.0, 1.0]))
    kappa = np.exp(np.clip(r[:, :, 3], LOG_KAPPA_MIN, LOG_KAPPA_MAX))
    lg = r[:, :, 4] - r[:, :, 4].max(axis=1, keepdims=True)
    pi = np.exp(lg) / np.exp(lg).sum(axis=1, keepdims=True)
    return mu, kappa, pi


def log_vmf_norm(kappa):
    return np.log(kappa) - math.log(2 * math.pi) - np.log1p(-np.exp(-2 * kappa))


def mixture_pdf(raw, w):
    mu, kappa, pi = decode(raw)
    cos = np.einsum("nkc,nc->nk", mu, w)
    return (pi * np.exp(log_vmf_norm(kappa) + kappa * (cos - 1))).sum(axis=1)


def loss_and_dy(raw, wi, wnorm):
    """Per-sample loss -w log q and its gradient w.r.t. the 48 raw outputs."""
    n = raw.shape[0]
    r = raw[:, :N_RAW].reshape(n, LOBES, 5)
    v = r[:, :, 0:3]
    ln = np.linalg.norm(v, axis=2)
    mu = np.where(ln[..., None] > 1e-12, v / np.maximum(ln, 1e-300)[..., None], np.array([0.0, 0.0, 1.0]))
    s = r[:, :, 3]
    kappa = np.exp(np.clip(s, LOG_KAPPA_MIN, LOG_KAPPA_MAX))
    lg = r[:, :, 4] - r[:, :, 4].max(axis=1, keepdims=True)
    logpi = lg - np.log(np.exp(lg).sum(axis=1, keepdims=True))
    cos = np.einsum("nkc,nc->nk", mu, wi)
    logc = logpi + log_vmf_norm(kappa) + kappa * (cos - 1)
    m = logc.max(axis=1, keepdims=True)
    logq = m[:, 0] + np.log(np.exp(logc - m).sum(axis=1))
    resp = np.exp(logc - logq[:, None])
    pi = np.exp(logpi)
    W = wnorm[:, None]
    dy = np.zeros((n, N_OUT))
    d = dy[:, :N_RAW].reshape(n, LOBES, 5)
    d[:, :, 4] = -W * (resp - pi)
    inside = (s > LOG_KAPPA_MIN) & (s < LOG_KAPPA_MAX)
    dk = 1 / kappa - 2 / np.expm1(2 * kappa) + (cos - 1)
    d[:, :, 3] = np.where(inside, -W * resp * kappa * dk, 0.0)
    g = wi[:, None, :] * (-W * resp * kappa)[..., None]
    gv = (g - mu * np.einsum("nkc,nkc->nk", mu, g)[..., None]) / np.maximum(ln, 1e-300)[..., None]
    d[:, :, 0:3] = np.where(ln[..., None] > 1e-12, gv, 0.0)
    dy[:, :N_RAW] = d.reshape(n, N_RAW)
    return -wnorm * logq, dy


def gradients(weights, grid, log2t, samples, lo, hi, rounding=True):
    """Loss, weight gradient [15360] and grid gradient of one batch.
    samples: [n,16] float32 rows (pos, weight, wo, -, nrm, -, wi, -)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    pos, wgt = samples[:, 0:3], samples[:, 3].astype(np.float64)
    wo, nrm, wi = samples[:, 4:7], samples[:, 8:11], samples[:, 12:15].astype(np.float64)
    p01 = normalise(pos, lo, hi)
    feats, cache = encode(grid, log2t, p01, wo, nrm)
    y, acts, Ws = forward(weights, feats, rounding)
    wnorm = wgt / max(wgt.sum(), 1e-30)
    loss, dy = loss_and_dy(y, wi, wnorm)
    dW = [None] * 4
    dz = r(dy)
    dz[:, N_RAW:] = 0
    for l in range(3, -1, -1):
        dW[l] = dz.T @ acts[l]
        da = dz @ Ws[l]
        if l > 0:
            dz = r(np.where(acts[l] > 0, da, 0.0))
    dx = da
    wg = np.zeros(W_OFF[4])
    for l in range(4):
        g = dW[l][:LAYER_OUT[l]]
        if l == 3:
            g = g.copy()
            g[N_RAW:] = 0
        wg[W_OFF[l]:W_OFF[l + 1]] = g.reshape(-1)
    gg = np.zeros((LEVELS, 1 << log2t, FEAT))
    for l in range(LEVELS):
        idx, w = cache[l]
        for f in range(FEAT):
            np.add.at(gg[l, :, f], idx.reshape(-1), (w * dx[:, 2 * l + f][:, None]).reshape(-1))
    return loss.sum(), wg, gg.reshape(-1)


def finite_difference_check(seed=0, n=64, log2t=8, eps=1e-6):
    """Largest relative error between the analytic float64 gradient and
    central differences, over a handful of weights and grid entries."""
    rng = np.random.default_rng(seed)
    weights = rng.normal(0, 0.3, W_OFF[4])
    weights[W_OFF[3] + N_RAW * N_IN:] = 0
    grid = rng.normal(0, 0.5, LEVELS * FEAT << log2t)
    samples = random_samples(rng, n)
    lo, hi = (0, 0, 0), (1, 1, 1)
    _, wg, gg = gradients(weights, grid, log2t, samples, lo, hi, rounding=False)

    def f(wv, gv):
        return gradients(wv, gv, log2t, samples, lo, hi, rounding=False)[0]

    worst = 0.0
    for i in rng.choice(W_OFF[4] - 8 * N_IN, 12, replace=False):
        a, b = weights.copy(), weights.copy()
        a[i] += eps
        b[i] -= eps
        num = (f(a, grid) - f(b, grid)) / (2 * eps)
        worst = max(worst, abs(num - wg[i]) / max(abs(num), abs(wg[i]), 1e-6))
    touched = np.nonzero(gg)[0]
    for i in rng.choice(touched, min(12, len(touched)), replace=False):
        a, b = grid.copy(), grid.copy()
        a[i] += eps
        b[i] -= eps
        num = (f(weights, a) - f(weights, b)) / (2 * eps)
        worst = max(worst, abs(num - gg[i]) / max(abs(num), abs(gg[i]), 1e-6))
    return worst


def random_samples(rng, n):
    """Training samples [n,16] float32 with unit directions."""
    def unit(k):
        v = rng.normal(size=(k, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)
    s = np.zeros((n, 16), np.float32)
    s[:, 0:3] = rng.uniform(0, 1, (n, 3))
    s[:, 3] = rng.uniform(0.1, 2.0, n)
    s[:, 4:7] = unit(n)
    s[:, 8:11] = unit(n)
    s[:, 12:15] = unit(n)
    return s
