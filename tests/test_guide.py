"""Learned path guiding: the tensor-core network against the CPU oracle
(oracle/guide_ref.py), and training on a known target distribution."""
import numpy as np
import pytest

from oracle import guide_ref as G

LOG2T = 12


def test_oracle_backward_matches_finite_differences():
    """The oracle's analytic loss gradient (float64, unrounded network)
    against central differences, weights and hash-grid entries."""
    assert G.finite_difference_check(seed=0) < 1e-4
    assert G.finite_difference_check(seed=3, n=16) < 1e-4


def test_oracle_mixture_is_normalised():
    """The decoded vMF mixture integrates to one over the sphere."""
    rng = np.random.default_rng(5)
    raw = rng.normal(0, 1.0, (1, G.N_RAW))
    raw[0, 3::5] = rng.uniform(-3, 4, G.LOBES)
    n = 200000
    u = rng.uniform(size=(n, 2))
    z = 1 - 2 * u[:, 0]
    r = np.sqrt(np.maximum(0, 1 - z * z))
    w = np.stack([r * np.cos(2 * np.pi * u[:, 1]), r * np.sin(2 * np.pi * u[:, 1]), z], axis=1)
    q = G.mixture_pdf(np.repeat(raw, n, axis=0), w)
    assert abs(q.mean() * 4 * np.pi - 1) < 0.02


def _random_net(seed):
    from vlr_b200.guide import GuideNet
    rng = np.random.default_rng(seed)
    net = GuideNet(LOG2T, seed=seed)
    w = rng.normal(0, 0.25, G.W_OFF[4]).astype(np.float32)
    w[G.W_OFF[3] + G.N_RAW * G.N_IN:] = 0
    g = rng.normal(0, 0.5, net.n_grid).astype(np.float32)
    net.set_params(w, g)
    net.set_bounds((-1, -1, -1), (1, 1, 1))
    return net, w, g


@pytest.mark.gpu
def test_inference_matches_oracle():
    """Forward pass (hash grid, SH, four BF16 tensor-core layers) against the
    oracle with the same BF16 rounding points.  Tolerance: 2% of the output
    scale per value (one BF16 ulp flip in an activation moves an output by
    well under that), median relative error below 1e-3."""
    net, w, g = _random_net(11)
    rng = np.random.default_rng(1)
    n = 1000                      # not a multiple of the 128-row tile
    s = G.random_samples(rng, n)
    pos = s[:, 0:3] * 2 - 1
    raw = net.infer(pos, s[:, 4:7], s[:, 8:11])
    p01 = G.normalise(pos, (-1, -1, -1), (1, 1, 1))
    feats, _ = G.encode(g, LOG2T, p01, s[:, 4:7], s[:, 8:11])
    ref, _, _ = G.forward(w, feats)
    ref = ref[:, :G.N_RAW]
    scale = np.abs(ref).max()
    assert np.abs(raw - ref).max() <= 0.02 * scale, np.abs(raw - ref).max() / scale
    rel = np.abs(raw - ref) / np.maximum(np.abs(ref), 1e-3 * scale)
    assert np.median(rel) < 1e-3


@pytest.mark.gpu
def test_gradients_match_oracle():
    """Loss, weight gradients (per layer) and hash-grid gradient of one
    batch against the oracle.  Tolerance: relative Frobenius error 3e-2 per
    layer and for the grid (BF16 operands; a transposed or misplaced operand
    gives errors of order one)."""
    net, w, g = _random_net(21)
    rng = np.random.default_rng(2)
    n = 3000
    s = G.random_samples(rng, n)
    s[:, 0:3] = s[:, 0:3] * 2 - 1
    loss, wg, gg = net.gradients(s)
    rl, rwg, rgg = G.gradients(w, g, LOG2T, s, (-1, -1, -1), (1, 1, 1))
    assert abs(loss - rl) <= 1e-3 * abs(rl), (loss, rl)
    for l in range(4):
        a, b = wg[G.W_OFF[l]:G.W_OFF[l + 1]], rwg[G.W_OFF[l]:G.W_OFF[l + 1]]
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < 3e-2, (l, err)
    err = np.linalg.norm(gg - rgg) / np.linalg.norm(rgg)
    assert err < 3e-2, err


def _target_batch(rng, n):
    """Samples whose incident direction follows a vMF lobe (kappa 20) with a
    position-dependent mean: +z for x < 0.5, (0.6, 0.8, 0) otherwise."""
    s = G.random_samples(rng, n)
    s[:, 3] = 1.0
    mu = np.where(s[:, 0:1] < 0.5, np.array([0.0, 0.0, 1.0]), np.array([0.6, 0.8, 0.0]))
    kappa = 20.0
    u = rng.uniform(size=(n, 2))
    cos = 1 + np.log(u[:, 0] + (1 - u[:, 0]) * np.exp(-2 * kappa)) / kappa
    sin = np.sqrt(np.maximum(0, 1 - cos * cos))
    t = np.where(np.abs(mu[:, 0:1]) > 0.9, np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    bx = np.cross(t, mu)
    bx /= np.linalg.norm(bx, axis=1, keepdims=True)
    by = np.cross(mu, bx)
    phi = 2 * np.pi * u[:, 1]
    s[:, 12:15] = bx * (sin * np.cos(phi))[:, None] + by * (sin * np.sin(phi))[:, None] + mu * cos[:, None]
    return s, mu


@pytest.mark.gpu
def test_training_learns_a_position_dependent_distribution():
    """Online training as the renderer does it (a fresh batch every step) on
    a known target distribution.  On held-out samples the KL loss must fall
    from about log(4 pi) = 2.5 nats to below 0.8 (the optimum, the target's
    entropy, is -0.16), and the learned density at the true mean direction
    must exceed 20x the uniform density 1/(4 pi)."""
    from vlr_b200.guide import GuideNet
    rng = np.random.default_rng(7)
    net = GuideNet(LOG2T, seed=3)
    net.set_bounds((0, 0, 0), (1, 1, 1))
    held, mu = _target_batch(rng, 4096)
    before, _, _ = net.gradients(held)
    losses = []
    for _ in range(200):
        batch, _ = _target_batch(rng, 1 << 14)
        losses.append(net.train(batch, lr=1e-2, steps=1)[0])
    after, _, _ = net.gradients(held)
    assert np.isfinite(losses).all()
    assert before > 1.5, before
    assert after < 0.8, (before, after, losses[-5:])
    raw = net.infer(held[:, 0:3], held[:, 4:7], held[:, 8:11])
    q = G.mixture_pdf(raw.astype(np.float64), mu)
    assert np.median(q) > 20 / (4 * np.pi), np.median(q)
