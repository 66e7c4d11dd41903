"""The guide oracle (oracle/guide.py) checked against itself: analytic
gradients against finite differences, the vMF mixture normalised and its
sampler matching its pdf. CPU only; these pin the specification the device
kernels are then compared with."""
import numpy as np
import pytest
from scipy import stats

from oracle import guide as G


def _batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    F = rng.uniform(0.1, 2.0, n)
    return x, nrm.astype(np.float32), wo.astype(np.float32), d, F


def test_output_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    o = rng.normal(size=(16, G.OUT))
    x, n, wo, d, F = _batch(16, 1)
    loss, g = G.loss_and_grad_outputs(o, d, F)
    eps = 1e-6
    for idx in [(0, 0), (3, 4), (5, 3), (7, 17), (9, 39), (15, 22)]:
        op = o.copy()
        op[idx] += eps
        om = o.copy()
        om[idx] -= eps
        fd = (G.loss_and_grad_outputs(op, d, F)[0] - G.loss_and_grad_outputs(om, d, F)[0]) / (2 * eps)
        assert abs(fd - g[idx]) < 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])


def test_parameter_gradient_matches_finite_differences():
    p = G.init_params(3).astype(np.float64)
    x, n, wo, d, F = _batch(32, 2)
    X = G.encode(x, n, wo, (-5, -5, -5), (5, 5, 5))

    def loss_of(pp):
        o, _ = G.forward(pp.astype(np.float32), X, emulate_bf16=False)
        return G.loss_and_grad_outputs(o, d, F)[0]

    o, acts = G.forward(p.astype(np.float32), X, emulate_bf16=False)
    _, go = G.loss_and_grad_outputs(o, d, F)
    g = G.backward(p.astype(np.float32), acts, go, emulate_bf16=False)
    rng = np.random.default_rng(4)
    idxs = rng.choice(np.flatnonzero(np.abs(g) > 1e-4), 12, replace=False)
    for i in idxs:
        h = 1e-2 * max(abs(p[i]), 1e-1)
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss_of(pp) - loss_of(pm)) / (2 * h)
        assert abs(fd - g[i]) < 2e-3 + 5e-2 * abs(g[i]), (i, fd, g[i])


def test_mixture_is_normalised_and_sampler_matches_pdf():
    rng = np.random.default_rng(5)
    o = rng.normal(size=(1, G.OUT)) * 2.0
    o[0, 3::5] = rng.uniform(-1, 4, 8)  # kappa up to ~55
    # Integrate the pdf over the sphere (fine (cos, phi) grid).
    nc, nphi = 2400, 4800
    c = -1 + (np.arange(nc) + 0.5) * 2 / nc
    ph = (np.arange(nphi) + 0.5) * 2 * np.pi / nphi
    C, P = np.meshgrid(c, ph, indexing="ij")
    s = np.sqrt(1 - C * C)
    dirs = np.stack([s * np.cos(P), s * np.sin(P), C], -1).reshape(-1, 3)
    pdf = G.mixture_pdf(np.repeat(o, len(dirs), 0), dirs)
    total = pdf.sum() * (2 / nc) * (2 * np.pi / nphi)
    assert abs(total - 1) < 2e-3, total
    # Sampler vs pdf: chi-squared over a coarse (cos, phi) grid.
    n = 200_000
    u = rng.random((n, 3))
    w = G.sample(np.repeat(o, n, 0), u)
    assert np.allclose(np.linalg.norm(w, axis=1), 1, atol=1e-9)
    nt, npb = 24, 48
    bi = np.minimum(((w[:, 2] + 1) / 2 * nt).astype(int), nt - 1)
    bj = np.minimum((np.mod(np.arctan2(w[:, 1], w[:, 0]), 2 * np.pi) / (2 * np.pi) * npb).astype(int), npb - 1)
    obs = np.bincount(bi * npb + bj, minlength=nt * npb)
    exp = pdf.reshape(nc, nphi).reshape(nt, nc // nt, npb, nphi // npb).sum((1, 3)).reshape(-1) * \
        (2 / nc) * (2 * np.pi / nphi) * n
    keep = exp >= 5
    chi = ((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum() + (obs[~keep].sum() - exp[~keep].sum()) ** 2 / max(
        exp[~keep].sum(), 1e-9)
    p = stats.chi2.sf(chi, keep.sum())
    assert p > 1e-3, (p, chi)


def test_training_reduces_the_loss():
    p = G.init_params(7)
    m = np.zeros_like(p, dtype=np.float64)
    v = np.zeros_like(p, dtype=np.float64)
    x, n, wo, _, _ = _batch(512, 8)
    # Radiance arrives from a fixed direction cone around +y: the guide must learn it.
    rng = np.random.default_rng(9)
    d = rng.normal(size=(512, 3)) * 0.2 + np.array([0, 1.0, 0])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    F = np.ones(512)
    X = G.encode(x, n, wo, (-5, -5, -5), (5, 5, 5))
    losses = []
    for t in range(1, 61):
        o, acts = G.forward(p, X)
        loss, go = G.loss_and_grad_outputs(o, d, F)
        losses.append(loss)
        g = G.backward(p, acts, go)
        p, m, v = G.adam(p, g, m, v, t)
    assert losses[-1] < losses[0] - 1.0, losses[::10]
