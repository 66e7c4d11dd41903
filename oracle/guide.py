"""ORACLE — test infrastructure only.

A numpy restatement of the learned path-guiding proposal that the device
kernels implement (no reference counterpart exists in Lucida; this module is
the specification the device is checked against):

  encoding   position normalised to the scene box, 12 frequencies per axis
             (sin, cos of 2^k pi q); normal and outgoing direction, 4 each
             (sin, cos of 2^k pi c); 120 features, zero-padded to 128
  network    128 -> 64 -> ReLU -> 64 -> ReLU -> 64 -> ReLU -> 40; BF16 matmul
             inputs (weights and activations rounded to bfloat16), FP32
             accumulate, FP32 bias
  outputs    8 lobes x (direction xyz, kappa, weight logit):
             mu = normalize(o[0:3]), kappa = min(1 + softplus(o[3]), 1e4),
             w = softmax over the 8 logits
  vMF lobe   p(w) = kappa / (2 pi (1 - exp(-2 kappa))) exp(kappa (mu.w - 1))
  loss       KL(radiance-weighted sample pdf || q): -sum F_i log q(w_i) / sum F_i,
             F_i = incident luminance / sampling pdf
  optimiser  Adam, beta1 0.9, beta2 0.999, eps 1e-8, lr 1e-2

Parameter vector (FP32): W1[64][128], b1[64], W2[64][64], b2[64], W3[64][64],
b3[64], W4[40][64], b4[40].
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT, LOBES = 128, 64, 40, 8
POS_FREQ, DIR_FREQ = 12, 4
KAPPA_MAX = 1.0e4
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("W4", (OUT, HID)), ("b4", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, o = {}, 0
    for name, s in SHAPES:
        n = int(np.prod(s))
        out[name] = p[o:o + n].reshape(s)
        o += n
    return out


def init_params(seed: int) -> np.ndarray:
    """Uniform(+-sqrt(6/(fan_in+fan_out))) weights, zero biases; W1's padding
    columns (features 120..127) are zero. Matches the device initialiser,
    which receives these values through luc_guide_set_params in tests."""
    rng = np.random.default_rng(seed)
    p = []
    for name, s in SHAPES:
        if name.startswith("b"):
            p.append(np.zeros(s, np.float32))
        else:
            lim = np.sqrt(6.0 / (s[0] + s[1]))
            w = rng.uniform(-lim, lim, s).astype(np.float32)
            if name == "W1":
                w[:, 120:] = 0
            p.append(w)
    return np.concatenate([a.reshape(-1) for a in p]).astype(np.float32)


def bf16(x):
    """Round float32 to bfloat16 (nearest, ties to even) and back."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = (u + np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32)


def encode(x, n, wo, lo, hi):
    """Features for points x (N,3), normals n and outgoing directions wo."""
    x, n, wo = (np.asarray(a, np.float32) for a in (x, n, wo))
    lo, hi = np.asarray(lo, np.float32), np.asarray(hi, np.float32)
    ext = np.where(hi > lo, hi - lo, np.float32(1))
    q = np.clip((x - lo) / ext, 0, 1).astype(np.float32)
    feats = []
    for a in range(3):
        for k in range(POS_FREQ):
            f = np.float32(np.pi * 2.0 ** k)
            arg = (q[:, a] * f).astype(np.float32)
            feats += [np.sin(arg), np.cos(arg)]
    for v in (n, wo):
        for a in range(3):
            for k in range(DIR_FREQ):
                f = np.float32(np.pi * 2.0 ** k)
                arg = (v[:, a] * f).astype(np.float32)
                feats += [np.sin(arg), np.cos(arg)]
    X = np.zeros((len(x), IN), np.float32)
    X[:, :120] = np.stack(feats, 1)
    return X


def forward(p, X, emulate_bf16=True):
    """Raw outputs (N, 40) and the hidden activations (for backward)."""
    P = unpack(p)
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    h = r(X)
    acts = [h]
    for i in (1, 2, 3):
        z = h.astype(np.float64) @ r(P[f"W{i}"]).astype(np.float64).T + P[f"b{i}"]
        h = r(np.maximum(z, 0).astype(np.float32))
        acts.append(h)
    o = (h.astype(np.float64) @ r(P["W4"]).astype(np.float64).T + P["b4"]).astype(np.float32)
    return o, acts


def softplus(x):
    return np.where(x > 20, x, np.log1p(np.exp(np.minimum(x, 20))))


def decode(o):
    o = np.asarray(o, np.float64).reshape(-1, LOBES, 5)
    v = o[..., 0:3]
    ln = np.linalg.norm(v, axis=-1, keepdims=True)
    mu = np.where(ln > 0, v / np.maximum(ln, 1e-30), np.array([0, 0, 1.0]))
    kappa = np.minimum(1.0 + softplus(o[..., 3]), KAPPA_MAX)
    lg = o[..., 4]
    e = np.exp(lg - lg.max(-1, keepdims=True))
    w = e / e.sum(-1, keepdims=True)
    return mu, kappa, w


def lobe_pdf(mu, kappa, d):
    """vMF density at unit directions d, per lobe: (..., LOBES)."""
    c = np.einsum("...lk,...k->...l", mu, d)
    norm = kappa / (2 * np.pi * (1 - np.exp(-2 * kappa)))
    return norm * np.exp(kappa * (c - 1))


def mixture_pdf(o, d):
    mu, kappa, w = decode(o)
    return (w * lobe_pdf(mu, kappa, np.asarray(d, np.float64))).sum(-1)


def sample(o, u3):
    """Draw directions: u3[:,0] picks the lobe by weight, u3[:,1:3] sample it."""
    mu, kappa, w = decode(o)
    u3 = np.asarray(u3, np.float64)
    cdf = np.cumsum(w, -1)
    j = np.minimum((u3[:, :1] >= cdf).sum(-1), LOBES - 1)
    m = mu[np.arange(len(j)), j]
    k = kappa[np.arange(len(j)), j]
    W = 1 + np.log(u3[:, 1] + (1 - u3[:, 1]) * np.exp(-2 * k)) / k
    W = np.clip(W, -1, 1)
    phi = 2 * np.pi * u3[:, 2]
    s = np.sqrt(np.maximum(1 - W * W, 0))
    local = np.stack([s * np.cos(phi), s * np.sin(phi), W], -1)
    # Duff et al. frame around m (math.rs:22-30)
    sign = np.copysign(1.0, m[:, 2])
    a = -1 / (sign + m[:, 2])
    b = m[:, 0] * m[:, 1] * a
    t = np.stack([1 + sign * m[:, 0] ** 2 * a, sign * b, -sign * m[:, 0]], -1)
    bb = np.stack([b, sign + m[:, 1] ** 2 * a, -m[:, 1]], -1)
    return t * local[:, :1] + bb * local[:, 1:2] + m * local[:, 2:3]


def loss_and_grad_outputs(o, d, F):
    """Loss -sum F log q(d) / sum F and its gradient w.r.t. the raw outputs (float64)."""
    o = np.asarray(o, np.float64).reshape(-1, LOBES, 5)
    d = np.asarray(d, np.float64)
    F = np.asarray(F, np.float64)
    v = o[..., 0:3]
    ln = np.maximum(np.linalg.norm(v, axis=-1, keepdims=True), 1e-30)
    mu = v / ln
    sp = softplus(o[..., 3])
    kappa_raw = 1.0 + sp
    clamped = kappa_raw >= KAPPA_MAX
    kappa = np.minimum(kappa_raw, KAPPA_MAX)
    lg = o[..., 4]
    e = np.exp(lg - lg.max(-1, keepdims=True))
    w = e / e.sum(-1, keepdims=True)
    c = np.einsum("nlk,nk->nl", mu, d)
    ex = np.exp(-2 * kappa)
    pj = kappa / (2 * np.pi * (1 - ex)) * np.exp(kappa * (c - 1))
    q = np.maximum((w * pj).sum(-1), 1e-30)
    S = F.sum()
    loss = -(F * np.log(q)).sum() / S
    rj = w * pj / q[:, None]
    g = np.zeros_like(o)
    scale = (-F / S)[:, None]
    # d log q / d logit_j = r_j - w_j
    g[..., 4] = scale * (rj - w)
    # d log q / d kappa_j = r_j (1/kappa - 2 e^{-2k}/(1-e^{-2k}) + c - 1); dkappa/do3 = sigmoid(o3)
    dk = rj * (1 / kappa - 2 * ex / (1 - ex) + c - 1)
    sig = 1 / (1 + np.exp(-np.clip(o[..., 3], -60, 60)))
    g[..., 3] = scale * dk * np.where(clamped, 0.0, sig)
    # d log q / d mu_j = r_j kappa_j d; through mu = v/|v|: (I - mu mu^T)/|v|
    gm = (rj * kappa)[..., None] * d[:, None, :]
    gv = (gm - (gm * mu).sum(-1, keepdims=True) * mu) / ln
    g[..., 0:3] = scale[..., None] * gv
    return loss, g.reshape(-1, OUT)


def backward(p, acts, g_out, emulate_bf16=True):
    """Parameter gradient (FP32 vector) for output gradient g_out, following
    the device's rounding: the output gradient and the hidden-layer
    gradients are rounded to bf16 before each matmul, weights are bf16."""
    P = unpack(p)
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    grads = {}
    dy = r(np.asarray(g_out, np.float32))
    grads["b4"] = np.asarray(g_out, np.float64).sum(0)
    for i in (4, 3, 2, 1):
        h = acts[i - 1]
        grads[f"W{i}"] = dy.astype(np.float64).T @ h.astype(np.float64)
        if i == 1:
            break
        dh = dy.astype(np.float64) @ r(P[f"W{i}"]).astype(np.float64)
        dh = np.where(acts[i - 1] > 0, dh, 0.0).astype(np.float32)
        grads[f"b{i - 1}"] = dh.astype(np.float64).sum(0)
        dy = r(dh)
    return np.concatenate([np.asarray(grads[n], np.float64).reshape(-1) for n, _ in SHAPES]).astype(np.float32)


def adam(p, g, m, v, t, lr=1e-2, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return (p - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32), m, v
