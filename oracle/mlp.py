"""CPU oracle of the learned guiding network -- TEST INFRASTRUCTURE ONLY.

Restates meturay_b200's MLP (no counterpart in the MRay reference): the
80-feature vertex encoding, the 80 -> 64 -> 64 -> 64 -> 40 ReLU network, the
mixture of 8 von Mises-Fisher lobes with its weighted negative
log-likelihood and gradient, the backward pass and Adam.  With
quantize=True every operand the device hands to its tensor cores is rounded
to bfloat16 at the same points (inputs, weights, hidden activations, output
and hidden gradients), products are exact and sums are taken in float64,
so the device agrees up to its FP32 summation order; with quantize=False it
is the float64 network used for the finite-difference check.
"""
from __future__ import annotations

import math

import numpy as np

N_IN, N_FEAT, WIDTH, N_OUT, LOBES = 80, 78, 64, 40, 8
LAYER_IN = (80, 64, 64, 64)
LOG_KAPPA_MAX = 8.0


def layer_offset(l: int) -> int:
    return 0 if l == 0 else (80 * 64 + 64) + (l - 1) * (64 * 64 + 64)


N_PARAMS = (80 * 64 + 64) + 3 * (64 * 64 + 64)


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest even) -> float32."""
    a = np.ascontiguousarray(x, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


def frozen_mask() -> np.ndarray:
    """Parameters held at zero: output columns 40..63, input rows 78..79."""
    m = np.zeros(N_PARAMS, bool)
    o = layer_offset(0)
    m[o + 78 * 64:o + 80 * 64] = True
    o = layer_offset(3)
    w = m[o:o + 64 * 64].reshape(64, 64)
    w[:, 40:] = True
    m[o + 64 * 64 + 40:o + 64 * 64 + 64] = True
    return m


def init_params(seed: int) -> np.ndarray:
    """He-uniform weights, zero biases, frozen entries zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    for l, k in enumerate(LAYER_IN):
        lim = math.sqrt(6.0 / k) if l < 3 else math.sqrt(3.0 / k)
        o = layer_offset(l)
        p[o:o + k * 64] = rng.uniform(-lim, lim, k * 64)
    p[frozen_mask()] = 0.0
    return p


def unpack(p: np.ndarray):
    out = []
    for l, k in enumerate(LAYER_IN):
        o = layer_offset(l)
        out.append((p[o:o + k * 64].reshape(k, 64), p[o + k * 64:o + k * 64 + 64]))
    return out


def encode(pos: np.ndarray, nrm: np.ndarray, wo: np.ndarray) -> np.ndarray:
    """sin / cos of 2^j pi p (j < 12) per axis at 24c + 2j (+1), the normal,
    the outgoing direction, two zeros."""
    pos = np.asarray(pos, np.float64)
    n = pos.shape[0]
    f = np.zeros((n, N_IN), np.float64)
    for c in range(3):
        for j in range(12):
            a = math.pi * (2.0 ** j) * pos[:, c]
            f[:, 24 * c + 2 * j] = np.sin(a)
            f[:, 24 * c + 2 * j + 1] = np.cos(a)
    f[:, 72:75] = nrm
    f[:, 75:78] = wo
    return f.astype(np.float32)


def forward(p: np.ndarray, x: np.ndarray, quantize: bool = True):
    """Returns (raw outputs n x 40, cache for backward)."""
    q = bf16 if quantize else (lambda v: np.asarray(v, np.float64))
    layers = unpack(np.asarray(p, np.float64) if not quantize else p)
    a = q(x).astype(np.float64)
    acts = [a]
    z = None
    for l, (w, b) in enumerate(layers):
        z = a @ q(w).astype(np.float64) + np.asarray(b, np.float64)
        if quantize:
            z = z.astype(np.float32).astype(np.float64)
        if l < 3:
            a = q(np.maximum(z, 0.0)).astype(np.float64)
            acts.append(a)
    return z[:, :N_OUT], acts


def mixture(raw: np.ndarray):
    """Per sample: mu (n,8,3), kappa (n,8), log normaliser, log pi, |raw dir|."""
    r = np.asarray(raw, np.float64).reshape(-1, LOBES, 5)
    d = r[..., 0:3]
    nn = np.sqrt((d * d).sum(-1) + 1e-12)
    mu = d / nn[..., None]
    lk = np.clip(r[..., 3], -10.0, LOG_KAPPA_MAX)
    kap = np.exp(lk)
    lognorm = lk - math.log(2.0 * math.pi) - np.log(-np.expm1(-2.0 * kap))
    logit = r[..., 4]
    lse = logit.max(-1, keepdims=True)
    lse = lse + np.log(np.exp(logit - lse).sum(-1, keepdims=True))
    return mu, kap, lognorm, logit - lse, nn


def log_pdf(raw: np.ndarray, dirs: np.ndarray):
    mu, kap, lognorm, logpi, _ = mixture(raw)
    c = (mu * np.asarray(dirs, np.float64)[:, None, :]).sum(-1)
    lobe = logpi + lognorm + kap * (c - 1.0)
    m = lobe.max(-1, keepdims=True)
    return (m + np.log(np.exp(lobe - m).sum(-1, keepdims=True)))[:, 0], lobe


def mixture_grad(raw: np.ndarray, dirs: np.ndarray, w: np.ndarray):
    """(-log q per sample, d(sum w * -log q)/d raw  n x 40)."""
    r = np.asarray(raw, np.float64).reshape(-1, LOBES, 5)
    mu, kap, _, logpi, nn = mixture(raw)
    lq, lobe = log_pdf(raw, dirs)
    d = np.asarray(dirs, np.float64)[:, None, :]
    w = np.asarray(w, np.float64)[:, None]
    gamma = np.exp(lobe - lq[:, None])
    pi = np.exp(logpi)
    c = (mu * d).sum(-1)
    g = np.zeros_like(r)
    sd = -w * gamma * kap / nn
    g[..., 0:3] = sd[..., None] * (d - c[..., None] * mu)
    dlog = 1.0 / kap - 2.0 / np.expm1(2.0 * kap) + (c - 1.0)
    inside = (r[..., 3] > -10.0) & (r[..., 3] < LOG_KAPPA_MAX)
    g[..., 3] = np.where(inside, -w * gamma * dlog * kap, 0.0)
    g[..., 4] = -w * (gamma - pi)
    return -lq, g.reshape(-1, N_OUT)


def gradients(p: np.ndarray, x: np.ndarray, targets: np.ndarray, quantize: bool = True):
    """(param gradient of sum_s w_s -log q, loss sum, weight sum)."""
    t = np.asarray(targets, np.float64)
    raw, acts = forward(p, x, quantize)
    w = np.where(t[:, 3] > 0, t[:, 3], 0.0)
    nlq, g = mixture_grad(raw, t[:, :3], w)
    q = bf16 if quantize else (lambda v: np.asarray(v, np.float64))
    layers = unpack(np.asarray(p, np.float64) if not quantize else p)
    grad = np.zeros(N_PARAMS, np.float64)
    G = np.zeros((x.shape[0], 64))
    G[:, :N_OUT] = g
    G = q(G.astype(np.float32) if quantize else G).astype(np.float64)
    for l in range(3, -1, -1):
        o, k = layer_offset(l), LAYER_IN[l]
        grad[o:o + k * 64] = (acts[l].T @ G).ravel()
        grad[o + k * 64:o + k * 64 + 64] = G.sum(0)
        if l > 0:
            dx = G @ q(layers[l][0]).astype(np.float64).T
            if quantize:
                dx = dx.astype(np.float32).astype(np.float64)
            dx = np.where(acts[l] > 0, dx, 0.0)
            G = q(dx.astype(np.float32) if quantize else dx).astype(np.float64)
    mask = w > 0
    return grad, float((w * nlq)[mask].sum()), float(w.sum())


def adam(p, m1, m2, t, grad, wsum, lr=1e-2, b1=0.9, b2=0.999, eps=1e-8):
    """One step (t: steps taken before); returns new (p, m1, m2)."""
    g = grad / max(wsum, 1e-20)
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** (t + 1), 1 - b2 ** (t + 1)
    upd = lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps)
    fz = frozen_mask()
    p = np.where(fz, p, p - upd)
    return p, np.where(fz, 0.0, m1), np.where(fz, 0.0, m2)


def sample_sphere(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)
