"""The learned-guiding network's CPU oracle checked against itself: analytic
gradients against central finite differences (float64 network), the vMF
mixture integrating to one, bfloat16 rounding, the encoding's definition."""
import math

import numpy as np
import pytest

from oracle import mlp as M


def _batch(seed, n):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1, (n, 3))
    nrm = M.sample_sphere(rng, n)
    wo = M.sample_sphere(rng, n)
    x = M.encode(pos, nrm, wo)
    t = np.zeros((n, 4))
    t[:, :3] = M.sample_sphere(rng, n)
    t[:, 3] = rng.uniform(0.1, 2.0, n)
    return x, t


def test_gradients_match_finite_differences():
    p = M.init_params(3).astype(np.float64) * 0.5
    p[~M.frozen_mask()] += np.random.default_rng(4).normal(0, 0.02, (~M.frozen_mask()).sum())
    x, t = _batch(5, 12)

    def loss(q):
        return M.gradients(q, x, t, quantize=False)[1]

    grad, _, _ = M.gradients(p, x, t, quantize=False)
    rng = np.random.default_rng(6)
    idx = rng.choice(np.nonzero(~M.frozen_mask())[0], 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (loss(p + e) - loss(p - e)) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])
    # the output layer's padded columns get no gradient
    o = M.layer_offset(3)
    assert np.all(grad[o:o + 64 * 64].reshape(64, 64)[:, 40:] == 0)


def test_mixture_integrates_to_one():
    rng = np.random.default_rng(7)
    raw = rng.normal(0, 1, (3, 40))
    raw[:, 3::5] = rng.uniform(-3, 4, (3, 8))   # concentrations e^-3 .. e^4
    # Fibonacci sphere quadrature
    n = 200_000
    k = np.arange(n) + 0.5
    z = 1 - 2 * k / n
    phi = math.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    for j in range(3):
        lq, _ = M.log_pdf(np.repeat(raw[j:j + 1], n, 0), d)
        assert abs(np.exp(lq).mean() * 4 * math.pi - 1.0) < 2e-3


def test_bf16_rounding():
    assert M.bf16(np.array([-2.5, 0.0, 3.0], np.float32)).tolist() == [-2.5, 0.0, 3.0]
    # ties to even: 1 + 2^-8 is exactly half way between 1 and 1 + 2^-7
    assert M.bf16(np.float32(1.0 + 2 ** -8)) == np.float32(1.0)
    assert M.bf16(np.float32(1.0 + 3 * 2 ** -8)) == np.float32(1.0 + 2 ** -6)
    assert M.bf16(np.float32(1.0 + 2 ** -8 + 2 ** -12)) == np.float32(1.0 + 2 ** -7)


def test_encoding_definition():
    pos = np.array([[0.25, 0.5, 0.125]])
    f = M.encode(pos, np.array([[0, 0, 1.0]]), np.array([[1.0, 0, 0]]))
    assert f.shape == (1, 80) and f[0, 78] == 0 and f[0, 79] == 0
    assert f[0, 0] == pytest.approx(math.sin(math.pi * 0.25), abs=1e-7)
    assert f[0, 24 + 2 * 3 + 1] == pytest.approx(math.cos(math.pi * 8 * 0.5), abs=1e-7)
    assert f[0, 72:78].tolist() == [0, 0, 1, 1, 0, 0]


def test_adam_keeps_frozen_parameters_zero():
    p = M.init_params(1).astype(np.float64)
    g = np.random.default_rng(2).normal(0, 1, M.N_PARAMS)
    p2, m1, m2 = M.adam(p, np.zeros_like(p), np.zeros_like(p), 0, g, 10.0)
    assert np.all(p2[M.frozen_mask()] == 0) and np.all(m1[M.frozen_mask()] == 0)
    # the first Adam step moves every free parameter by lr against its gradient sign
    free = ~M.frozen_mask()
    assert np.allclose((p - p2)[free], 1e-2 * np.sign(g[free]), rtol=0, atol=2e-4)
