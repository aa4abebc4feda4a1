"""Learned guiding network on the tcgen05 tensor cores against the CPU oracle.

The oracle rounds every tensor-core operand to bfloat16 at the points the
device does and sums in float64, so the device differs only by its FP32
summation order (and the occasional bfloat16 rounding flip that follows):
outputs within 1e-3 mean relative error, gradients within 2 % relative L2
error per layer.
"""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu


def _batch(seed, n, concentrated=False):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1, (n, 3))
    nrm = M.sample_sphere(rng, n)
    wo = M.sample_sphere(rng, n)
    t = np.zeros((n, 4), np.float32)
    if concentrated:
        # incident light from a direction that depends on the position
        d = (pos - 0.5) * np.array([1.0, -1.0, 0.5]) + 0.3 * rng.normal(size=(n, 3))
        t[:, :3] = d / np.linalg.norm(d, axis=1, keepdims=True)
    else:
        t[:, :3] = M.sample_sphere(rng, n)
    t[:, 3] = rng.uniform(0.1, 2.0, n)
    t[rng.uniform(size=n) < 0.1, 3] = 0.0   # samples without weight
    return pos, nrm, wo, t


def _params(seed):
    p = M.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    free = ~M.frozen_mask()
    for l, k in enumerate(M.LAYER_IN):     # non-zero biases
        o = M.layer_offset(l) + k * 64
        p[o:o + 64] = rng.normal(0, 0.1, 64)
    p[~free] = 0.0
    return p


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_encode_matches_oracle(system, cuda):
    from meturay_b200.learned import GuideMLP
    pos, nrm, wo, _ = _batch(1, 1000)
    out = cuda.zeros((1000, 80), dtype=cuda.float32, device="cuda")
    GuideMLP.encode(_dev(cuda, pos), _dev(cuda, nrm), _dev(cuda, wo), out)
    cuda.cuda.synchronize()
    ref = M.encode(pos.astype(np.float32), nrm.astype(np.float32), wo.astype(np.float32))
    assert np.abs(out.cpu().numpy() - ref).max() < 2e-6


@pytest.mark.parametrize("n", [1, 128, 1000, 5000])
def test_forward_matches_oracle(system, cuda, n):
    from meturay_b200.learned import GuideMLP
    p = _params(2)
    net = GuideMLP(system, p)
    pos, nrm, wo, _ = _batch(3, n)
    x = M.encode(pos, nrm, wo)
    out = cuda.zeros((n, 40), dtype=cuda.float32, device="cuda")
    net.forward(_dev(cuda, x), out)
    cuda.cuda.synchronize()
    got = out.cpu().numpy()
    ref, _ = M.forward(p, x, quantize=True)
    err = np.abs(got - ref)
    assert err.mean() / np.abs(ref).mean() < 1e-3, err.mean()
    assert err.max() < 0.05 * np.abs(ref).max()


def test_gradients_match_oracle(system, cuda):
    from meturay_b200.learned import GuideMLP, PARAM_COUNT
    p = _params(4)
    net = GuideMLP(system, p)
    n = 3000
    pos, nrm, wo, t = _batch(5, n)
    x = M.encode(pos, nrm, wo)
    grad = cuda.zeros(PARAM_COUNT, dtype=cuda.float32, device="cuda")
    loss = cuda.zeros(4, dtype=cuda.float32, device="cuda")
    net.gradients(_dev(cuda, x), _dev(cuda, t), grad, loss)
    cuda.cuda.synchronize()
    g = grad.cpu().numpy().astype(np.float64)
    ref, lsum, wsum = M.gradients(p, x, t, quantize=True)
    l = loss.cpu().numpy()
    assert abs(l[0] - lsum) < 1e-3 * abs(lsum) and abs(l[1] - wsum) < 1e-4 * wsum
    for layer, k in enumerate(M.LAYER_IN):
        o = M.layer_offset(layer)
        for name, sl in (("W", slice(o, o + k * 64)), ("b", slice(o + k * 64, o + k * 64 + 64))):
            rel = np.linalg.norm(g[sl] - ref[sl]) / max(np.linalg.norm(ref[sl]), 1e-12)
            assert rel < 2e-2, (layer, name, rel)
    o = M.layer_offset(3)
    assert np.all(g[o:o + 64 * 64].reshape(64, 64)[:, 40:] == 0)


def test_training_lowers_the_loss_and_keeps_padding_zero(system, cuda):
    from meturay_b200.learned import GuideMLP
    net = GuideMLP(system, M.init_params(6))
    n = 8192
    pos, nrm, wo, t = _batch(7, n, concentrated=True)
    x, tt = _dev(cuda, M.encode(pos, nrm, wo)), _dev(cuda, t)
    losses = []
    for _ in range(150):
        ls, ws = net.train_step(x, tt, lr=1e-2)
        losses.append(ls / ws)
    # -log q of a uniform density is log(4 pi) = 2.53; the trained mixture
    # concentrates on the position-dependent incident direction
    assert losses[0] > 2.0 and losses[-1] < losses[0] - 1.0, (losses[0], losses[-1])
    p = net.params()
    assert np.all(p[M.frozen_mask()] == 0)
    # one optimiser step matches the oracle's from the same state
    net2 = GuideMLP(system, _params(8))
    net2.train_step(x[:2048], tt[:2048], lr=1e-2)
    p0 = _params(8).astype(np.float64)
    g, _, wsum = M.gradients(_params(8), M.encode(pos, nrm, wo)[:2048], t[:2048], quantize=True)
    p1, _, _ = M.adam(p0, np.zeros_like(p0), np.zeros_like(p0), 0, g, wsum)
    d = net2.params() - p1
    # Adam's first step is lr * sign(g) wherever |g| dominates eps
    big = np.abs(g / wsum) > 1e-4
    assert np.mean(np.abs(d[big]) < 1e-4) > 0.97
