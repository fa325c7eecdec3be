"""The warm-start network's CPU oracle: its FP64 gradient against central finite
differences, and its BF16 rounding against torch's."""
import numpy as np
import torch

from oracle import mlp_oracle as M


def _case(T=2, B=2, N=5, Et=6, seed=0):
    rng = np.random.default_rng(seed)
    params = M.init_params(T, seed)
    xyz = rng.normal(size=(N, 3))
    tri7 = rng.normal(size=(B, Et, 7))
    labels = rng.normal(size=(B, N, 3 * T)) * 0.3
    return params, xyz, tri7, labels


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).normal(size=4096).astype(np.float32) * 10.0 ** np.random.default_rng(2).integers(-6, 6, 4096)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.to_bf16(x), ref)


def test_oracle_gradient_finite_differences():
    T, scale = 2, 0.7
    params, xyz, tri7, labels = _case(T)
    loss, g = M.loss_and_grad(params, xyz, tri7, labels, T, scale, bf=False)
    assert g.shape == (M.num_params(T),)
    rng = np.random.default_rng(3)
    # every layer's weights and biases (real entries), a few each
    idx, off = [], 0
    for (i, o), (ir, orr) in zip(M.layer_dims(T), [(7, 64), (64, 64), (67, 256), (256, 256), (256, 3 * T)]):
        for _ in range(6):
            idx.append(off + int(rng.integers(0, orr)) * i + int(rng.integers(0, ir)))
        off += o * i
        for _ in range(2):
            idx.append(off + int(rng.integers(0, orr)))
        off += o
    h = 1e-6
    for k in idx:
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        fd = (M.loss_and_grad(p1, xyz, tri7, labels, T, scale, bf=False)[0]
              - M.loss_and_grad(p2, xyz, tri7, labels, T, scale, bf=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-8, (k, fd, g[k])


def test_padding_gradients_are_zero():
    T = 2
    params, xyz, tri7, labels = _case(T)
    _, g = M.loss_and_grad(params, xyz, tri7, labels, T, 1.0, bf=True)
    off = 0
    for (i, o), (ir, orr) in zip(M.layer_dims(T), [(7, 64), (64, 64), (67, 256), (256, 256), (256, 3 * T)]):
        W = g[off:off + o * i].reshape(o, i)
        assert np.all(W[:, ir:] == 0) and np.all(W[orr:, :] == 0)
        off += o * i
        assert np.all(g[off + orr:off + o] == 0)
        off += o


def test_outer_gradient_term_finite_differences():
    """The gradient of sum(dalpha * alpha(params)) (an outer loss's gradient at the
    prediction, back-propagated through the network) against central differences of
    the oracle's own prediction."""
    T, scale = 2, 0.7
    params, xyz, tri7, _ = _case(T, seed=4)
    B, N = tri7.shape[0], xyz.shape[0]
    dalpha = np.random.default_rng(5).normal(size=(B, T, N, 3))
    _, g = M.loss_and_grad(params, xyz, tri7, None, T, scale, bf=False, dalpha=dalpha)

    def outer(p):
        a = M.predict(p, xyz, tri7, T, scale, bf=False)
        return float(np.sum(a.reshape(dalpha.shape) * dalpha))

    rng = np.random.default_rng(6)
    h = 1e-6
    for k in rng.choice(np.flatnonzero(g != 0), 24, replace=False):
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        fd = (outer(p1) - outer(p2)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-8, (k, fd, g[k])
