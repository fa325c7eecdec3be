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


def test_local_features_gradient_finite_differences():
    """With local target features (local_k = 3) the oracle's FP64 gradient against
    central differences; the features are inputs, so only the weights move."""
    T, scale, k = 2, 0.7, 3
    _, xyz, tri7, labels = _case(T, seed=7)
    params = M.init_params(T, seed=8, local_k=k)
    assert params.shape == (M.num_params(T, k),)
    _, g = M.loss_and_grad(params, xyz, tri7, labels, T, scale, bf=False, local_k=k)
    rng = np.random.default_rng(9)
    h = 1e-6
    for idx in rng.choice(np.flatnonzero(g != 0), 24, replace=False):
        p1, p2 = params.copy(), params.copy()
        p1[idx] += h
        p2[idx] -= h
        fd = (M.loss_and_grad(p1, xyz, tri7, labels, T, scale, bf=False, local_k=k)[0]
              - M.loss_and_grad(p2, xyz, tri7, labels, T, scale, bf=False, local_k=k)[0]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 * max(1.0, abs(g[idx])) + 1e-8, (idx, fd, g[idx])


def test_nearest_triangles_order_and_ties():
    """Nearest first by FP32 squared distance, equal distances to the lower index."""
    xyz = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    cen = np.array([[2.0, 0, 0], [0, 1.0, 0], [0, -1.0, 0], [0.5, 0, 0], [3.0, 0, 0]])
    tri7 = np.zeros((1, 5, 7))
    tri7[0, :, :3] = cen
    nb = M.nearest_triangles(xyz, tri7, 4)
    assert nb[0, 0].tolist() == [3, 1, 2, 0]      # 0.25, then the tie 1 = 1 (1 before 2)
    assert nb[0, 1].tolist() == [3, 0, 1, 2]      # 0.25, 1, then the tie 2 = 2
    rng = np.random.default_rng(3)
    q, t = rng.normal(size=(20, 3)), rng.normal(size=(2, 30, 7))
    nb = M.nearest_triangles(q, t, 5)
    d = ((t[:, None, :, :3] - q[None, :, None, :]) ** 2).sum(-1)
    assert np.array_equal(nb, np.argsort(d, axis=2)[:, :, :5])
