"""Warm-start network on the GPU (C ABI lddmm_ws_*): the tensor-core GEMM against an
FP32 product of the same BF16 operands, the network's loss, gradient and prediction
against the CPU oracle (oracle/mlp_oracle.py, BF16 rounding at the same points), and
training reducing the loss."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws_mod():
    from lddmm_b200 import warmstart

    return warmstart


# (40000, 256, 256) and (3000, 48, 128): several 128-row tiles per persistent CTA of
# the warp-specialised kernel, both TMEM accumulators and the stage ring wrapping
@pytest.mark.parametrize("m,n,k", [(300, 256, 80), (1000, 32, 256), (64, 16, 16),
                                   (513, 64, 1024), (40000, 256, 256), (3000, 48, 128)])
def test_gemm_bf16_vs_fp32_product(ws_mod, m, n, k):
    import ctypes as C

    from lddmm_b200 import _lib

    g = torch.Generator(device="cpu").manual_seed(m + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16).cuda()
    b = (0.1 * torch.randn(n, k, generator=g)).to(torch.bfloat16).cuda()
    c = torch.full((m, n), float("nan"), dtype=torch.float32, device="cuda")
    _lib.check_ws(_lib.lib.lddmm_ws_gemm_bf16(C.c_void_p(a.data_ptr()), k,
                                              C.c_void_p(b.data_ptr()), k, m, n, k,
                                              C.c_void_p(c.data_ptr()), n, None))
    torch.cuda.synchronize()
    ref = a.double() @ b.double().T
    err = (c.double() - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


def _case(T=3, B=3, N=50, Et=40, seed=0):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(size=(N, 3))
    tri7 = rng.normal(size=(B, Et, 7))
    labels = rng.normal(size=(B, N, 3 * T)) * 0.05
    return xyz, tri7, labels


def _per_layer_rel(g, ref, T):
    out, off = [], 0
    for i, o in M.layer_dims(T):
        for n in (o * i, o):
            a, b = g[off:off + n], ref[off:off + n]
            out.append(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)))
            off += n
    return out


def test_loss_and_gradient_vs_oracle(ws_mod):
    T, scale = 3, 0.05
    xyz, tri7, labels = _case(T)
    params = M.init_params(T, seed=4).astype(np.float32)
    with ws_mod.WarmStart(xyz, T, batch_max=4, tri_max=64, label_scale=scale) as ws:
        ws.params = params
        loss, g = ws.grad(torch.from_numpy(tri7.astype(np.float32)).cuda(),
                          torch.from_numpy(labels.astype(np.float32)).cuda())
    lo, go = M.loss_and_grad(params.astype(np.float64), xyz.astype(np.float32).astype(np.float64),
                             tri7.astype(np.float32).astype(np.float64),
                             labels.astype(np.float32).astype(np.float64), T, scale, bf=True)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    rels = _per_layer_rel(g.astype(np.float64), go, T)
    assert max(rels) < 2e-2, rels
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 5e-3


def test_backward_with_an_outer_gradient_vs_oracle(ws_mod):
    """lddmm_ws_backward after a prediction: the gradient of label_weight * MSE + the
    outer loss sum(dalpha * alpha) against the oracle, with and without labels; the
    weights stay as they are with lr = 0."""
    T, scale = 3, 0.05
    B, N = 3, 50
    xyz, tri7, labels = _case(T)
    params = M.init_params(T, seed=6).astype(np.float32)
    dalpha = np.random.default_rng(3).normal(size=(B, T, N, 3)) * 1e-3
    t = torch.from_numpy(tri7.astype(np.float32)).cuda()
    y = torch.from_numpy(labels.astype(np.float32)).cuda()
    d = torch.from_numpy(dalpha.reshape(B, -1)).cuda()
    args = (params.astype(np.float64), xyz.astype(np.float32).astype(np.float64),
            tri7.astype(np.float32).astype(np.float64))
    with ws_mod.WarmStart(xyz, T, batch_max=4, tri_max=64, label_scale=scale) as ws:
        ws.params = params
        ws.predict(t)
        loss, g = ws.backward(labels=y, label_weight=0.5, dalpha=d, want_grad=True)
        lo, go = M.loss_and_grad(*args, labels.astype(np.float32).astype(np.float64), T, scale,
                                 bf=True, label_weight=0.5, dalpha=dalpha)
        assert abs(loss - lo) <= 1e-4 * abs(lo)
        assert np.linalg.norm(g - go) / np.linalg.norm(go) < 5e-3
        _, g2 = ws.backward(dalpha=d, want_grad=True)
        _, go2 = M.loss_and_grad(*args, None, T, scale, bf=True, dalpha=dalpha)
        assert np.linalg.norm(g2 - go2) / np.linalg.norm(go2) < 5e-3
        assert np.array_equal(ws.params, params)


def test_predict_vs_oracle(ws_mod):
    T, scale = 3, 0.05
    xyz, tri7, _ = _case(T, seed=1)
    params = M.init_params(T, seed=5).astype(np.float32)
    with ws_mod.WarmStart(xyz, T, batch_max=4, tri_max=64, label_scale=scale) as ws:
        ws.params = params
        a = ws.predict(torch.from_numpy(tri7.astype(np.float32)).cuda()).cpu().numpy()
    ref = M.predict(params.astype(np.float64), xyz.astype(np.float32).astype(np.float64),
                    tri7.astype(np.float32).astype(np.float64), T, scale, bf=True)
    ref = ref.reshape(a.shape)
    assert np.max(np.abs(a - ref)) <= 1e-3 * np.max(np.abs(ref))


@pytest.mark.parametrize("local_k", [1, 4, 27])
def test_local_features_vs_oracle(ws_mod, local_k):
    """The network with every landmark's local_k nearest target triangles in its point
    input (lddmm_ws_create_ex): loss, gradient and prediction against the oracle, which
    finds the neighbours with the same FP32 distances and tie rule."""
    T, scale = 3, 0.05
    xyz, tri7, labels = _case(T, seed=3)
    params = M.init_params(T, seed=9, local_k=local_k).astype(np.float32)
    t = torch.from_numpy(tri7.astype(np.float32)).cuda()
    x64 = xyz.astype(np.float32).astype(np.float64)
    t64 = tri7.astype(np.float32).astype(np.float64)
    with ws_mod.WarmStart(xyz, T, batch_max=4, tri_max=64, label_scale=scale,
                          local_k=local_k) as ws:
        assert ws.n_params == M.num_params(T, local_k)
        ws.params = params
        loss, g = ws.grad(t, torch.from_numpy(labels.astype(np.float32)).cuda())
        a = ws.predict(t).cpu().numpy()
    lo, go = M.loss_and_grad(params.astype(np.float64), x64, t64,
                             labels.astype(np.float32).astype(np.float64), T, scale, bf=True,
                             local_k=local_k)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    assert np.linalg.norm(g - go) / np.linalg.norm(go) < 5e-3
    ref = M.predict(params.astype(np.float64), x64, t64, T, scale, bf=True,
                    local_k=local_k).reshape(a.shape)
    assert np.max(np.abs(a - ref)) <= 1e-3 * np.max(np.abs(ref))


def test_cached_neighbours_train_bit_for_bit(ws_mod):
    """lddmm_ws_neighbours finds the oracle's neighbours, and training steps that take
    them (lddmm_ws_train_step_nbr) give the same losses and weights, bit for bit, as
    steps that search themselves."""
    T, scale, k = 3, 0.05, 4
    xyz, tri7, labels = _case(T, seed=5)
    params = M.init_params(T, seed=10, local_k=k).astype(np.float32)
    t = torch.from_numpy(tri7.astype(np.float32)).cuda()
    y = torch.from_numpy(labels.astype(np.float32)).cuda()
    runs = []
    for cached in (False, True):
        with ws_mod.WarmStart(xyz, T, batch_max=4, tri_max=64, label_scale=scale,
                              local_k=k) as ws:
            ws.params = params
            nbr = None
            if cached:
                nbr = ws.neighbours(t)
                ref = M.nearest_triangles(xyz.astype(np.float32), tri7.astype(np.float32), k)
                assert np.array_equal(nbr.cpu().numpy(), ref)
            losses = [ws.train_step(t, y, 1e-3, nbr) for _ in range(3)]
            runs.append((losses, ws.params))
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])


def test_local_features_need_enough_triangles(ws_mod):
    from lddmm_b200 import _lib

    xyz, tri7, _ = _case(3, Et=40)
    with ws_mod.WarmStart(xyz, 3, batch_max=4, tri_max=64, label_scale=0.05, local_k=8) as ws:
        with pytest.raises(_lib.LddmmError):
            ws.predict(torch.from_numpy(tri7[:, :5].astype(np.float32)).contiguous().cuda())


def test_training_reduces_loss(ws_mod):
    """Adam steps on a batch whose labels are a smooth function of the landmark
    positions (learnable from the network's inputs)."""
    T, scale = 3, 0.05
    xyz, tri7, _ = _case(T, B=4, seed=2)
    w = np.random.default_rng(9).normal(size=(3, 3 * T))
    labels = np.broadcast_to(0.05 * np.sin(xyz @ w), (4, xyz.shape[0], 3 * T)).copy()
    t = torch.from_numpy(tri7.astype(np.float32)).cuda()
    y = torch.from_numpy(labels.astype(np.float32)).cuda()
    with ws_mod.WarmStart(xyz, T, batch_max=4, tri_max=64, label_scale=scale, seed=7) as ws:
        first = ws.train_step(t, y, 3e-3)
        for _ in range(200):
            last = ws.train_step(t, y, 3e-3)
        p1 = ws.params
    assert last < 0.2 * first, (first, last)
    assert np.all(np.isfinite(p1))
