"""CPU oracle of the warm-start network (test infrastructure only).

A numpy restatement of the network and its gradient with the parameter layout of the
library's flat vector (per layer Wt[out][in] then b[out]; layers: target 1 (16 -> 64),
target 2 (64 -> 64), point 1 (80 -> 256), point 2 (256 -> 256), point 3
(256 -> round16(3T))), evaluated in FP64.  With ``bf=True`` it rounds to BF16 (round
to nearest even) at the points where the CUDA path stores BF16: every GEMM operand
(inputs, activations, weights, loss gradients), so the two agree up to FP32
accumulation order; with ``bf=False`` it is the exact FP64 network whose gradient the
finite-difference test checks.  There is no reference implementation of this part.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

TRI_IN, TRI_H, PT_IN, PT_H = 16, 64, 80, 256
LOCAL_REL = np.float32(10.0)  # scale of a neighbour's centre offset


def round16(n: int) -> int:
    return (n + 15) // 16 * 16


def pt_in(local_k: int = 0) -> int:
    """Width of the point input: q, the pooled target features, 7 per neighbour."""
    return round16(3 + TRI_H + 7 * local_k)


def layer_dims(T: int, local_k: int = 0):
    """(in, out) of the five layers, padded."""
    return [(TRI_IN, TRI_H), (TRI_H, TRI_H), (pt_in(local_k), PT_H), (PT_H, PT_H),
            (PT_H, round16(3 * T))]


def num_params(T: int, local_k: int = 0) -> int:
    return sum(o * i + o for i, o in layer_dims(T, local_k))


def nearest_triangles(xyz, tri7, k):
    """(B, N, k) indices of every landmark's k nearest target triangle centres, as the
    library's knn_kernel: squared distance in FP32, ((dx dx + dy dy) + dz dz) with each
    operation rounded, ascending, ties to the lower index."""
    q = np.asarray(xyz, dtype=np.float32)
    c = np.asarray(tri7, dtype=np.float32)[:, :, :3]
    d = c[:, None, :, :] - q[None, :, None, :]          # (B, N, Et, 3) FP32
    d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    return np.argsort(d2, axis=2, kind="stable")[:, :, :k]


def point_inputs(xyz, tri7, g, local_k=0):
    """(B, N, pt_in) point inputs before BF16 rounding: q, g, then per neighbour
    (c - q) * 10, the unit normal and area * Et / (4 pi), computed in FP32."""
    B, N = tri7.shape[0], xyz.shape[0]
    xp = np.zeros((B, N, pt_in(local_k)))
    xp[:, :, :3] = xyz[None]
    xp[:, :, 3:3 + TRI_H] = g[:, None, :]
    if local_k:
        nb = nearest_triangles(xyz, tri7, local_k)
        t = np.asarray(tri7, dtype=np.float32)[np.arange(B)[:, None, None], nb]  # B,N,k,7
        f = t.copy()
        f[..., :3] = (t[..., :3] - np.asarray(xyz, dtype=np.float32)[None, :, None, :]) * LOCAL_REL
        xp[:, :, 3 + TRI_H:3 + TRI_H + 7 * local_k] = f.reshape(B, N, 7 * local_k)
    return xp


def unpack(params, T, local_k=0):
    out, off = [], 0
    for i, o in layer_dims(T, local_k):
        Wt = params[off:off + o * i].reshape(o, i)
        off += o * i
        b = params[off:off + o]
        off += o
        out.append((Wt, b))
    return out


def to_bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def loss_and_grad(params, xyz, tri7, labels, T, label_scale, bf=True, label_weight=1.0,
                  dalpha=None, local_k=0):
    """Mean squared error of a batch and the gradient (flat, the library's layout) of
    label_weight * MSE + sum(dalpha * alpha), alpha = label_scale * y the predicted
    momenta.

    xyz (N, 3) source landmarks; tri7 (B, Et, 7) target features; labels (B, N, 3T) or
    None (no MSE term); dalpha (B, T, N, 3) or None."""
    r = to_bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    params = np.asarray(params, dtype=np.float64)
    L = unpack(params, T, local_k)
    B, Et, _ = tri7.shape
    N = xyz.shape[0]
    n_out = 3 * T
    # target branch
    xt = np.zeros((B, Et, TRI_IN))
    xt[:, :, :7] = tri7
    xt = r(xt)
    (W1, b1), (W2, b2), (P1, c1), (P2, c2), (P3, c3) = L
    pre_t = xt @ r(W1).T + b1
    h1 = r(gelu(pre_t))
    h2 = h1 @ r(W2).T + b2
    arg = np.argmax(h2, axis=1)                     # (B, 64): first maximum
    g = np.take_along_axis(h2, arg[:, None, :], axis=1)[:, 0, :]
    # point branch
    xp = r(point_inputs(xyz, tri7, g, local_k))
    pre1 = xp @ r(P1).T + c1
    a1 = r(gelu(pre1))
    pre2 = a1 @ r(P2).T + c2
    a2 = r(gelu(pre2))
    y = a2 @ r(P3).T + c3
    count = B * N * n_out
    dy = np.zeros_like(y)
    loss = 0.0
    if labels is not None:
        e = y[:, :, :n_out] - labels / label_scale
        loss = float(np.sum(e * e) / count)
        dy[:, :, :n_out] = label_weight * 2.0 * e / count
    if dalpha is not None:
        dy[:, :, :n_out] += label_scale * np.asarray(dalpha).transpose(0, 2, 1, 3).reshape(
            B, N, n_out)
    dy = r(dy)
    grads = []
    dP3 = np.einsum("bno,bni->oi", dy, a2)
    dc3 = dy.sum(axis=(0, 1))
    da2 = r((dy @ r(P3)) * gelu_grad(pre2))
    dP2 = np.einsum("bno,bni->oi", da2, a1)
    dc2 = da2.sum(axis=(0, 1))
    da1 = r((da2 @ r(P2)) * gelu_grad(pre1))
    dP1 = np.einsum("bno,bni->oi", da1, xp)
    dc1 = da1.sum(axis=(0, 1))
    dg = da1.sum(axis=1) @ P1[:, 3:3 + TRI_H]       # FP32 master weights, as on the GPU
    dh2 = np.zeros((B, Et, TRI_H))
    bi = np.arange(B)[:, None]
    ci = np.arange(TRI_H)[None, :]
    dh2[bi, arg, ci] = dg
    dh2 = r(dh2)
    dW2 = np.einsum("bno,bni->oi", dh2, h1)
    db2 = dh2.sum(axis=(0, 1))
    dh1 = r((dh2 @ r(W2)) * gelu_grad(pre_t))
    dW1 = np.einsum("bno,bni->oi", dh1, xt)
    db1 = dh1.sum(axis=(0, 1))
    for dW, db in ((dW1, db1), (dW2, db2), (dP1, dc1), (dP2, dc2), (dP3, dc3)):
        grads += [dW.ravel(), db.ravel()]
    return loss, np.concatenate(grads)


def init_params(T, seed=0, local_k=0):
    """Random parameters in the library's layout (real entries only, padding zero)."""
    rng = np.random.default_rng(seed)
    real = [(7, TRI_H), (TRI_H, TRI_H), (3 + TRI_H + 7 * local_k, PT_H), (PT_H, PT_H),
            (PT_H, 3 * T)]
    out = []
    for (i, o), (ir, orr) in zip(layer_dims(T, local_k), real):
        W = np.zeros((o, i))
        W[:orr, :ir] = rng.uniform(-1, 1, size=(orr, ir)) / np.sqrt(ir)
        b = np.zeros(o)
        b[:orr] = rng.uniform(-1, 1, size=orr) / np.sqrt(ir)
        out += [W.ravel(), b]
    return np.concatenate(out)


def predict(params, xyz, tri7, T, label_scale, bf=True, local_k=0):
    """Predicted momenta, (B, T, N, 3): the library's lddmm_ws_predict in FP64."""
    r = to_bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    L = unpack(np.asarray(params, dtype=np.float64), T, local_k)
    B, Et, _ = tri7.shape
    N = xyz.shape[0]
    (W1, b1), (W2, b2), (P1, c1), (P2, c2), (P3, c3) = L
    xt = np.zeros((B, Et, TRI_IN))
    xt[:, :, :7] = tri7
    h1 = r(gelu(r(xt) @ r(W1).T + b1))
    g = (h1 @ r(W2).T + b2).max(axis=1)
    xp = point_inputs(xyz, tri7, g, local_k)
    a1 = r(gelu(r(xp) @ r(P1).T + c1))
    a2 = r(gelu(a1 @ r(P2).T + c2))
    y = (a2 @ r(P3).T + c3)[:, :, :3 * T] * label_scale
    return y.reshape(B, N, T, 3).transpose(0, 2, 1, 3)
