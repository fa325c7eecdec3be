"""Learned warm start for L-BFGS (host side).  No counterpart in the reference.

A small network (csrc/warmstart.cu, C ABI ``lddmm_ws_*``) predicts a registration's
initial momenta from the source landmarks and the target's varifold; the plain
method then runs from that start as usual and judges the result.  This module holds:

* the workload of the learned part: a 2562-landmark icosphere onto perturbed spheres
  r = 1 + sum_{l<=6} c_lm Y_lm, c_lm ~ N(0, 0.08^2), 5120 triangles; Gaussian
  deformation kernel 0.3, varifold Gaussian 0.1 x Binet, T = 10 steps, varifold
  weight 10 (with weight 1 a registration lowers the objective by only ~20 % and a
  warm start has nothing to gain);
* ``generate``: the training labels, momenta of plain-method registrations run in
  batches on the device;
* ``WarmStart``: the network (training steps, prediction, parameters, gradient);
* ``train`` and ``evaluate`` (cold start from zero vs warm start from the prediction:
  iterations and evaluations until the objective is within 1e-5 of the cold start's
  converged objective, and batch wall time to convergence).

Device memory is held in torch tensors; all arithmetic is in the library.
"""
from __future__ import annotations

import ctypes as C
import functools
import math
import time

import numpy as np

from . import _lib, api, problem, shapes
from ._lib import check, check_ws, lib

T_STEPS = 10           # time steps of the learned workload (3T = 30 outputs per landmark)


def pair(seed: int, src_subdiv: int = 4, tgt_subdiv: int = 4, lmax: int = 6,
         sigma: float = 0.08, time_num: int = T_STEPS + 1,
         dis_wgt: float = 10.0) -> problem.Problem:
    """Icosphere source (2562 landmarks at subdivision 4) onto a perturbed sphere
    (5120 triangles at subdivision 4) drawn with `seed`."""
    V, F, ifo = _source(src_subdiv)
    tv, tf = shapes.star_surface(tgt_subdiv, lmax, sigma, seed)
    cen, dr, vol = shapes.varifold_of(tv, tf)
    T = time_num - 1
    return problem.Problem(V, F, cen, dr, vol, elm_ifo=ifo, knl_order=-1, knl_width=0.3,
                           time_num=time_num,
                           time_stp=1.0 / T, cen_type="G", cen_width=0.1, dir_type="B",
                           dis_wgt=dis_wgt, name=f"warm{seed}")


@functools.lru_cache(maxsize=None)
def _source(subdiv):
    V, F = shapes.icosphere(subdiv)
    return V, F, problem.elm_ifo(F, V.shape[0])


def features(P: problem.Problem) -> np.ndarray:
    """Target features per triangle: centre, unit normal, area * Et / (4 pi)."""
    Et = P.tgt_elm_num
    f = np.empty((Et, 7), dtype=np.float32)
    f[:, 0:3] = P.tgt_cen
    f[:, 3:6] = P.tgt_dir
    f[:, 6] = P.tgt_vol * Et / (4.0 * math.pi)
    return f


def _labels(alpha, n_pairs, T, N):
    """(pairs, T * N * 3) momenta in the variable layout -> (pairs, N, 3T) labels."""
    return alpha.view(n_pairs, T, N, 3).permute(0, 2, 1, 3).reshape(n_pairs, N, 3 * T)


def register_batch(probs, alp0=None, itr_max=300, tol=1e-12, rel_obj_tol=1e-6, mem_num=5,
                   trace=False):
    """L-BFGS of a batch of pairs in one context, device-resident.  Returns (alpha as a
    (pairs, var) torch float64 tensor, per-pair results, seconds, traces or None)."""
    import torch

    with api.Context(probs) as ctx:
        n = len(probs)
        d = torch.zeros(ctx.var_total, dtype=torch.float64, device="cuda")
        if alp0 is not None:
            d.copy_(alp0.reshape(-1))
        opt = _lib.Opt(itr_max, tol, 1e-4, 0.9, mem_num, 0, rel_obj_tol)
        res = (_lib.Result * n)()
        torch.cuda.synchronize()
        t = time.perf_counter()
        check(lib.lddmm_lbfgs_device(ctx.handle, C.byref(opt), C.c_void_p(d.data_ptr()), res))
        sec = time.perf_counter() - t
        out = [dict(f=r.fcn, status=r.status, iters=r.iters, evals=r.evals) for r in res]
        traces = [ctx.trace(p) for p in range(n)] if trace else None
    return d.view(n, -1), out, sec, traces


def generate(seeds, batch=64, itr_max=300, rel_obj_tol=1e-6, log=None, make=pair):
    """Training data: plain-method registrations of make(seed) for every seed, run
    `batch` pairs per context.  Returns (tri7 (n, Et, 7) float32, labels (n, N, 3T)
    float32, source landmarks (N, 3), per-pair results) with tensors on the device."""
    import torch

    tri, lab, results = [], [], []
    src = None
    for k in range(0, len(seeds), batch):
        probs = [make(s) for s in seeds[k:k + batch]]
        src = probs[0].ini_nde
        alpha, res, sec, _ = register_batch(probs, itr_max=itr_max, rel_obj_tol=rel_obj_tol)
        T, N = probs[0].T, probs[0].nde_num
        lab.append(_labels(alpha, len(probs), T, N).float())
        tri.append(torch.from_numpy(np.stack([features(P) for P in probs])).cuda())
        results += res
        if log:
            log(f"generated {k + len(probs)}/{len(seeds)} pairs ({sec:.1f} s for {len(probs)}, "
                f"median iterations {np.median([r['iters'] for r in res]):.0f})")
    return torch.cat(tri), torch.cat(lab), src, results


class WarmStart:
    """The network (C ABI lddmm_ws_*): one source shape, T steps, batches of up to
    `batch_max` pairs with up to `tri_max` target triangles; `local_k` > 0 adds every
    landmark's local_k nearest target triangles to its point input
    (lddmm_ws_create_ex)."""

    def __init__(self, src_nde, T, batch_max, tri_max, label_scale, seed=0, stream=None,
                 local_k=0):
        src = np.ascontiguousarray(src_nde, dtype=np.float64)
        self.N, self.T, self.local_k = src.shape[0], T, local_k
        h = C.c_void_p()
        check_ws(lib.lddmm_ws_create_ex(self.N, _lib.dptr(src), T, batch_max, tri_max,
                                        label_scale, seed, local_k, stream, C.byref(h)))
        self._h = h
        self.n_params = lib.lddmm_ws_num_params(h)

    def close(self):
        if self._h:
            lib.lddmm_ws_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        check_ws(lib.lddmm_ws_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), 0))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        check_ws(lib.lddmm_ws_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), 1))

    def grad(self, tri7, labels):
        """(loss, flat gradient) of a batch (device tensors) without an update."""
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_double()
        check_ws(lib.lddmm_ws_grad(self._h, C.c_void_p(tri7.data_ptr()), tri7.shape[0],
                                   tri7.shape[1], C.c_void_p(labels.data_ptr()),
                                   g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return loss.value, g

    def train_step(self, tri7, labels, lr=1e-3, nbr=None):
        """One Adam step; nbr: the batch's neighbours from neighbours() (networks with
        local features: spares the search, same result)."""
        loss = C.c_double()
        if nbr is None:
            check_ws(lib.lddmm_ws_train_step(self._h, C.c_void_p(tri7.data_ptr()),
                                             tri7.shape[0], tri7.shape[1],
                                             C.c_void_p(labels.data_ptr()), lr,
                                             C.byref(loss)))
        else:
            check_ws(lib.lddmm_ws_train_step_nbr(self._h, C.c_void_p(tri7.data_ptr()),
                                                 tri7.shape[0], tri7.shape[1],
                                                 C.c_void_p(labels.data_ptr()),
                                                 C.c_void_p(nbr.data_ptr()), lr,
                                                 C.byref(loss)))
        return loss.value

    def neighbours(self, tri7, batch=64):
        """(pairs, N, local_k) int32 device tensor: every landmark's nearest target
        triangles, searched in chunks of `batch` pairs."""
        import torch

        out = torch.empty((tri7.shape[0], self.N, self.local_k), dtype=torch.int32,
                          device="cuda")
        for k in range(0, tri7.shape[0], batch):
            t = tri7[k:k + batch].contiguous()
            check_ws(lib.lddmm_ws_neighbours(self._h, C.c_void_p(t.data_ptr()), t.shape[0],
                                             t.shape[1], C.c_void_p(out[k:k + batch].data_ptr())))
        return out

    def backward(self, labels=None, label_weight=1.0, dalpha=None, lr=0.0, want_grad=False):
        """Backward pass of the last predict()'s batch for the loss
        label_weight * MSE(labels) + sum(dalpha * alpha) (dalpha: (pairs, T * N * 3)
        float64 on the device, the outer loss's gradient at the prediction); one Adam step
        when lr > 0.  Returns (the MSE term, the gradient when want_grad else None)."""
        g = np.zeros(self.n_params, dtype=np.float32) if want_grad else None
        loss = C.c_double()
        check_ws(lib.lddmm_ws_backward(
            self._h, C.c_void_p(labels.data_ptr()) if labels is not None else None,
            label_weight, C.c_void_p(dalpha.data_ptr()) if dalpha is not None else None, lr,
            g.ctypes.data_as(C.POINTER(C.c_float)) if g is not None else None, C.byref(loss)))
        return loss.value, g

    def predict(self, tri7):
        """Predicted momenta, (pairs, T * N * 3) float64 on the device."""
        import torch

        out = torch.empty((tri7.shape[0], self.T * self.N * 3), dtype=torch.float64,
                          device="cuda")
        check_ws(lib.lddmm_ws_predict(self._h, C.c_void_p(tri7.data_ptr()), tri7.shape[0],
                                      tri7.shape[1], C.c_void_p(out.data_ptr())))
        return out


def lr_at(step, steps, lr, lr_final=None):
    """Learning rate of training step `step` of `steps`: lr throughout, or a half
    cosine from lr (step 0) down to lr_final (step `steps`)."""
    if lr_final is None:
        return lr
    return lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * step / steps))


def train(ws: WarmStart, tri7, labels, epochs=20, batch=64, lr=1e-3, seed=0, log=None,
          lr_final=None):
    """Adam over shuffled mini-batches (each pair's rows stay together), at a constant
    learning rate, or decayed from lr to lr_final along a half cosine over all steps
    when lr_final is given.  Returns the mean loss of every epoch."""
    import torch

    n = tri7.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    steps, step = epochs * (n // batch), 0
    # networks with local features: every pair's neighbours once, not in every step
    nbr = ws.neighbours(tri7, batch) if getattr(ws, "local_k", 0) else None
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).cuda()
        tot, cnt = 0.0, 0
        for k in range(0, n - batch + 1, batch):
            idx = perm[k:k + batch]
            lr_k = lr_at(step, steps, lr, lr_final)
            tot += ws.train_step(tri7.index_select(0, idx).contiguous(),
                                 labels.index_select(0, idx).contiguous(), lr_k,
                                 None if nbr is None else nbr.index_select(0, idx).contiguous())
            cnt += 1
            step += 1
        hist.append(tot / max(cnt, 1))
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {hist[-1]:.4e}")
    return hist


def train_objective(ws: WarmStart, probs, tri7, labels=None, epochs=50, batch=64, lr=3e-4,
                    label_weight=0.0, seed=0, log=None):
    """Amortised training on the registration objective itself.  The pairs are cut
    into fixed batches of `batch`, one batched context each; every step predicts a
    batch's momenta, evaluates the plain method's objective and gradient there
    (lddmm_objgrd_device) and back-propagates

        sum_p f_p(alpha_p) / (B f_p(0))  (+ label_weight * MSE(labels)),

    f_p(0) the objective at zero momenta, so every pair weighs the same.  The loss is
    the quantity a warm start should make small, in the metric of the objective (the
    kernel-weighted energy and the matching term), where the label loss weighs every
    momentum component alike.  Batches are visited in a shuffled order each epoch.
    Returns the mean normalised objective of every epoch."""
    import torch

    nb = len(probs) // batch
    ctxs, f0s = [], []
    try:
        for b in range(nb):
            ctx = api.Context(probs[b * batch:(b + 1) * batch])
            ctxs.append(ctx)
            z = torch.zeros(ctx.var_total, dtype=torch.float64, device="cuda")
            f = torch.empty(batch, dtype=torch.float64, device="cuda")
            g = torch.empty_like(z)
            torch.cuda.synchronize()
            check(lib.lddmm_objgrd_device(ctx.handle, C.c_void_p(z.data_ptr()),
                                          C.c_void_p(f.data_ptr()), C.c_void_p(g.data_ptr()), 0))
            f0s.append(f.clone())
        gen = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        for ep in range(epochs):
            tot, cnt = 0.0, 0
            for b in torch.randperm(nb, generator=gen).tolist():
                sl = slice(b * batch, (b + 1) * batch)
                tri = tri7[sl].contiguous()
                a = ws.predict(tri)
                f = torch.empty(batch, dtype=torch.float64, device="cuda")
                g = torch.empty_like(a)
                check(lib.lddmm_objgrd_device(ctxs[b].handle, C.c_void_p(a.data_ptr()),
                                              C.c_void_p(f.data_ptr()),
                                              C.c_void_p(g.data_ptr()), 0))
                rel_f = f / f0s[b]
                if not bool(torch.isfinite(rel_f).all()):
                    continue
                dalpha = (g / (f0s[b] * batch)[:, None]).contiguous()
                torch.cuda.synchronize()
                lab = labels[sl].contiguous() if (labels is not None and label_weight > 0) else None
                ws.backward(labels=lab, label_weight=label_weight, dalpha=dalpha, lr=lr)
                tot += float(rel_f.mean())
                cnt += 1
            hist.append(tot / max(cnt, 1))
            if log:
                log(f"objective epoch {ep + 1}/{epochs}: mean f / f(0) {hist[-1]:.5e}")
        return hist
    finally:
        for ctx in ctxs:
            ctx.close()


def _time_to(trace, f_target):
    """(iterations, evaluations) until the iteration table first reaches f_target."""
    ev = 1
    for k in range(trace.shape[0]):
        if k > 0:
            ev += int(trace[k, 3])
        if trace[k, 0] <= f_target:
            return k, ev
    return None, None


def evaluate(ws: WarmStart, seeds, batch=64, itr_max=300, rel_obj_tol=1e-6, rel=1e-5,
             make=pair):
    """Cold start (zero momenta) vs warm start (predicted momenta) on the pairs of
    `seeds`.  Per pair: iterations and objective evaluations until the objective is
    within `rel` of the cold start's converged objective, and whether the warm run's
    converged objective is within `rel` of it.  Batch wall times to convergence."""
    import torch

    rows = []
    t_cold = t_warm = 0.0
    for k in range(0, len(seeds), batch):
        probs = [make(s) for s in seeds[k:k + batch]]
        tri = torch.from_numpy(np.stack([features(P) for P in probs])).cuda()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        a0 = ws.predict(tri)
        torch.cuda.synchronize()
        t_pred = time.perf_counter() - t0
        _, cold, sc, tc = register_batch(probs, itr_max=itr_max, rel_obj_tol=rel_obj_tol,
                                         trace=True)
        _, warm, sw, tw = register_batch(probs, alp0=a0, itr_max=itr_max,
                                         rel_obj_tol=rel_obj_tol, trace=True)
        t_cold += sc
        t_warm += sw + t_pred
        for p in range(len(probs)):
            f_ref = cold[p]["f"]
            target = f_ref * (1.0 + rel) if f_ref >= 0 else f_ref * (1.0 - rel)
            ic, ec = _time_to(tc[p], target)
            iw, ew = _time_to(tw[p], target)
            rows.append(dict(seed=seeds[k + p], f_cold=f_ref, f_warm=warm[p]["f"],
                             f_start_warm=float(tw[p][0, 0]), f_start_cold=float(tc[p][0, 0]),
                             it_cold=ic, ev_cold=ec, it_warm=iw, ev_warm=ew,
                             match=warm[p]["f"] <= target))
    ok = [r for r in rows if r["ev_warm"] is not None and r["ev_cold"] is not None]
    return dict(
        pairs=len(rows),
        reached=len(ok),
        matched=sum(r["match"] for r in rows),
        median_evals_cold=float(np.median([r["ev_cold"] for r in ok])) if ok else None,
        median_evals_warm=float(np.median([r["ev_warm"] for r in ok])) if ok else None,
        median_speedup_evals=float(np.median([r["ev_cold"] / r["ev_warm"] for r in ok]))
        if ok else None,
        median_iters_cold=float(np.median([r["it_cold"] for r in ok])) if ok else None,
        median_iters_warm=float(np.median([r["it_warm"] for r in ok])) if ok else None,
        seconds_cold=t_cold, seconds_warm=t_warm,
        rows=rows)


def experiment(n_train=4096, n_test=512, subdiv=4, epochs=400, batch=64, lr=1e-3, seed=0,
               log=print, eval_itr_max=1000, eval_rel_obj_tol=1e-9, local_k=0,
               gen_itr_max=300, gen_rel_obj_tol=1e-6, lr_final=None):
    """The learned-warm-start workload end to end: plain-method registrations of
    n_train + n_test pairs (training seeds 1000.., held-out seeds 50000..), training,
    then cold vs warm start on the held-out pairs, both run to convergence (relative
    objective change below eval_rel_obj_tol, at most eval_itr_max iterations).
    local_k > 0: the network also reads every landmark's local_k nearest target
    triangles.  The training labels are registrations stopped at a relative objective
    change of gen_rel_obj_tol or gen_itr_max iterations.  Returns a JSON-ready dict."""
    import functools

    import torch

    make = functools.partial(pair, src_subdiv=subdiv, tgt_subdiv=subdiv)
    t0 = time.perf_counter()
    tri, lab, src, res = generate(list(range(1000, 1000 + n_train)), batch=batch, make=make,
                                  log=log, itr_max=gen_itr_max, rel_obj_tol=gen_rel_obj_tol)
    t_gen = time.perf_counter() - t0
    scale = float(lab.pow(2).mean().sqrt())
    with WarmStart(src, T_STEPS, batch_max=batch, tri_max=tri.shape[1], label_scale=scale,
                   seed=seed, local_k=local_k) as ws:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        hist = train(ws, tri, lab, epochs=epochs, batch=batch, lr=lr, seed=seed,
                     lr_final=lr_final)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        ev = evaluate(ws, list(range(50000, 50000 + n_test)), batch=batch, make=make,
                      itr_max=eval_itr_max, rel_obj_tol=eval_rel_obj_tol)
    rows = ev.pop("rows")
    ratio = [r["f_start_warm"] / r["f_start_cold"] for r in rows]
    return dict(n_train=n_train, n_test=n_test, local_k=local_k, gen_itr_max=gen_itr_max,
                gen_rel_obj_tol=gen_rel_obj_tol, lr_final=lr_final,
                landmarks=int(src.shape[0]),
                triangles=int(tri.shape[1]), epochs=epochs, batch=batch, lr=lr,
                label_rms=scale, seconds_generate=t_gen, seconds_train=t_train,
                steps=epochs * (n_train // batch), loss_first_epoch=hist[0],
                loss_last_epoch=hist[-1],
                median_start_objective_ratio=float(np.median(ratio)),
                median_plain_iterations=float(np.median([r["iters"] for r in res])), **ev)


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="learned warm start, end to end")
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--test", type=int, default=512)
    ap.add_argument("--subdiv", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--local-k", type=int, default=0,
                    help="nearest target triangles per landmark in the point input (0: the "
                         "configured network)")
    ap.add_argument("--label-tol", type=float, default=1e-6,
                    help="relative objective change at which the label registrations stop")
    ap.add_argument("--label-itr", type=int, default=300)
    ap.add_argument("--lr-final", type=float, default=None,
                    help="decay the learning rate to this value along a half cosine")
    a = ap.parse_args()
    print(json.dumps(experiment(a.train, a.test, a.subdiv, a.epochs, local_k=a.local_k,
                                gen_itr_max=a.label_itr, gen_rel_obj_tol=a.label_tol,
                                lr_final=a.lr_final)),
          flush=True)
