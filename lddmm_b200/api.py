"""Python host interface over the C ABI.

Two layers:

* ``Context`` -- a batch of registration pairs resident on the GPU, with
  ``objgrd`` / ``lbfgs`` / ``shoot`` on concatenated C-layout vectors.
* ``LDDMM``, ``objgrd``, ``multiplyKernel``, ``dqKernel``, ``varifold``,
  ``getElmIfo``, ``computeNodePosition`` -- the reference's MATLAB-level interface
  (``Cpp/src/LDDMM.m``, ``Cpp/src/computeNodePosition.m``, the MEX kernels), with
  MATLAB's array conventions (dim x N matrices, 1-based element tables in
  ``disObj``) so that driver scripts of the reference port line by line.
"""
from __future__ import annotations

import ctypes as C
import math
from types import SimpleNamespace

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr, lib
from .problem import Problem


def _problem_struct(P: Problem, keep: list) -> _lib.Problem:
    arrs = [P.ini_nde, P.elm_vtx, P.elm_ifo, P.tgt_cen, P.tgt_dir, P.tgt_vol]
    keep.extend(arrs)
    has_e = P.dfm_elm_num > 0
    return _lib.Problem(
        P.dim, P.nde_num, P.time_num, P.time_stp, P.knl_order, P.knl_width, dptr(P.ini_nde),
        P.dis_wgt, P.dfm_elm_num, iptr(P.elm_vtx) if has_e else None,
        int(P.elm_ifo.shape[1]) if has_e else 0, iptr(P.elm_ifo) if has_e else None,
        P.tgt_elm_num, dptr(P.tgt_cen), dptr(P.tgt_dir), dptr(P.tgt_vol),
        P.cen_type.encode(), P.cen_width, P.dir_type.encode(), P.dir_width)


class Context:
    """A batch of pairs on the GPU (``lddmm_ctx``)."""

    def __init__(self, problems, cluster=(0, 0, 0), autotune=None, use_graph=True,
                 stream=None, device=0, persistent=0):
        if isinstance(problems, Problem):
            problems = [problems]
        self.problems = list(problems)
        keep: list = []
        arr = (_lib.Problem * len(self.problems))(
            *[_problem_struct(P, keep) for P in self.problems])
        # autotune: None -> the library default (on), True -> on, False -> off (the
        # built-in launch-shape rule)
        tune = 0 if autotune is None else (1 if autotune else -1)
        cfg = _lib.Config(cluster[0], cluster[1], cluster[2], tune,
                          1 if use_graph else -1, stream, device, persistent)
        h = C.c_void_p()
        check(lib.lddmm_ctx_create(arr, len(self.problems), C.byref(cfg), C.byref(h)))
        self._h = h
        self.P = len(self.problems)
        self.var_num = [lib.lddmm_ctx_var_num(h, p) for p in range(self.P)]
        self.var_off = [lib.lddmm_ctx_var_offset(h, p) for p in range(self.P)]
        self.var_total = lib.lddmm_ctx_var_total(h)

    def close(self):
        if getattr(self, "_h", None):
            lib.lddmm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return lib.lddmm_ctx_stream(self._h) or 0

    def launch_config(self):
        o = np.zeros(3, dtype=np.int32)
        check(lib.lddmm_ctx_launch_config(self._h, iptr(o)))
        return tuple(int(x) for x in o)

    def launch_shape(self):
        """dict(cluster=(shoot, adjoint, varifold), tiles=(shoot, adjoint),
        persistent=0 | 1 | 2, plans=...): the launch shape the context runs (after
        autotuning); persistent 0: per-step launches, 1: persistent time loops
        combining split row groups in L2, 2: the cluster form.  plans: the cluster
        form's cluster size and CTAs, the L2 form's CTAs, and each plan's largest CTA
        share."""
        o = np.zeros(11, dtype=np.int32)
        check(lib.lddmm_ctx_launch_shape(self._h, iptr(o), 11))
        return dict(cluster=tuple(int(x) for x in o[:3]), tiles=(int(o[3]), int(o[4])),
                    persistent=int(o[5]),
                    plans=dict(cluster_size=int(o[6]), cluster_ctas=int(o[7]),
                               l2_ctas=int(o[8]), cluster_share=int(o[9]),
                               l2_share=int(o[10])))

    def time_sweeps(self, reps=3):
        """Average ms per launch: shooting step, adjoint step, varifold sweep, and
        the whole evaluation (CUDA events on the context stream)."""
        ms = np.zeros(4)
        check(lib.lddmm_ctx_time_sweeps(self._h, reps, dptr(ms)))
        return dict(shoot=ms[0], adjoint=ms[1], varifold=ms[2], eval=ms[3])

    def timeline(self):
        """Last cycle's device timeline (microseconds from the forward sweep's entry):
        entry/exit of the forward sweep, backward sweep and optimiser update."""
        t = np.zeros(6)
        check(lib.lddmm_ctx_timeline(self._h, dptr(t)))
        return dict(fwd=(t[0], t[1]), bwd=(t[2], t[3]), opt=(t[4], t[5]))

    def counters(self):
        o = (C.c_longlong * 4)()
        check(lib.lddmm_ctx_counters(self._h, o, 4))
        return dict(cycles=o[0], kernels_per_cycle=o[1], launches=o[2], evals=o[3])

    def split(self, vec):
        return [vec[o:o + n] for o, n in zip(self.var_off, self.var_num)]

    def objgrd(self, alp):
        alp = np.ascontiguousarray(alp, dtype=np.float64).reshape(-1)
        if alp.size != self.var_total:
            raise ValueError(f"alp has {alp.size} values, the batch {self.var_total}")
        f = np.zeros(self.P)
        g = np.zeros_like(alp)
        check(lib.lddmm_objgrd(self._h, dptr(alp), dptr(f), dptr(g)))
        return f, g

    def lbfgs(self, alp0, itr_max=1000, tol=1e-6, wolfe1=1e-4, wolfe2=0.9, mem_num=5,
              verbose=False, rel_obj_tol=0.0):
        """L-BFGS from alp0 for every pair of the batch (Cpp/src/LBFGS.cpp:25).
        Returns the final momenta and one dict per pair (f, glen, status, iters,
        evals).  A pair's own outcome is its ``status``: 0, the line-search codes 1-3,
        or -3 (LDDMM_ERR_NONFINITE) for a pair whose objective was not finite; those
        do not raise, so the other pairs' results stay available.  Errors of the call
        itself (arguments, CUDA, timeouts, memory) raise LddmmError."""
        x = np.ascontiguousarray(alp0, dtype=np.float64).reshape(-1).copy()
        if x.size != self.var_total:
            raise ValueError(f"alp0 has {x.size} values, the batch {self.var_total}")
        opt = _lib.Opt(itr_max, tol, wolfe1, wolfe2, mem_num, 1 if verbose else 0, rel_obj_tol)
        res = (_lib.Result * self.P)()
        rc = lib.lddmm_lbfgs(self._h, C.byref(opt), dptr(x), res)
        if rc < 0 and rc != -3:
            check(rc)
        out = [dict(f=r.fcn, glen=r.grd_len, status=r.status, iters=r.iters, evals=r.evals)
               for r in res]
        return x, out

    def lbfgs_grad(self):
        """Gradient at the last accepted point of the last ``lbfgs`` call (the
        reference's grdNow), concatenated over the pairs like the momenta."""
        g = np.zeros(self.var_total)
        check(lib.lddmm_lbfgs_grad(self._h, dptr(g)))
        return g

    def trace(self, pair=0, cap=100001):
        rows = np.zeros((cap, 4))
        n = check(lib.lddmm_lbfgs_trace(self._h, pair, dptr(rows), cap))
        return rows[:n]

    def shoot(self, alp):
        alp = np.ascontiguousarray(alp, dtype=np.float64).reshape(-1)
        tot_n = sum(P.dim * P.nde_num * P.time_num for P in self.problems)
        tot_v = sum(P.dim * P.nde_num * (P.time_num - 1) for P in self.problems)
        nde = np.zeros(tot_n)
        vlc = np.zeros(tot_v)
        check(lib.lddmm_shoot(self._h, dptr(alp), dptr(nde), dptr(vlc)))
        out, a, b = [], 0, 0
        for P in self.problems:
            n1 = P.dim * P.nde_num * P.time_num
            n2 = P.dim * P.nde_num * (P.time_num - 1)
            out.append((nde[a:a + n1].reshape(P.time_num, P.nde_num, P.dim),
                        vlc[b:b + n2].reshape(P.time_num - 1, P.nde_num, P.dim)))
            a += n1
            b += n2
        return out


# ------------------------------------------------------ reference-level functions

def objgrd(P: Problem, alp):
    """``objgrd`` (Cpp/src/objgrd.cpp:26) for one problem: (f, grad)."""
    with Context(P) as ctx:
        f, g = ctx.objgrd(alp)
    return float(f[0]), g


def _pts(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def computeKernel(*args):
    """Dense kernel matrix, as the MEX ``computeKernel`` (MATLAB/src/computeKernelITF.cpp):
    ``computeKernel(lmk, knl_order, knl_width)`` -> (N, N), or
    ``computeKernel(lmki, lmkj, knl_order, knl_width)`` -> (Ni, Nj) with entry (i, j) =
    K(lmki_i, lmkj_j) (Cpp/src/computeKernel.cpp:21 and :246).  Points are (N, D)."""
    if len(args) == 3:
        qi, qj, (order, width) = _pts(args[0]), None, args[1:]
    elif len(args) == 4:
        qi, qj, (order, width) = _pts(args[0]), _pts(args[1]), args[2:]
    else:
        raise TypeError("computeKernel takes 3 or 4 arguments")
    nj = qi.shape[0] if qj is None else qj.shape[0]
    K = np.zeros((nj, qi.shape[0]))  # the reference's column-major Ni x Nj
    check(lib.lddmm_compute_kernel(qi.shape[1], qi.shape[0], dptr(qi), nj,
                                   None if qj is None else dptr(qj), order, width, dptr(K)))
    return K.T.copy()


def multiplyKernel(*args):
    """As the MEX ``multiplyKernel`` (MATLAB/src/multiplyKernelITF.cpp):
    ``multiplyKernel(q, a, knl_order, knl_width)``: v_i = sum_j K(q_i, q_j) a_j
    (Cpp/src/multiplyKernel.cpp:22); ``multiplyKernel(qi, qj, a, knl_order, knl_width)``:
    v_i = sum_j K(qi_i, qj_j) a_j with a on the j set (multiplyKernel.cpp:294).
    Points and vectors are (N, D)."""
    if len(args) == 4:
        q, a, order, width = _pts(args[0]), _pts(args[1]), args[2], args[3]
        v = np.zeros_like(q)
        check(lib.lddmm_multiply_kernel(q.shape[1], q.shape[0], dptr(q), dptr(a), order,
                                        width, dptr(v)))
        return v
    if len(args) == 5:
        qi, qj, a, order, width = _pts(args[0]), _pts(args[1]), _pts(args[2]), args[3], args[4]
        v = np.zeros_like(qi)
        check(lib.lddmm_multiply_kernel2(qi.shape[1], qi.shape[0], dptr(qi), qj.shape[0],
                                         dptr(qj), dptr(a), order, width, dptr(v)))
        return v
    raise TypeError("multiplyKernel takes 4 or 5 arguments")


def dqKernel(*args):
    """As the MEX ``dqKernel`` (MATLAB/src/dqKernelITF.cpp):
    ``dqKernel(q, l, r, knl_order, knl_width)``: dq_i = sum_j (l_i.r_j + l_j.r_i) dK/dq_i
    (Cpp/src/dqKernel.cpp:31); ``dqKernel(qi, qj, l, r, knl_order, knl_width)`` ->
    (dqi, dqj), the gradients of sum_ij l_i.r_j K(qi_i, qj_j) with respect to qi and qj,
    l on the i set, r on the j set (dqKernel.cpp:307)."""
    if len(args) == 5:
        q, l, r = (_pts(x) for x in args[:3])
        order, width = args[3], args[4]
        dq = np.zeros_like(q)
        check(lib.lddmm_dq_kernel(q.shape[1], q.shape[0], dptr(q), dptr(l), dptr(r), order,
                                  width, dptr(dq)))
        return dq
    if len(args) == 6:
        qi, qj, l, r = (_pts(x) for x in args[:4])
        order, width = args[4], args[5]
        dqi, dqj = np.zeros_like(qi), np.zeros_like(qj)
        check(lib.lddmm_dq_kernel2(qi.shape[1], qi.shape[0], dptr(qi), qj.shape[0], dptr(qj),
                                   dptr(l), dptr(r), order, width, dptr(dqi), dptr(dqj)))
        return dqi, dqj
    raise TypeError("dqKernel takes 5 or 6 arguments")


def varifold(P: Problem, nde):
    """Varifold discrepancy and its gradient at landmark positions ``nde`` (N, D)
    (Cpp/src/varifoldITF.cpp:7)."""
    nde = np.ascontiguousarray(nde, dtype=np.float64)
    keep: list = []
    s = _problem_struct(P, keep)
    v = C.c_double()
    dq = np.zeros_like(nde)
    check(lib.lddmm_varifold(C.byref(s), dptr(nde), C.byref(v), dptr(dq)))
    return v.value, dq


def getElmIfo(elmVtxMat, ndeNum):
    """``getElmIfo.m`` with MATLAB conventions: elmVtxMat is (2 or 3) x E, 1-based;
    returns the int32 rows x N table (0-based entries), as LDDMM.m passes it on."""
    ev = np.ascontiguousarray(np.asarray(elmVtxMat).T - 1, dtype=np.int32)
    rows = check(lib.lddmm_elm_ifo(iptr(ev), ev.shape[1], ev.shape[0], ndeNum, None))
    out = np.zeros((ndeNum, rows), dtype=np.int32)
    check(lib.lddmm_elm_ifo(iptr(ev), ev.shape[1], ev.shape[0], ndeNum, iptr(out)))
    return out.T


def computeNodePosition(iniNdeMat, alpStk, knlOrder, knlWidth, timeStp, timeNum):
    """``computeNodePosition.m``: iniNdeMat dim x N, alpStk dim x N x (timeNum-1);
    returns ndeStk dim x N x timeNum and vlcStk dim x N x (timeNum-1)."""
    ini = np.asarray(iniNdeMat, dtype=np.float64)
    dim, n = ini.shape
    P = Problem(ini.T, np.zeros((0, dim), np.int32), np.zeros((0, dim)), np.zeros((0, dim)),
                np.zeros(0), knl_order=knlOrder, knl_width=knlWidth, time_num=timeNum,
                time_stp=timeStp, elm_ifo=np.zeros((n, 1), np.int32))
    alp = np.transpose(np.asarray(alpStk, dtype=np.float64), (2, 1, 0)).reshape(-1)
    with Context(P) as ctx:
        (nde, vlc), = ctx.shoot(alp)
    return np.transpose(nde, (2, 1, 0)), np.transpose(vlc, (2, 1, 0))


def _scalar(v):
    """A MATLAB scalar or char array as loaded from a .mat file (1 x 1 arrays, 1-element
    string arrays) or as given in Python."""
    a = np.asarray(v)
    if a.dtype.kind in "US":
        return str(a.ravel()[0]) if a.size else ""
    return a.ravel()[0].item() if a.size == 1 else v


def problem_from_matlab(iniNdeMat, disObj, knlOrder, knlWidth, timeEnd, timeStp) -> Problem:
    """The problem that ``LDDMM`` (Cpp/src/LDDMM.m) solves, from its MATLAB-layout
    arguments: iniNdeMat dim x N; disObj (dict or object) with dfmElmVtxMat
    ((2|3) x E_d, 1-based), tgtCenPosMat / tgtUniDirMat (dim x E_t), tgtElmVolVec
    (E_t values), cenKnlType, cenKnlWidth, dirKnlType, dirKnlWidth, disWgt; timeNum =
    floor(timeEnd / timeStp) + 1.  Fields may be numpy values or the 1 x 1 arrays that
    ``scipy.io.loadmat`` returns."""
    d = disObj if isinstance(disObj, dict) else vars(disObj)
    ini = np.asarray(iniNdeMat, dtype=np.float64)
    timeEnd, timeStp = float(_scalar(timeEnd)), float(_scalar(timeStp))
    timeNum = int(math.floor(timeEnd / timeStp)) + 1
    ev = np.asarray(d["dfmElmVtxMat"]).T.astype(np.int32) - 1
    return Problem(ini.T, ev, np.asarray(d["tgtCenPosMat"], dtype=np.float64).T,
                   np.asarray(d["tgtUniDirMat"], dtype=np.float64).T,
                   np.asarray(d["tgtElmVolVec"], dtype=np.float64).ravel(),
                   knl_order=int(_scalar(knlOrder)), knl_width=float(_scalar(knlWidth)),
                   time_num=timeNum, time_stp=timeStp, cen_type=str(_scalar(d["cenKnlType"])),
                   cen_width=float(_scalar(d["cenKnlWidth"])),
                   dir_type=str(_scalar(d["dirKnlType"])),
                   dir_width=float(_scalar(d["dirKnlWidth"])),
                   dis_wgt=float(_scalar(d["disWgt"])))


def LDDMM(iniNdeMat, iniAlpStk, disObj, knlOrder, knlWidth, timeEnd, timeStp, optObj):
    """``Cpp/src/LDDMM.m``: [ndeStk, vlcStk, alpStk] = LDDMM(iniNdeMat, iniAlpStk,
    disObj, knlOrder, knlWidth, timeEnd, timeStp, optObj).

    MATLAB conventions: iniNdeMat dim x N; disObj has dfmElmVtxMat ((2|3) x E_d,
    1-based), tgtCenPosMat, tgtElmVolVec, tgtUniDirMat, cenKnlType, cenKnlWidth,
    dirKnlType, dirKnlWidth, disWgt; optObj has MaxIterations, OptimalityTolerance,
    Wolfe1, Wolfe2, Columns, Verbose.  Missing optObj fields take the defaults of
    MATLAB/src/LBFGS.m:86-110.  iniAlpStk may be None (zeros)."""
    o = optObj if isinstance(optObj, dict) else vars(optObj)
    ini = np.asarray(iniNdeMat, dtype=np.float64)
    dim, n = ini.shape
    P = problem_from_matlab(iniNdeMat, disObj, knlOrder, knlWidth, timeEnd, timeStp)
    timeNum = P.time_num
    nvar = dim * n * (timeNum - 1)
    if iniAlpStk is None or np.size(iniAlpStk) == 0:
        alp0 = np.zeros(nvar)
    else:
        alp0 = np.transpose(np.asarray(iniAlpStk, dtype=np.float64).reshape(
            dim, n, timeNum - 1, order="F"), (2, 1, 0)).reshape(-1)
    with Context(P) as ctx:
        x, res = ctx.lbfgs(alp0, itr_max=int(_scalar(o.get("MaxIterations", 1000))),
                           tol=float(_scalar(o.get("OptimalityTolerance", 1e-6))),
                           wolfe1=float(_scalar(o.get("Wolfe1", 1e-4))),
                           wolfe2=float(_scalar(o.get("Wolfe2", 0.9))),
                           mem_num=int(_scalar(o.get("Columns", min(100, nvar)))),
                           verbose=bool(_scalar(o.get("Verbose", False))))
    alpStk = np.transpose(x.reshape(timeNum - 1, n, dim), (2, 1, 0))
    ndeStk, vlcStk = computeNodePosition(ini, alpStk, P.knl_order, P.knl_width, P.time_stp,
                                         timeNum)
    return SimpleNamespace(ndeStk=ndeStk, vlcStk=vlcStk, alpStk=alpStk, result=res[0])
