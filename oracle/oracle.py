"""ctypes access to the CPU oracle (test infrastructure only).

Two back-ends with the same Python surface:

* ``Oracle``    -- liblddmm_oracle.so, the project's FP64 C restatement of the
  reference path (oracle/lddmm_oracle.c).  Built from this repository; travels
  with it.
* ``Reference`` -- oracle/_ref/libref{2,3}d.so, the reference's own Cpp/src sources
  compiled in place by ``make -C oracle ref`` (needs the reference tree at build
  time; the built .so files travel, the tree does not).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU baseline may use this
module, as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class _Prob(C.Structure):
    _fields_ = [("dim", C.c_int), ("nde_num", C.c_int), ("time_num", C.c_int),
                ("time_stp", C.c_double), ("knl_order", C.c_int), ("knl_width", C.c_double),
                ("ini_nde", _dp), ("dis_wgt", C.c_double), ("dfm_elm_num", C.c_int),
                ("dfm_elm_vtx", _ip), ("dfm_elm_ifo_num", C.c_int), ("dfm_elm_ifo", _ip),
                ("tgt_elm_num", C.c_int), ("tgt_cen_pos", _dp), ("tgt_uni_dir", _dp),
                ("tgt_elm_vol", _dp), ("cen_knl_type", C.c_char), ("cen_knl_width", C.c_double),
                ("dir_knl_type", C.c_char), ("dir_knl_width", C.c_double)]


def _prob_struct(P):
    s = _Prob(P.dim, P.nde_num, P.time_num, P.time_stp, P.knl_order, P.knl_width,
              _d(P.ini_nde), P.dis_wgt, P.dfm_elm_num, _i(P.elm_vtx), P.elm_ifo.shape[1],
              _i(P.elm_ifo), P.tgt_elm_num, _d(P.tgt_cen), _d(P.tgt_dir), _d(P.tgt_vol),
              P.cen_type.encode(), P.cen_width, P.dir_type.encode(), P.dir_width)
    return s


class Oracle:
    """The project's FP64 C restatement."""

    def __init__(self, path: str | None = None, threads: int = 0):
        path = path or os.path.join(HERE, "liblddmm_oracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_objgrd.restype = C.c_int
        L.orc_varifold.restype = C.c_int
        L.orc_varifold_tt.restype = C.c_double
        L.orc_lbfgs.restype = C.c_int
        L.orc_elm_ifo.restype = C.c_int
        L.orc_p0.restype = C.c_double
        L.orc_p0.argtypes = [C.c_double]
        L.orc_p1.restype = C.c_double
        L.orc_p1.argtypes = [C.c_double]
        if threads:
            L.orc_set_threads(C.c_int(threads))

    def set_threads(self, n: int):
        self.lib.orc_set_threads(C.c_int(n))

    def objgrd(self, P, alp):
        alp = np.ascontiguousarray(alp, dtype=np.float64).reshape(-1)
        assert alp.size == P.var_num
        g = np.zeros_like(alp)
        f = C.c_double()
        s = _prob_struct(P)
        rc = self.lib.orc_objgrd(C.byref(s), _d(alp), C.byref(f), _d(g))
        if rc:
            raise RuntimeError(f"orc_objgrd rc={rc}")
        return f.value, g

    def varifold(self, P, nde):
        nde = np.ascontiguousarray(nde, dtype=np.float64)
        dq = np.zeros_like(nde)
        v = C.c_double()
        s = _prob_struct(P)
        rc = self.lib.orc_varifold(C.byref(s), _d(nde), C.byref(v), _d(dq))
        if rc:
            raise RuntimeError(f"orc_varifold rc={rc}")
        return v.value, dq

    def varifold_tt(self, P):
        s = _prob_struct(P)
        return self.lib.orc_varifold_tt(C.byref(s))

    def lbfgs(self, P, alp0, itr_max=300, tol=1e-6, wolfe1=1e-4, wolfe2=0.9, mem_num=5,
              trace_cap=100000):
        x = np.ascontiguousarray(alp0, dtype=np.float64).reshape(-1).copy()
        g = np.zeros_like(x)
        f = C.c_double()
        code, iters, evals = C.c_int(), C.c_int(), C.c_int()
        tf = np.zeros(trace_cap)
        tg = np.zeros(trace_cap)
        s = _prob_struct(P)
        ret = self.lib.orc_lbfgs(C.byref(s), C.c_int(itr_max), C.c_double(tol),
                                 C.c_double(wolfe1), C.c_double(wolfe2), C.c_int(mem_num),
                                 _d(x), C.byref(f), _d(g), C.byref(code), C.byref(iters),
                                 C.byref(evals), _d(tf), _d(tg), C.c_int(trace_cap))
        n = min(evals.value, trace_cap)
        return dict(ret=ret, ls_code=code.value, x=x, f=f.value, g=g, iters=iters.value,
                    evals=evals.value, trace_f=tf[:n].copy(), trace_g2=tg[:n].copy())

    def multiply_kernel(self, q, a, order, width):
        q = np.ascontiguousarray(q, dtype=np.float64)
        a = np.ascontiguousarray(a, dtype=np.float64)
        v = np.zeros_like(q)
        self.lib.orc_multiply_kernel(_d(v), _d(q), _d(a), C.c_int(order), C.c_double(width),
                                     C.c_int(q.shape[0]), C.c_int(q.shape[1]))
        return v

    def dq_kernel(self, q, l, r, order, width):
        q, l, r = (np.ascontiguousarray(x, dtype=np.float64) for x in (q, l, r))
        dq = np.zeros_like(q)
        self.lib.orc_dq_kernel(_d(dq), _d(q), _d(l), _d(r), C.c_int(order), C.c_double(width),
                               C.c_int(q.shape[0]), C.c_int(q.shape[1]))
        return dq

    def compute_kernel(self, q, order, width):
        """(n, n) matrix K(q_i, q_j) (computeKernel.cpp:21)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        K = np.zeros((q.shape[0], q.shape[0]))
        self.lib.orc_compute_kernel(_d(K), _d(q), C.c_int(order), C.c_double(width),
                                    C.c_int(q.shape[0]), C.c_int(q.shape[1]))
        return K

    # two point sets (computeKernel.cpp:246, multiplyKernel.cpp:294, dqKernel.cpp:307)
    def compute_kernel2(self, qi, qj, order, width):
        """(ni, nj) matrix K(qi_i, qj_j)."""
        qi, qj = (np.ascontiguousarray(x, dtype=np.float64) for x in (qi, qj))
        K = np.zeros((qj.shape[0], qi.shape[0]))  # column-major ni x nj
        self.lib.orc_compute_kernel2(_d(K), _d(qi), C.c_int(qi.shape[0]), _d(qj),
                                     C.c_int(qj.shape[0]), C.c_int(order), C.c_double(width),
                                     C.c_int(qi.shape[1]))
        return K.T.copy()

    def multiply_kernel2(self, qi, qj, a, order, width):
        qi, qj, a = (np.ascontiguousarray(x, dtype=np.float64) for x in (qi, qj, a))
        v = np.zeros_like(qi)
        self.lib.orc_multiply_kernel2(_d(v), _d(qi), C.c_int(qi.shape[0]), _d(qj),
                                      C.c_int(qj.shape[0]), _d(a), C.c_int(order),
                                      C.c_double(width), C.c_int(qi.shape[1]))
        return v

    def dq_kernel2(self, qi, qj, l, r, order, width):
        qi, qj, l, r = (np.ascontiguousarray(x, dtype=np.float64) for x in (qi, qj, l, r))
        dqi, dqj = np.zeros_like(qi), np.zeros_like(qj)
        self.lib.orc_dq_kernel2(_d(dqi), _d(dqj), _d(qi), C.c_int(qi.shape[0]), _d(qj),
                                C.c_int(qj.shape[0]), _d(l), _d(r), C.c_int(order),
                                C.c_double(width), C.c_int(qi.shape[1]))
        return dqi, dqj

    def elm_ifo(self, elm_vtx, nde_num):
        ev = np.ascontiguousarray(elm_vtx, dtype=np.int32)
        rows = self.lib.orc_elm_ifo(_i(ev), C.c_int(ev.shape[1]), C.c_int(ev.shape[0]),
                                    C.c_int(nde_num), None)
        out = np.zeros((nde_num, rows), dtype=np.int32)
        self.lib.orc_elm_ifo(_i(ev), C.c_int(ev.shape[1]), C.c_int(ev.shape[0]),
                             C.c_int(nde_num), _i(out))
        return out

    def shoot(self, ini, alp, order, width, dt, time_num):
        ini = np.ascontiguousarray(ini, dtype=np.float64)
        n, dim = ini.shape
        alp = np.ascontiguousarray(alp, dtype=np.float64).reshape(-1)
        nde = np.zeros((time_num, n, dim))
        vlc = np.zeros((time_num - 1, n, dim))
        self.lib.orc_shoot(_d(ini), _d(alp), C.c_int(order), C.c_double(width), C.c_double(dt),
                           C.c_int(time_num), C.c_int(n), C.c_int(dim), _d(nde), _d(vlc))
        return nde, vlc

    def p0(self, x):
        return self.lib.orc_p0(float(x))

    def p1(self, x):
        return self.lib.orc_p1(float(x))


class Reference:
    """The reference's own C++ path compiled in place (oracle/_ref)."""

    def __init__(self, dim: int):
        path = os.path.join(HERE, "_ref", f"libref{dim}d.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.dim = dim
        self.lib = C.CDLL(path)

    @staticmethod
    def available(dim: int = 3) -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", f"libref{dim}d.so"))

    def _common(self, P):
        return [_d(P.ini_nde), C.c_int(P.nde_num), C.c_int(P.time_num), C.c_double(P.time_stp),
                C.c_int(P.knl_order), C.c_double(P.knl_width), _i(P.elm_vtx),
                C.c_int(P.dfm_elm_num), _i(P.elm_ifo), C.c_int(P.elm_ifo.shape[1]),
                _d(P.tgt_cen), _d(P.tgt_dir), _d(P.tgt_vol), C.c_int(P.tgt_elm_num),
                C.c_char(P.cen_type.encode()), C.c_double(P.cen_width),
                C.c_char(P.dir_type.encode()), C.c_double(P.dir_width), C.c_double(P.dis_wgt)]

    def objgrd(self, P, alp):
        assert P.dim == self.dim
        alp = np.ascontiguousarray(alp, dtype=np.float64).reshape(-1)
        g = np.zeros_like(alp)
        f = C.c_double()
        rc = self.lib.ref_objgrd(*self._common(P), _d(alp), C.byref(f), _d(g))
        if rc:
            raise RuntimeError(f"ref_objgrd rc={rc}")
        return f.value, g

    def lbfgs(self, P, alp0, itr_max=300, tol=1e-6, wolfe1=1e-4, wolfe2=0.9, mem_num=5,
              trace_cap=100000, verbose=False):
        assert P.dim == self.dim
        x = np.ascontiguousarray(alp0, dtype=np.float64).reshape(-1).copy()
        g = np.zeros_like(x)
        f = C.c_double()
        tf = np.zeros(trace_cap)
        tg = np.zeros(trace_cap)
        n = C.c_int()
        ret = self.lib.ref_lbfgs(*self._common(P), C.c_int(itr_max), C.c_double(tol),
                                 C.c_double(wolfe1), C.c_double(wolfe2), C.c_int(mem_num),
                                 C.c_int(1 if verbose else 0), _d(x), C.byref(f), _d(g),
                                 _d(tf), _d(tg), C.c_int(trace_cap), C.byref(n))
        k = min(n.value, trace_cap)
        return dict(ret=ret, x=x, f=f.value, g=g, evals=n.value, trace_f=tf[:k].copy(),
                    trace_g2=tg[:k].copy())

    def varifold(self, P, nde):
        nde = np.ascontiguousarray(nde, dtype=np.float64)
        dq = np.zeros_like(nde)
        v = C.c_double()
        rc = self.lib.ref_varifold(_d(nde), C.c_int(P.nde_num), _i(P.elm_vtx),
                                   C.c_int(P.dfm_elm_num), _i(P.elm_ifo),
                                   C.c_int(P.elm_ifo.shape[1]), _d(P.tgt_cen), _d(P.tgt_dir),
                                   _d(P.tgt_vol), C.c_int(P.tgt_elm_num),
                                   C.c_char(P.cen_type.encode()), C.c_double(P.cen_width),
                                   C.c_char(P.dir_type.encode()), C.c_double(P.dir_width),
                                   C.byref(v), _d(dq))
        if rc:
            raise RuntimeError(f"ref_varifold rc={rc}")
        return v.value, dq

    def multiply_kernel(self, q, a, order, width):
        q = np.ascontiguousarray(q, dtype=np.float64)
        a = np.ascontiguousarray(a, dtype=np.float64)
        v = np.zeros_like(q)
        self.lib.ref_multiply_kernel(_d(v), _d(q), _d(a), C.c_int(order), C.c_double(width),
                                     C.c_int(q.shape[0]), C.c_int(q.shape[1]))
        return v

    def dq_kernel(self, q, l, r, order, width):
        q, l, r = (np.ascontiguousarray(x, dtype=np.float64) for x in (q, l, r))
        dq = np.zeros_like(q)
        self.lib.ref_dq_kernel(_d(dq), _d(q), _d(l), _d(r), C.c_int(order), C.c_double(width),
                               C.c_int(q.shape[0]), C.c_int(q.shape[1]))
        return dq

    def compute_kernel(self, q, order, width):
        q = np.ascontiguousarray(q, dtype=np.float64)
        K = np.zeros((q.shape[0], q.shape[0]))  # column-major n x n
        self.lib.ref_compute_kernel(_d(K), _d(q), C.c_int(order), C.c_double(width),
                                    C.c_int(q.shape[0]), C.c_int(q.shape[1]))
        return K.T.copy()

    def compute_kernel2(self, qi, qj, order, width):
        qi, qj = (np.ascontiguousarray(x, dtype=np.float64) for x in (qi, qj))
        K = np.zeros((qj.shape[0], qi.shape[0]))
        self.lib.ref_compute_kernel2(_d(K), _d(qi), C.c_int(qi.shape[0]), _d(qj),
                                     C.c_int(qj.shape[0]), C.c_int(order), C.c_double(width),
                                     C.c_int(qi.shape[1]))
        return K.T.copy()

    def multiply_kernel2(self, qi, qj, a, order, width):
        qi, qj, a = (np.ascontiguousarray(x, dtype=np.float64) for x in (qi, qj, a))
        v = np.zeros_like(qi)
        self.lib.ref_multiply_kernel2(_d(v), _d(qi), C.c_int(qi.shape[0]), _d(qj),
                                      C.c_int(qj.shape[0]), _d(a), C.c_int(order),
                                      C.c_double(width), C.c_int(qi.shape[1]))
        return v

    def dq_kernel2(self, qi, qj, l, r, order, width):
        qi, qj, l, r = (np.ascontiguousarray(x, dtype=np.float64) for x in (qi, qj, l, r))
        dqi, dqj = np.zeros_like(qi), np.zeros_like(qj)
        self.lib.ref_dq_kernel2(_d(dqi), _d(dqj), _d(qi), C.c_int(qi.shape[0]), _d(qj),
                                C.c_int(qj.shape[0]), _d(l), _d(r), C.c_int(order),
                                C.c_double(width), C.c_int(qi.shape[1]))
        return dqi, dqj


class ReferenceCuda:
    """The reference's plain FP64 GPU path (CUDA/src, cuBLAS) compiled in place
    (oracle/_ref/librefcu{2,3}d.so, ``make -C oracle refcu``) behind a project host
    driver that replaces its MEX entry (CUDA/src/LDDMM.cu:13-151).  Same argument
    meaning and C++ layouts as :class:`Reference`.  Needs a GPU; measurement and test
    infrastructure only."""

    def __init__(self, dim: int):
        path = os.path.join(HERE, "_ref", f"librefcu{dim}d.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle refcu`")
        self.dim = dim
        self.lib = C.CDLL(path)
        assert self.lib.refcu_dim() == dim

    @staticmethod
    def available(dim: int = 3) -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", f"librefcu{dim}d.so"))

    _common = Reference._common

    def objgrd(self, P, alp):
        assert P.dim == self.dim
        alp = np.ascontiguousarray(alp, dtype=np.float64).reshape(-1)
        g = np.zeros_like(alp)
        f = C.c_double()
        rc = self.lib.refcu_objgrd(*self._common(P), _d(alp), C.byref(f), _d(g))
        if rc:
            raise RuntimeError(f"refcu_objgrd rc={rc}")
        return f.value, g

    def lbfgs(self, P, alp0, itr_max=300, tol=1e-6, wolfe1=1e-4, wolfe2=0.9, mem_num=5,
              verbose=False):
        """One registration; returns status, momenta, final objective, evaluations and
        the milliseconds spent inside LBFGS (CUDA events) and in the whole call."""
        assert P.dim == self.dim
        x = np.ascontiguousarray(alp0, dtype=np.float64).reshape(-1).copy()
        out = np.zeros(4)
        ret = self.lib.refcu_lbfgs(*self._common(P), C.c_int(itr_max), C.c_double(tol),
                                   C.c_double(wolfe1), C.c_double(wolfe2), C.c_int(mem_num),
                                   C.c_int(1 if verbose else 0), _d(x), _d(out))
        if ret < 0:
            raise RuntimeError(f"refcu_lbfgs rc={ret}")
        return dict(ret=ret, x=x, f=float(out[3]), evals=int(out[2]), ms_lbfgs=float(out[0]),
                    ms_total=float(out[1]))
