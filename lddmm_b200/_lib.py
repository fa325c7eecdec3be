"""ctypes bindings to liblddmm_b200.so (the C ABI declared in include/lddmm_b200.h).

The shared library is the product: there is no CPU fallback.  Importing this module
on a machine without the built library raises ImportError; calling a compute entry
point without a GPU returns a CUDA error (LddmmError).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblddmm_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

# every function the header declares, for the export check
EXPORTS = [
    "lddmm_last_error", "lddmm_version", "lddmm_ctx_create", "lddmm_ctx_destroy",
    "lddmm_ctx_num_pairs", "lddmm_ctx_var_num", "lddmm_ctx_var_offset", "lddmm_ctx_var_total",
    "lddmm_ctx_stream", "lddmm_ctx_launch_config", "lddmm_ctx_launch_shape", "lddmm_objgrd", "lddmm_objgrd_device", "lddmm_objgrd_costate",
    "lddmm_lbfgs", "lddmm_lbfgs_device", "lddmm_lbfgs_trace", "lddmm_shoot", "lddmm_LDDMM",
    "lddmm_elm_ifo", "lddmm_multiply_kernel", "lddmm_dq_kernel", "lddmm_varifold",
    "lddmm_flops_per_pair", "lddmm_ctx_time_sweeps", "lddmm_ctx_counters",
    "lddmm_fp32_peak", "lddmm_pipe_peaks", "lddmm_spatial_order", "lddmm_multiply_kernel_noalloc", "lddmm_ctx_timeline",
    "lddmm_ws_create", "lddmm_ws_create_ex", "lddmm_ws_destroy", "lddmm_ws_last_error", "lddmm_ws_num_params",
    "lddmm_ws_params", "lddmm_ws_grad", "lddmm_ws_train_step", "lddmm_ws_neighbours", "lddmm_ws_train_step_nbr",
    "lddmm_ws_predict", "lddmm_ws_backward",
    "lddmm_ws_gemm_bf16", "lddmm_wait_selftest", "lddmm_compute_kernel",
    "lddmm_multiply_kernel2", "lddmm_dq_kernel2", "lddmm_lbfgs_grad",
]

ERRORS = {
    -1: "LDDMM_ERR_ARG", -2: "LDDMM_ERR_CUDA", -3: "LDDMM_ERR_NONFINITE",
    -4: "LDDMM_ERR_TIMEOUT", -5: "LDDMM_ERR_NOMEM", -6: "LDDMM_ERR_UNSUPPORTED",
}


class LddmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Problem(C.Structure):
    _fields_ = [("dim", C.c_int), ("nde_num", C.c_int), ("time_num", C.c_int),
                ("time_stp", C.c_double), ("knl_order", C.c_int), ("knl_width", C.c_double),
                ("ini_nde", _dp), ("dis_wgt", C.c_double), ("dfm_elm_num", C.c_int),
                ("dfm_elm_vtx", _ip), ("dfm_elm_ifo_num", C.c_int), ("dfm_elm_ifo", _ip),
                ("tgt_elm_num", C.c_int), ("tgt_cen_pos", _dp), ("tgt_uni_dir", _dp),
                ("tgt_elm_vol", _dp), ("cen_knl_type", C.c_char), ("cen_knl_width", C.c_double),
                ("dir_knl_type", C.c_char), ("dir_knl_width", C.c_double)]


class Opt(C.Structure):
    _fields_ = [("itr_max", C.c_int), ("tol_val", C.c_double), ("wolfe1", C.c_double),
                ("wolfe2", C.c_double), ("mem_num", C.c_int), ("vbs_flg", C.c_int),
                ("rel_obj_tol", C.c_double)]


class Config(C.Structure):
    _fields_ = [("cluster_shoot", C.c_int), ("cluster_adjoint", C.c_int),
                ("cluster_varifold", C.c_int), ("autotune", C.c_int), ("use_graph", C.c_int),
                ("stream", C.c_void_p), ("device", C.c_int), ("persistent", C.c_int)]


class Result(C.Structure):
    _fields_ = [("fcn", C.c_double), ("grd_len", C.c_double), ("status", C.c_int),
                ("iters", C.c_int), ("evals", C.c_int), ("pad_", C.c_int)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m lddmm_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.lddmm_last_error.restype = C.c_char_p
    L.lddmm_version.restype = C.c_char_p
    L.lddmm_ctx_create.argtypes = [C.POINTER(Problem), C.c_int, C.POINTER(Config),
                                   C.POINTER(C.c_void_p)]
    L.lddmm_ctx_destroy.argtypes = [C.c_void_p]
    L.lddmm_ctx_destroy.restype = None
    L.lddmm_ctx_num_pairs.argtypes = [C.c_void_p]
    for f in ("lddmm_ctx_var_num", "lddmm_ctx_var_offset"):
        getattr(L, f).argtypes = [C.c_void_p, C.c_int]
        getattr(L, f).restype = C.c_longlong
    L.lddmm_ctx_var_total.argtypes = [C.c_void_p]
    L.lddmm_ctx_var_total.restype = C.c_longlong
    L.lddmm_ctx_stream.argtypes = [C.c_void_p]
    L.lddmm_ctx_stream.restype = C.c_void_p
    L.lddmm_ctx_launch_config.argtypes = [C.c_void_p, _ip]
    L.lddmm_ctx_launch_shape.argtypes = [C.c_void_p, _ip, C.c_int]
    L.lddmm_objgrd.argtypes = [C.c_void_p, _dp, _dp, _dp]
    L.lddmm_objgrd_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.lddmm_objgrd_costate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
    L.lddmm_lbfgs.argtypes = [C.c_void_p, C.POINTER(Opt), _dp, C.POINTER(Result)]
    L.lddmm_lbfgs_device.argtypes = [C.c_void_p, C.POINTER(Opt), C.c_void_p, C.POINTER(Result)]
    L.lddmm_lbfgs_trace.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int]
    L.lddmm_lbfgs_grad.argtypes = [C.c_void_p, _dp]
    L.lddmm_shoot.argtypes = [C.c_void_p, _dp, _dp, _dp]
    L.lddmm_LDDMM.argtypes = [C.c_int] * 5 + [_dp, _dp, _ip, _ip, _dp, _dp, _dp, C.c_char,
                                               C.c_double, C.c_char, C.c_double, C.c_double,
                                               C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                               C.c_double, C.c_double, C.c_double, C.c_int,
                                               C.c_int, _dp]
    L.lddmm_elm_ifo.argtypes = [_ip, C.c_int, C.c_int, C.c_int, _ip]
    L.lddmm_multiply_kernel.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, C.c_double, _dp]
    L.lddmm_dq_kernel.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, C.c_int, C.c_double, _dp]
    L.lddmm_compute_kernel.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int,
                                       C.c_double, _dp]
    L.lddmm_multiply_kernel2.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, C.c_int,
                                         C.c_double, _dp]
    L.lddmm_dq_kernel2.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, _dp, C.c_int,
                                   C.c_double, _dp, _dp]
    L.lddmm_varifold.argtypes = [C.POINTER(Problem), _dp, _dp, _dp]
    L.lddmm_flops_per_pair.argtypes = [C.c_int, C.c_int, C.c_int, C.c_char, C.c_char]
    L.lddmm_flops_per_pair.restype = C.c_double
    L.lddmm_ctx_time_sweeps.argtypes = [C.c_void_p, C.c_int, _dp]
    L.lddmm_ctx_counters.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.c_int]
    L.lddmm_fp32_peak.argtypes = [C.c_int, _dp]
    L.lddmm_pipe_peaks.argtypes = [C.c_int, _dp]
    L.lddmm_spatial_order.argtypes = [_dp, C.c_int, C.POINTER(C.c_int)]
    L.lddmm_ctx_timeline.argtypes = [C.c_void_p, _dp]
    L.lddmm_wait_selftest.argtypes = [C.c_int, C.c_int, _dp]
    L.lddmm_multiply_kernel_noalloc.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                C.c_int, C.c_double, C.c_void_p, C.c_void_p]
    # learned warm start
    _fp = C.POINTER(C.c_float)
    L.lddmm_ws_create.argtypes = [C.c_int, _dp, C.c_int, C.c_int, C.c_int, C.c_double,
                                  C.c_ulonglong, C.c_void_p, C.POINTER(C.c_void_p)]
    L.lddmm_ws_create_ex.argtypes = [C.c_int, _dp, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_ulonglong, C.c_int, C.c_void_p,
                                     C.POINTER(C.c_void_p)]
    L.lddmm_ws_destroy.argtypes = [C.c_void_p]
    L.lddmm_ws_destroy.restype = None
    L.lddmm_ws_last_error.restype = C.c_char_p
    L.lddmm_ws_num_params.argtypes = [C.c_void_p]
    L.lddmm_ws_num_params.restype = C.c_longlong
    L.lddmm_ws_params.argtypes = [C.c_void_p, _fp, C.c_int]
    L.lddmm_ws_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, _fp, _dp]
    L.lddmm_ws_train_step.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                      C.c_double, _dp]
    L.lddmm_ws_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.lddmm_ws_neighbours.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.lddmm_ws_train_step_nbr.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_double, C.POINTER(C.c_double)]
    L.lddmm_ws_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_double,
                                    C.POINTER(C.c_float), C.POINTER(C.c_double)]
    L.lddmm_ws_gemm_bf16.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p, C.c_longlong,
                                     C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_longlong,
                                     C.c_void_p]
    return L


lib = _load()


def check(rc: int) -> int:
    """Raise LddmmError for negative return codes; pass line-search codes through."""
    if rc < 0:
        raise LddmmError(rc, lib.lddmm_last_error().decode(errors="replace"))
    return rc


def check_ws(rc: int) -> int:
    """check() for the warm-start entry points (their own error message)."""
    if rc < 0:
        raise LddmmError(rc, lib.lddmm_ws_last_error().decode(errors="replace"))
    return rc


def dptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)
