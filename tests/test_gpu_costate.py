"""lddmm_objgrd_costate: the adjoint costate of the backward recursion
(Cpp/src/objgrd.cpp:67-87) alongside the objective and gradient, checked through the
identities that define it, with the library's own kernel sums and varifold:
  * the last step's costate is p_T = -w dD/dq (q_T), the weighted varifold gradient at
    the shot end positions;
  * every step's gradient is dt K(q_t) (alpha_t - p_{t+1});
and the objective and gradient are those of lddmm_objgrd_device (the same path)."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden, problem_from, rel

pytestmark = pytest.mark.gpu


def test_costate_identities():
    from lddmm_b200 import _lib, api

    P = problem_from(golden("sphere2cube_example"))
    rng = np.random.default_rng(11)
    alp = rng.normal(size=P.var_num) * 0.02
    T, N, D = P.time_num - 1, P.nde_num, P.dim
    with api.Context(P) as ctx:
        a = torch.from_numpy(alp).cuda()
        f, f2 = (torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(2))
        g, g2, p = (torch.zeros_like(a) for _ in range(3))
        _lib.check(_lib.lib.lddmm_objgrd_costate(ctx.handle, C.c_void_p(a.data_ptr()),
                                                 C.c_void_p(f.data_ptr()),
                                                 C.c_void_p(g.data_ptr()),
                                                 C.c_void_p(p.data_ptr())))
        _lib.check(_lib.lib.lddmm_objgrd_device(ctx.handle, C.c_void_p(a.data_ptr()),
                                                C.c_void_p(f2.data_ptr()),
                                                C.c_void_p(g2.data_ptr()), 0))
        (nde, _), = ctx.shoot(alp)
    assert torch.equal(f, f2) and torch.equal(g, g2)
    g = g.cpu().numpy().reshape(T, N, D)
    p = p.cpu().numpy().reshape(T, N, D)
    A = alp.reshape(T, N, D)
    _, dq = api.varifold(P, nde[T])
    e = rel(p[T - 1], -P.dis_wgt * dq)
    assert e < 1e-6, e
    for t in range(T):
        Ku = api.multiplyKernel(nde[t], A[t] - p[t], P.knl_order, P.knl_width)
        e = rel(g[t], P.time_stp * Ku)
        assert e < 1e-5, (t, e)
