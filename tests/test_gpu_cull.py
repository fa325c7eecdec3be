"""The varifold sweep's distance culling (Gaussian centre kernel): blocks of 32
columns whose bounding box lies beyond the kernel's 2^-64 cut-off from a 64-row tile
are skipped.  On geometries where most blocks are skipped the objective, gradient and
varifold gradient still agree with the FP64 oracle (which evaluates every pair) within
the parity tolerance, and a non-finite centre is never skipped."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-5


def small_sigma_problem(sigma_w=0.03):
    from lddmm_b200 import problem

    return problem.sphere_to_cube(subdiv=3, cube_n=10, time_num=6, sigma_w=sigma_w)


@pytest.mark.parametrize("sigma_w", [0.02, 0.03])
def test_culled_objgrd_matches_oracle(oracle, sigma_w):
    from lddmm_b200 import api, culling

    P = small_sigma_problem(sigma_w)
    assert culling.varifold_kept_fraction(P) < 0.4  # most blocks are skipped
    alp = np.random.default_rng(11).normal(size=P.var_num) * 0.05
    f, g = api.objgrd(P, alp)
    fo, go = oracle.objgrd(P, alp)
    assert abs(f - fo) / abs(fo) < TOL
    assert rel(g, go) < TOL


def test_culled_varifold_far_target(oracle):
    """Target 20 units away: every deformed-target block is skipped, and the value is
    the deformed-deformed plus the target-target term alone."""
    from lddmm_b200 import api, culling

    P = small_sigma_problem()
    P.tgt_cen = P.tgt_cen + np.array([20.0, 0.0, 0.0])
    assert culling.varifold_kept_fraction(P) < 0.25
    q = P.ini_nde + np.random.default_rng(12).normal(size=P.ini_nde.shape) * 0.01
    v, dq = api.varifold(P, q)
    vo, dqo = oracle.varifold(P, q)
    assert abs(v - vo) < TOL * (abs(vo) + 1.0)
    assert rel(dq, dqo) < 2 * TOL


def test_nonfinite_target_centre_is_not_culled(oracle):
    """A NaN target centre turns every deformed element's varifold gradient into NaN
    in the all-pairs reference; its block's box covers all of space, so the culled
    sweep reaches the same (instead of skipping it for the rows far from its block)."""
    from lddmm_b200 import api

    P = small_sigma_problem()
    t = P.tgt_cen.copy()
    t[5, 0] = np.nan
    P.tgt_cen = t
    q = P.ini_nde
    v, dq = api.varifold(P, q)
    vo, dqo = oracle.varifold(P, q)
    assert not np.isfinite(vo) and not np.isfinite(v)
    assert not np.any(np.isfinite(dqo))  # the reference: every vertex
    assert not np.any(np.isfinite(dq))


def test_degenerate_element_is_not_culled(oracle):
    """A collapsed triangle (zero area, 0/0 normal) makes every pair with it NaN in the
    all-pairs reference; the culled sweep never skips its block."""
    from lddmm_b200 import api

    P = small_sigma_problem()
    q = P.ini_nde.copy()
    a, b = P.elm_vtx[7, 0], P.elm_vtx[7, 1]
    q[b] = q[a]
    v, dq = api.varifold(P, q)
    vo, dqo = oracle.varifold(P, q)
    assert not np.isfinite(vo) and not np.isfinite(v)
    assert not np.any(np.isfinite(dqo))
    assert not np.any(np.isfinite(dq))


def test_reordered_surface_matches_oracle(oracle):
    """A decimated, re-triangulated surface pair, whose deformed and target elements
    the context stores in Morton order (lddmm_spatial_order says so): objective and
    gradient against the FP64 oracle, which keeps the caller's order; the adjacency
    that gathers element gradients onto vertices goes through the permutation."""
    import ctypes as C

    from lddmm_b200 import _lib, api, problem

    P = problem.population(n_pairs=4, seed=5, n_min=600, n_max=1500, t_min=1000,
                           t_max=2500)[1]
    for cen in (P.ini_nde[P.elm_vtx].mean(axis=1), P.tgt_cen):
        cen = np.ascontiguousarray(cen, dtype=np.float64)
        perm = np.zeros(cen.shape[0], dtype=np.int32)
        assert _lib.lib.lddmm_spatial_order(cen.ctypes.data_as(C.POINTER(C.c_double)),
                                            cen.shape[0],
                                            perm.ctypes.data_as(C.POINTER(C.c_int))) == 1
    alp = np.random.default_rng(31).normal(size=P.var_num) * 0.05
    f, g = api.objgrd(P, alp)
    fo, go = oracle.objgrd(P, alp)
    assert abs(f - fo) / abs(fo) < TOL
    assert rel(g, go) < TOL
    v, dq = api.varifold(P, P.ini_nde)
    vo, dqo = oracle.varifold(P, P.ini_nde)
    assert abs(v - vo) < TOL * (abs(vo) + 1.0)
    assert rel(dq, dqo) < 2 * TOL
