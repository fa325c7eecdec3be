"""Host restatement of the varifold sweep's culling test (no GPU): which
(64-row tile, 32-column block) pairs survive the 2^-64 cut-off."""
import numpy as np

from lddmm_b200 import culling, problem


def test_wide_kernel_keeps_every_pair():
    P = problem.sphere_to_cube(subdiv=2, cube_n=6, time_num=3, sigma_w=10.0)
    assert culling.varifold_kept_fraction(P) == 1.0


def test_cauchy_kernel_has_no_culling():
    P = problem.sphere_to_cube(subdiv=2, cube_n=6, time_num=3)
    P.cen_type = "C"
    assert culling.varifold_kept_fraction(P) is None


def test_far_target_keeps_only_deformed_blocks():
    P = problem.sphere_to_cube(subdiv=2, cube_n=6, time_num=3, sigma_w=10.0)
    P.tgt_cen = P.tgt_cen + np.array([1e4, 0.0, 0.0])
    Ed, Et = P.elm_vtx.shape[0], P.tgt_cen.shape[0]
    pad = lambda n: -(-n // 64) * 64
    assert culling.varifold_kept_fraction(P) == pad(Ed) / (pad(Ed) + pad(Et))


def test_nonfinite_centre_widens_its_block():
    P = problem.sphere_to_cube(subdiv=2, cube_n=6, time_num=3, sigma_w=10.0)
    P.tgt_cen = P.tgt_cen + np.array([1e4, 0.0, 0.0])
    base = culling.varifold_kept_fraction(P)
    t = P.tgt_cen.copy()
    t[0, 1] = np.nan
    P.tgt_cen = t
    # the first target block now meets every row tile
    rows = -(-P.elm_vtx.shape[0] // 64)
    Ed, Et = P.elm_vtx.shape[0], P.tgt_cen.shape[0]
    pad = lambda n: -(-n // 64) * 64
    extra = rows * 64 * 32 / (pad(Ed) * (pad(Ed) + pad(Et)))
    assert abs(culling.varifold_kept_fraction(P) - (base + extra)) < 1e-12


def _lib_order(cen):
    import ctypes as C

    from lddmm_b200 import _lib

    cen = np.ascontiguousarray(cen, dtype=np.float64)
    perm = np.zeros(cen.shape[0], dtype=np.int32)
    rc = _lib.lib.lddmm_spatial_order(cen.ctypes.data_as(C.POINTER(C.c_double)), cen.shape[0],
                                      perm.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc in (0, 1)
    return rc, perm


def test_spatial_order_restatement_matches_library():
    """The host restatement of the element storage order (culling.spatial_order) makes
    the library's decision and permutation (lddmm_spatial_order, host code)."""
    sets = []
    for P in problem.population(n_pairs=6, seed=2, n_min=300, n_max=3000, t_min=500,
                                t_max=4000):
        sets += [P.ini_nde[P.elm_vtx].mean(axis=1), P.tgt_cen]
    P = problem.sphere_to_cube(subdiv=3, cube_n=12, time_num=3)
    sets += [P.ini_nde[P.elm_vtx].mean(axis=1), P.tgt_cen]
    decisions = set()
    for cen in sets:
        rc, perm = _lib_order(cen)
        mine = culling.spatial_order(cen)
        decisions.add(rc)
        if rc == 0:
            assert mine is None and np.array_equal(perm, np.arange(cen.shape[0]))
        else:
            assert mine is not None and np.array_equal(perm, mine)
    assert decisions == {0, 1}  # both outcomes are exercised
