"""Host-side checks that need no GPU: the C ABI library loads and exports every
declared symbol, the adjacency table matches getElmIfo.m's semantics, workload
generators produce the documented sizes, and a compute call without a GPU fails
loudly instead of falling back to the CPU."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "lddmm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lddmm_\w+)\s*\(", src)))


def test_library_exports_every_declared_function():
    from lddmm_b200 import _lib

    declared = header_functions()
    assert declared, "no declarations parsed"
    assert sorted(_lib.EXPORTS) == declared
    for name in declared:
        assert hasattr(_lib.lib, name), name


def test_library_is_sm100a_build():
    from lddmm_b200 import _lib

    assert b"sm_100a" in _lib.lib.lddmm_version()


def test_compute_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lddmm_b200 import api, problem
    from lddmm_b200._lib import LddmmError

    P = problem.circle_to_square(n_src=16, n_tgt=16, time_num=3)
    with pytest.raises(LddmmError):
        api.objgrd(P, np.zeros(P.var_num))


@pytest.mark.parametrize("dim", [2, 3])
def test_elm_ifo_c_python_oracle_agree(oracle, dim):
    from lddmm_b200 import api, problem

    P = problem.sphere_to_cube(subdiv=2, cube_n=3) if dim == 3 else problem.circle_to_square(37, 40)
    py = problem.elm_ifo(P.elm_vtx, P.nde_num)
    orc = oracle.elm_ifo(P.elm_vtx, P.nde_num)
    c = api.getElmIfo(P.elm_vtx.T + 1, P.nde_num).T
    assert np.array_equal(py, orc)
    assert np.array_equal(py, c)


def test_elm_ifo_semantics_small():
    """Two triangles sharing an edge: hand-checked against getElmIfo.m:25-53."""
    from lddmm_b200 import problem

    ev = np.array([[0, 1, 2], [2, 1, 3]], dtype=np.int32)
    t = problem.elm_ifo(ev, 4)
    # vertex 1: in element 0 as local 2 -> (0, v0, v2); in element 1 as local 2 -> (1, v2, v3)
    assert list(t[1][:7]) == [2, 0, 0, 2, 1, 2, 3]
    # vertex 3: element 1 as local 3 -> (1, v1, v2)
    assert list(t[3][:4]) == [1, 1, 1, 2]
    ev2 = np.array([[0, 1], [1, 2], [2, 0]], dtype=np.int32)
    t2 = problem.elm_ifo(ev2, 3)
    assert list(t2[1]) == [2, 0, 1, 1, -1]


def test_workload_sizes():
    from lddmm_b200 import problem

    c1 = problem.circle_to_square()
    assert (c1.nde_num, c1.dfm_elm_num, c1.tgt_elm_num, c1.T) == (200, 200, 256, 20)
    assert c1.var_num == 8000
    c2 = problem.sphere_to_cube()
    assert (c2.nde_num, c2.dfm_elm_num, c2.tgt_elm_num, c2.T) == (2562, 5120, 12288, 20)
    assert c2.var_num == 153720
    assert c2.knl_order == 1 and c2.knl_width == 0.4 and c2.cen_width == 0.15
    pp = c2.pairs_per_eval()
    assert pp["shoot"] == 20 * 2562 ** 2
    assert pp["varifold"] == 5120 ** 2 + 5120 * 12288


def test_star_surface_and_population_sizes():
    from lddmm_b200 import problem, shapes

    V, F = shapes.star_surface(3, 8, 0.05, 0)
    assert V.shape == (642, 3) and F.shape == (1280, 3)
    cen, n, a = shapes.varifold_of(V, F)
    assert np.all(a > 0)
    assert np.all(np.einsum("ij,ij->i", cen, n) > 0)  # outward
    pop = problem.population(n_pairs=3, seed=1, n_min=100, n_max=400, t_min=200, t_max=600)
    for P in pop:
        assert 100 <= P.nde_num <= 400
        assert P.T == 10
        assert np.all(P.tgt_vol > 0)


def test_elm_ifo_matches_the_element_loop():
    """The vectorised getElmIfo table equals a direct loop over the elements
    (Cpp/src/getElmIfo.m:1-59 semantics) on a 3D mesh and a 2D polyline."""
    from lddmm_b200 import problem, shapes

    def loop(ev, n):
        E, V = ev.shape
        cnt = np.bincount(ev.ravel(), minlength=n)
        out = np.zeros((n, 1 + int(cnt.max()) * V), dtype=np.int32)
        fill = np.zeros(n, dtype=np.int64)
        other = {0: (2, 1), 1: (0, 2), 2: (1, 0)}
        for e in range(E):
            for k in range(V):
                v = ev[e, k]
                a = fill[v]
                fill[v] += 1
                if V == 2:
                    out[v, 1 + 2 * a], out[v, 2 + 2 * a] = e, (-1 if k == 0 else 1)
                else:
                    out[v, 1 + 3 * a] = e
                    out[v, 2 + 3 * a] = ev[e, other[k][0]]
                    out[v, 3 + 3 * a] = ev[e, other[k][1]]
        out[:, 0] = fill
        return out

    V, F = shapes.decimated_star(700, 6, 0.05, 3)
    assert np.array_equal(problem.elm_ifo(F, V.shape[0]), loop(F, V.shape[0]))
    cv, ce = shapes.circle(50)
    assert np.array_equal(problem.elm_ifo(ce, 50), loop(ce, 50))


def test_population_workers_build_the_same_pairs():
    from lddmm_b200 import problem

    a = problem.population(n_pairs=3, seed=4, n_max=2000, t_max=3000)
    b = problem.population(n_pairs=3, seed=4, n_max=2000, t_max=3000, workers=2)
    for x, y in zip(a, b):
        assert np.array_equal(x.ini_nde, y.ini_nde) and np.array_equal(x.elm_vtx, y.elm_vtx)
        assert np.array_equal(x.tgt_cen, y.tgt_cen) and np.array_equal(x.elm_ifo, y.elm_ifo)


def test_warm_start_learning_rate_schedule():
    """Constant without lr_final; with it a half cosine from lr to lr_final, halfway at
    the middle step, monotone."""
    from lddmm_b200.warmstart import lr_at

    assert lr_at(0, 100, 1e-3) == lr_at(99, 100, 1e-3) == 1e-3
    assert lr_at(0, 100, 1e-3, 1e-5) == pytest.approx(1e-3)
    assert lr_at(100, 100, 1e-3, 1e-5) == pytest.approx(1e-5)
    assert lr_at(50, 100, 1e-3, 1e-5) == pytest.approx(0.5 * (1e-3 + 1e-5))
    seq = [lr_at(k, 100, 1e-3, 1e-5) for k in range(101)]
    assert all(a >= b for a, b in zip(seq, seq[1:]))
