"""The MEX-level drop-in, lddmm_LDDMM (Cpp/src/LDDMM.cpp:11-98), called through the C
ABI with the reference's own example options, Columns = 10000 included
(Cpp/examples/sphere2cube/run_sphere2cube.m:27-31).

The reference keeps a ring of memNum (s, y) pairs (Cpp/src/LBFGS.cpp:96-99) and
builds each direction from min(iteration - 1, memNum) of them
(Cpp/src/getDirection.cpp:9-66).  Here the ring has min(Columns, MaxIterations)
slots, which never wraps earlier than the reference's; beyond 32 slots the direction
runs on the long-memory phases of the device L-BFGS.  The fixture
sphere2cube_example_columns.npz is the compiled reference's own run at
Columns = 10000 (tests/golden/make_golden.py).
"""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import golden, problem_from

pytestmark = pytest.mark.gpu

_ROW = re.compile(r"^\s*(\d+):\s+(\S+)\s+(\S+)(?:\s+(\S+)\s+(\d+))?\s*$")


def _table(text):
    """Rows (f, |g|, step length, evaluations) of the reference's verbose iteration
    table (Cpp/src/LBFGS.cpp:54-61, 107-108) as lddmm_LDDMM prints it."""
    rows = []
    for line in text.splitlines():
        m = _ROW.match(line)
        if m:
            k = int(m.group(1))
            assert k == len(rows), line
            rows.append([float(m.group(2)), float(m.group(3)),
                         float(m.group(4) or 0.0), float(m.group(5) or 0)])
    return np.array(rows)


def _call_LDDMM(P, itr, tol, w1, w2, columns, verbose):
    from lddmm_b200 import _lib

    L = _lib.lib
    ini = np.ascontiguousarray(P.ini_nde)
    alp0 = np.zeros(P.var_num)
    out = np.full(P.var_num, np.nan)
    ifo = np.ascontiguousarray(P.elm_ifo)
    rc = L.lddmm_LDDMM(P.dim, P.nde_num, P.dfm_elm_num, ifo.shape[1], P.tgt_elm_num,
                       _lib.dptr(ini), _lib.dptr(alp0), _lib.iptr(P.elm_vtx), _lib.iptr(ifo),
                       _lib.dptr(P.tgt_cen), _lib.dptr(P.tgt_vol), _lib.dptr(P.tgt_dir),
                       P.cen_type.encode(), P.cen_width, P.dir_type.encode(), P.dir_width,
                       P.dis_wgt, P.knl_order, P.knl_width, P.time_stp, P.time_num, int(itr),
                       float(tol), float(w1), float(w2), int(columns), 1 if verbose else 0,
                       _lib.dptr(out))
    return rc, out


def _early_trace(tr, ref_trace_f, n_iter):
    """Iteration k was accepted at evaluation 1 + the line-search evaluations of
    iterations 1..k; the printed objective has 7 significant digits."""
    assert abs(tr[0, 0] - ref_trace_f[0]) / abs(ref_trace_f[0]) < 1e-6
    ev = 0
    for k in range(1, n_iter + 1):
        ev += int(tr[k, 3])
        assert abs(tr[k, 0] - ref_trace_f[ev]) / abs(ref_trace_f[ev]) < 1e-5, k


def test_LDDMM_with_the_reference_example_columns(capfd):
    z = golden("sphere2cube_example")
    zc = golden("sphere2cube_example_columns")
    P = problem_from(z)
    itr, tol, w1, w2, cols = zc["opt"]
    assert int(cols) == 10000
    capfd.readouterr()
    rc, x = _call_LDDMM(P, itr, tol, w1, w2, cols, verbose=True)
    out = capfd.readouterr().out
    assert rc == int(zc["ret"]), rc
    tr = _table(out)
    assert len(tr) == int(itr) + 1  # 40 iterations: the history grows past 32 pairs
    _early_trace(tr, zc["trace_f"], 8)
    # the objective after 40 iterations agrees with the reference's to the FP32
    # path's drift (the paths part after tens of iterations)
    assert abs(tr[-1, 0] - float(zc["f"])) / float(zc["f"]) < 1e-2
    assert np.all(np.isfinite(x))


def test_LDDMM_equals_lddmm_lbfgs_on_the_same_inputs():
    """optAlpVec of the MEX-level call is the momenta lddmm_lbfgs returns for the same
    problem and options (the same device path, bit for bit)."""
    from lddmm_b200 import api

    z = golden("sphere2cube_example")
    zc = golden("sphere2cube_example_columns")
    P = problem_from(z)
    itr, tol, w1, w2, cols = zc["opt"]
    rc, x = _call_LDDMM(P, itr, tol, w1, w2, cols, verbose=False)
    with api.Context(P) as ctx:
        x2, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=int(itr), tol=tol, wolfe1=w1,
                            wolfe2=w2, mem_num=int(cols))
    assert rc == res[0]["status"]
    assert np.array_equal(x, x2)


def test_long_memory_matches_compact_solve_while_both_apply():
    """Up to 32 pairs of history the long-memory phases (explicit R^-1, grid-wide
    products) and the one-thread compact solve compute the same direction up to
    rounding: with memory 40 and 32 the first 32 iterations build identical histories,
    so the traces agree to rounding over them."""
    from lddmm_b200 import api, problem

    P = problem.circle_to_square(n_src=120, n_tgt=128, time_num=11)
    runs = []
    for mem in (32, 40):
        with api.Context(P) as ctx:
            x, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=32, mem_num=mem)
            runs.append((ctx.trace(0), res[0]))
    (t32, r32), (t40, r40) = runs
    assert r32["iters"] == r40["iters"] == 32
    rel = np.abs(t32[:, 0] - t40[:, 0]) / np.abs(t32[:, 0])
    assert rel.max() < 1e-6, rel.max()


def test_memory_beyond_the_device_is_refused_cleanly():
    """A ring that cannot fit in device memory is an LDDMM_ERR_NOMEM with a message,
    before anything is allocated (the reference would fail its calloc)."""
    from lddmm_b200 import _lib, api, problem

    P = problem.sphere_to_cube(subdiv=6, cube_n=8, time_num=21)  # 2.5 M variables
    with api.Context(P) as ctx:
        opt = _lib.Opt(100000, 1e-6, 1e-4, 0.9, 100000, 0, 0.0)  # 100000 pairs: 4 TB
        res = (_lib.Result * 1)()
        x = np.zeros(ctx.var_total)
        rc = _lib.lib.lddmm_lbfgs(ctx.handle, C.byref(opt), _lib.dptr(x), res)
        assert rc == -5, rc  # LDDMM_ERR_NOMEM
        assert b"memory" in _lib.lib.lddmm_last_error()
        # the context stays usable
        x, r = ctx.lbfgs(np.zeros(ctx.var_total), itr_max=2, mem_num=5)
        assert r[0]["iters"] == 2


def test_LDDMM_runs_the_reference_example_to_its_end():
    """The reference's example exactly as it calls the MEX (MaxIterations 100000,
    OptimalityTolerance 1e-2, Wolfe 0 / 0.5, Columns 10000), through lddmm_LDDMM,
    run until the |g| test stops it (the reference: 139 evaluations; here ~101
    iterations): the returned momenta's objective within 1e-5 relative of the
    reference's final objective and the deformed landmarks within 1e-4 of the shape
    diameter of the reference's (tests/golden/make_golden.py
    sphere2cube_example_full)."""
    from lddmm_b200 import api

    z = golden("sphere2cube_example")
    zf = golden("sphere2cube_example_full")
    P = problem_from(z)
    itr, tol, w1, w2, cols = zf["opt"]
    rc, x = _call_LDDMM(P, itr, tol, w1, w2, cols, verbose=False)
    assert rc == int(zf["ret"]) == 0
    with api.Context(P) as ctx:
        f, _ = ctx.objgrd(x)
        (nde, _), = ctx.shoot(x)
    rel_f = abs(f[0] - float(zf["f"])) / abs(float(zf["f"]))
    err = np.sqrt(np.mean(np.sum((nde[-1] - zf["nde_final"]) ** 2, axis=1))) / P.diameter()
    print(f"f {f[0]:.9g} vs reference {float(zf['f']):.9g} (rel {rel_f:.1e}); landmarks "
          f"RMS {err:.1e} of the diameter")
    assert rel_f < 1e-5, rel_f
    assert err < 1e-4, err
