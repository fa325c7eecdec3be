"""Device-resident L-BFGS against the reference's optimiser (golden traces from the
compiled reference and the oracle's restatement)."""
import numpy as np
import pytest

from conftest import golden, problem_from, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def api():
    from lddmm_b200 import api as A

    return A


def early_trace_check(tr, ref_trace_f, n_iter):
    """Per-iteration objective of the device L-BFGS against the reference's per-
    evaluation trace: iteration k was accepted at evaluation 1 + sum of the line-search
    evaluations of iterations 1..k (tr[k, 3]).  The FP32 objective perturbs the path
    at the 1e-7 level, and L-BFGS amplifies that over tens of iterations, so the trace
    is pinned over the first iterations only."""
    assert abs(tr[0, 0] - ref_trace_f[0]) / abs(ref_trace_f[0]) < 1e-6
    ev = 0
    for k in range(1, n_iter + 1):
        ev += int(tr[k, 3])
        assert abs(tr[k, 0] - ref_trace_f[ev]) / abs(ref_trace_f[ev]) < 1e-5, k


def test_lbfgs_trace_circle2square(api):
    """Against the compiled reference's own L-BFGS trace (Cpp/src/LBFGS.cpp)."""
    z = golden("circle2square_lbfgs")
    P = problem_from(z)
    itr, tol, w1, w2, m = z["opt"]
    with api.Context(P) as ctx:
        x, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=int(itr), tol=tol, wolfe1=w1,
                           wolfe2=w2, mem_num=int(m))
        tr = ctx.trace(0)
    r = res[0]
    assert r["status"] == 0
    assert r["iters"] == int(itr)
    early_trace_check(tr, z["trace_f"], 10)
    # after 40 iterations both runs are well into the flat part of the descent
    assert abs(r["f"] - float(z["f"])) / abs(float(z["f"])) < 1e-2


def test_lbfgs_trace_sphere2cube_example(api):
    """The reference's own example data and options (Wolfe 0 / 0.5, memory 10)."""
    z = golden("sphere2cube_example")
    zl = golden("sphere2cube_example_lbfgs")
    P = problem_from(z)
    itr, tol, w1, w2, m = zl["opt"]
    with api.Context(P) as ctx:
        x, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=int(itr), tol=tol, wolfe1=w1,
                           wolfe2=w2, mem_num=int(m))
        tr = ctx.trace(0)
    assert res[0]["status"] == int(zl["ret"])
    early_trace_check(tr, zl["trace_f"], 8)


def test_lbfgs_trace_circle2square_example(api):
    """The reference's 2D example setting: 2D Matern order 3 (Bessel K form), Cauchy
    centre kernel, Wolfe 0 / 0.5, memory 10.  The objective falls 200-fold within six
    iterations here, so the FP32 path is pinned over the first five."""
    z = golden("circle2square_example")
    P = problem_from(z)
    itr, tol, w1, w2, m = z["opt"]
    with api.Context(P) as ctx:
        x, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=int(itr), tol=tol, wolfe1=w1,
                           wolfe2=w2, mem_num=int(m))
        tr = ctx.trace(0)
    assert res[0]["status"] == int(z["ret"])
    early_trace_check(tr, z["trace_f"], 5)


def test_lbfgs_batch_equals_individual(api):
    """Each pair of a batch runs its own optimiser state: with the same launch shape
    (per-step sweeps, one CTA per tile) it follows exactly the path it takes alone."""
    from lddmm_b200 import problem

    probs = [problem.circle_to_square(n_src=n, n_tgt=64, time_num=6) for n in (40, 100, 70)]
    x0 = [np.zeros(P.var_num) for P in probs]
    shape = dict(cluster=(1, 1, 1), persistent=-1)
    with api.Context(probs, **shape) as ctx:
        xb, rb = ctx.lbfgs(np.concatenate(x0), itr_max=25)
        xs = ctx.split(xb)
    for k, P in enumerate(probs):
        with api.Context(P, **shape) as c1:
            x1, r1 = c1.lbfgs(x0[k], itr_max=25)
        assert rb[k]["iters"] == r1[0]["iters"]
        assert rb[k]["evals"] == r1[0]["evals"]
        assert rb[k]["f"] == r1[0]["f"]
        assert np.array_equal(xs[k], x1)


def test_lbfgs_nonfinite_pair_fails_alone(api):
    """A pair whose starting objective is not finite stops with LDDMM_ERR_NONFINITE
    (-3); the other pairs of the batch run exactly as they would alone, and the call
    returns the first non-zero pair status, as LBFGS.cpp:92 reports a failure."""
    import ctypes as C

    from lddmm_b200 import _lib, problem

    probs = [problem.circle_to_square(n_src=n, n_tgt=64, time_num=6) for n in (40, 100)]
    shape = dict(cluster=(1, 1, 1), persistent=-1)
    with api.Context(probs, **shape) as ctx:
        x = np.zeros(ctx.var_total)
        x[0] = np.nan  # first variable of pair 0
        opt = _lib.Opt(25, 1e-6, 1e-4, 0.9, 5, 0, 0.0)
        res = (_lib.Result * 2)()
        rc = _lib.lib.lddmm_lbfgs(ctx.handle, C.byref(opt), _lib.dptr(x), res)
        xs = ctx.split(x)
    assert rc == -3
    assert res[0].status == -3 and res[0].iters == 0
    assert res[1].status == 0
    with api.Context(probs[1], **shape) as c1:
        x1, r1 = c1.lbfgs(np.zeros(probs[1].var_num), itr_max=25)
    assert res[1].iters == r1[0]["iters"] and res[1].fcn == r1[0]["f"]
    assert np.array_equal(xs[1], x1)
    # the Python API reports the failed pair in its status instead of raising
    with api.Context(probs, **shape) as ctx:
        x = np.zeros(ctx.var_total)
        x[0] = np.nan
        xp, rp = ctx.lbfgs(x, itr_max=25)
    assert [r["status"] for r in rp] == [-3, 0] and rp[1]["f"] == r1[0]["f"]


def test_lbfgs_grad_is_the_gradient_at_the_returned_point(api):
    """lddmm_lbfgs_grad returns the reference's grdNow: the gradient at the last
    accepted point, the same evaluation objgrd gives there."""
    from lddmm_b200 import problem

    P = problem.circle_to_square(n_src=64, n_tgt=64, time_num=6)
    with api.Context(P) as ctx:
        x, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=15)
        g = ctx.lbfgs_grad()
        f2, g2 = ctx.objgrd(x)
    assert np.isclose(np.linalg.norm(g), res[0]["glen"], rtol=1e-12)
    assert f2[0] == res[0]["f"] and np.array_equal(g, g2)


def test_lbfgs_graph_and_direct_launches_agree(api):
    from lddmm_b200 import problem

    P = problem.circle_to_square(n_src=64, n_tgt=64, time_num=6)
    with api.Context(P, use_graph=True) as c1:
        x1, r1 = c1.lbfgs(np.zeros(P.var_num), itr_max=20)
    with api.Context(P, use_graph=False) as c2:
        x2, r2 = c2.lbfgs(np.zeros(P.var_num), itr_max=20)
    assert r1[0]["f"] == r2[0]["f"] and np.array_equal(x1, x2)


_FP64_REG = {}


@pytest.mark.parametrize("persistent", [2, 1, -1])
def test_registration_matches_fp64_registration(api, oracle, persistent):
    """The north-star criterion on a 3D registration run to convergence (400
    iterations), with each form of the time-loop sweeps (cluster persistent, L2
    persistent, per-step launches; launch shape pinned): the FP32 path's objective is
    within 1e-5 relative of the FP64 registration's and its deformed landmarks within
    1e-4 of the shape diameter (RMS over landmarks).  Measured: 1.6e-6 and 5.7e-5.
    Near the optimum the two paths differ by FP32 noise, and the FP32 line search may
    stop a little earlier with the reference's code 3 (bracketed, not satisfied),
    already inside the tolerance."""
    from lddmm_b200 import problem

    P = problem.sphere_to_cube(subdiv=3, cube_n=12, time_num=11)
    x0 = np.zeros(P.var_num)
    if "ro" not in _FP64_REG:  # one FP64 registration for the three forms
        ro = oracle.lbfgs(P, x0, itr_max=400)
        nde_o, _ = oracle.shoot(P.ini_nde, ro["x"], P.knl_order, P.knl_width, P.time_stp,
                                P.time_num)
        _FP64_REG.update(ro=ro, nde_o=nde_o)
    ro, nde_o = _FP64_REG["ro"], _FP64_REG["nde_o"]
    with api.Context(P, autotune=False, persistent=persistent) as ctx:
        x, res = ctx.lbfgs(x0, itr_max=400)
        (nde, _), = ctx.shoot(x)
    assert ro["ret"] == 0 and res[0]["status"] in (0, 3)
    assert abs(res[0]["f"] - ro["f"]) / abs(ro["f"]) < 1e-5, (res[0]["f"], ro["f"])
    err = np.sqrt(np.mean(np.sum((nde[-1] - nde_o[-1]) ** 2, axis=1)))
    assert err < 1e-4 * P.diameter(), err / P.diameter()


def test_rel_obj_tol_stops_early(api):
    from lddmm_b200 import problem

    P = problem.circle_to_square(n_src=48, n_tgt=64, time_num=5)
    with api.Context(P) as ctx:
        _, r_full = ctx.lbfgs(np.zeros(P.var_num), itr_max=200, tol=0.0)
        _, r_rel = ctx.lbfgs(np.zeros(P.var_num), itr_max=200, tol=0.0, rel_obj_tol=1e-5)
    assert r_rel[0]["iters"] < r_full[0]["iters"] or r_full[0]["status"] != 0
    assert r_rel[0]["status"] == 0


def test_lddmm_matlab_interface(api):
    """LDDMM.m-level call on the circle -> square setting of the reference example
    (Cpp/examples/circle2square/run_circle2square.m), fewer points and iterations."""
    from lddmm_b200 import shapes

    n = 100
    ang = np.linspace(0, 2 * np.pi, n + 1)[:-1]
    ini = np.stack([np.cos(ang), np.sin(ang)])
    elm = np.stack([np.arange(1, n + 1), np.r_[np.arange(2, n + 1), 1]])
    tv, te = shapes.square_boundary(200, 0.8)
    cen, dr, vol = shapes.varifold_of(tv, te)
    dis = dict(dfmElmVtxMat=elm, tgtCenPosMat=cen.T, tgtElmVolVec=vol, tgtUniDirMat=dr.T,
               cenKnlType="C", cenKnlWidth=0.1, dirKnlType="B", dirKnlWidth=0, disWgt=100)
    opt = dict(MaxIterations=30, OptimalityTolerance=1e-2, Wolfe1=0, Wolfe2=0.5, Columns=10)
    out = api.LDDMM(ini, None, dis, -1, 0.25, 1.0, 0.05, opt)
    assert out.ndeStk.shape == (2, n, 21)
    assert out.vlcStk.shape == (2, n, 20)
    assert out.alpStk.shape == (2, n, 20)
    assert out.result["status"] in (0, 1, 2, 3)
    assert np.all(np.isfinite(out.ndeStk))


@pytest.mark.parametrize("persistent", [-1, 1, 2])
def test_uneven_3d_batch_objgrd_equals_individual(api, persistent):
    """Uneven 3D surface pairs (star surfaces of 600-2600 vertices onto targets of
    1000-4000 triangles, as in the 256-pair population) evaluated in one batched
    context: every pair's objective and gradient equal its own single-pair
    evaluation with the same launch shape (per-step sweeps with one CTA per tile, or
    the persistent sweeps in either form: split row groups combined through L2 (1) or
    by thread-block clusters through distributed shared memory (2)), so batching
    changes nothing but the launches."""
    from lddmm_b200 import problem

    probs = problem.population(n_pairs=4, seed=3, n_min=600, n_max=2600, t_min=1000,
                               t_max=4000)
    rng = np.random.default_rng(5)
    xs = [rng.normal(size=P.var_num) * 0.01 for P in probs]
    shape = dict(cluster=(1, 1, 1), persistent=persistent)
    with api.Context(probs, **shape) as ctx:
        fb, gb = ctx.objgrd(np.concatenate(xs))
        gbs = ctx.split(gb)
    for k, P in enumerate(probs):
        with api.Context(P, **shape) as c1:
            f1, g1 = c1.objgrd(xs[k])
        if persistent < 0:
            assert fb[k] == f1[0] and np.array_equal(gbs[k], g1)
        else:  # the persistent work plan cuts the batch's rows differently
            assert abs(fb[k] - f1[0]) <= 1e-6 * abs(f1[0])
            assert np.max(np.abs(gbs[k] - g1)) <= 1e-5 * np.max(np.abs(g1))
