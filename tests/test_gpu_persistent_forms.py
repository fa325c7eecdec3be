"""The three launch forms of the time loops give the same objective and gradient:
per-step sweeps (persistent=-1), the persistent sweeps whose split row groups meet in
L2 (persistent=1), and the cluster form (persistent=2), where each thread-block
cluster owns whole row groups and combines their parts in distributed shared memory.
Checked on the full sphere -> cube workload (2562 landmarks, Matern nu = 3/2, T = 20)
and on the 2D circle -> square workload against the FP64 oracle, for run-to-run
bitwise determinism, and through a short L-BFGS run."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _objgrd(P, alp, persistent):
    from lddmm_b200 import api

    with api.Context(P, persistent=persistent) as ctx:
        shape = ctx.launch_shape()
        f, g = ctx.objgrd(alp)
        f2, g2 = ctx.objgrd(alp)
    assert f2[0] == f[0] and np.array_equal(g, g2)  # bit-reproducible
    return f[0], g, shape


@pytest.mark.parametrize("which", ["sphere2cube", "circle2square"])
def test_forms_agree_with_the_oracle(oracle, which):
    from lddmm_b200 import problem

    P = problem.sphere_to_cube() if which == "sphere2cube" else problem.circle_to_square()
    alp = np.random.default_rng(3).normal(size=P.var_num) * 0.02
    fo, go = oracle.objgrd(P, alp)
    out = {}
    for form in (-1, 1, 2):
        f, g, shape = _objgrd(P, alp, form)
        assert shape["persistent"] == max(form, 0), (form, shape)
        assert abs(f - fo) / abs(fo) < TOL, (form, f, fo)
        assert rel(g, go) < TOL, (form, rel(g, go))
        out[form] = (f, g)
    # the forms cut the rows' j ranges at different points, so their FP32 partial sums
    # differ at the FP32 rounding level only
    for form in (1, 2):
        assert abs(out[form][0] - out[-1][0]) <= 1e-7 * abs(out[-1][0])
        assert rel(out[form][1], out[-1][1]) < 1e-6


def test_cluster_form_lbfgs_follows_the_l2_form():
    """The first 8 iterations of the two persistent forms' L-BFGS runs agree."""
    from lddmm_b200 import api, problem

    P = problem.sphere_to_cube(subdiv=3, cube_n=12, time_num=11)
    traces = []
    for form in (1, 2):
        with api.Context(P, persistent=form) as ctx:
            x, res = ctx.lbfgs(np.zeros(P.var_num), itr_max=15)
            traces.append(ctx.trace(0))
            assert res[0]["status"] == 0 and res[0]["iters"] == 15
    # the same early path (rounding-level differences grow over the iterations, as
    # between any two launch shapes)
    r = np.abs(traces[0][:9, 0] - traces[1][:9, 0]) / np.abs(traces[0][:9, 0])
    assert r.max() < 1e-5, r.max()
