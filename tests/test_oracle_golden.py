"""The CPU oracle (FP64 C restatement) against golden vectors produced by the
reference's own C++ code (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import golden, problem_from, rel

ORDERS = [(-1, "g"), (0, "m0"), (1, "m1"), (2, "m2"), (3, "m3"), (4, "m4")]


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order,tag", ORDERS)
def test_kernels_vs_reference(oracle, dim, order, tag):
    z = golden(f"kernels_{dim}d")
    w = float(z["width"])
    v = oracle.multiply_kernel(z["q"], z["a"], order, w)
    dq = oracle.dq_kernel(z["q"], z["l"], z["a"], order, w)
    assert rel(v, z[f"v_{tag}"]) < 1e-13
    if np.linalg.norm(z[f"dq_{tag}"]) == 0:
        assert np.linalg.norm(dq) == 0  # Matern order 0: no gradient in the reference
    else:
        assert rel(dq, z[f"dq_{tag}"]) < 1e-13


def test_objgrd_circle2square(oracle):
    z = golden("circle2square_objgrd")
    P = problem_from(z)
    f, g = oracle.objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < 1e-10
    assert rel(g, z["g"]) < 1e-12


def test_objgrd_circle2square_example(oracle):
    """The reference's 2D example setting (2D Matern order 3 via p0 / p1, Cauchy)."""
    z = golden("circle2square_example")
    P = problem_from(z)
    f, g = oracle.objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < 1e-10
    assert rel(g, z["g"]) < 1e-9


def test_objgrd_sphere2cube_example(oracle):
    z = golden("sphere2cube_example")
    P = problem_from(z)
    f, g = oracle.objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < 1e-10
    assert rel(g, z["g"]) < 1e-12
    v, dq = oracle.varifold(P, P.ini_nde)
    assert abs(v - float(z["vfd"])) / abs(float(z["vfd"])) < 1e-10
    assert rel(dq, z["vfd_dq"]) < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_varifold_kernel_types(oracle, dim):
    z = golden(f"varifold_types_{dim}d")
    for ct in "GC":
        for dt in "BLOU":
            P = problem_from(z, cen_type=ct, dir_type=dt, cen_width=0.3, dir_width=0.8)
            v, dq = oracle.varifold(P, z["q"])
            assert abs(v - float(z[f"v_{ct}{dt}"])) <= 1e-10 * abs(float(z[f"v_{ct}{dt}"])) + 1e-14
            assert rel(dq, z[f"dq_{ct}{dt}"]) < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order,tag", ORDERS)
def test_objgrd_orders(oracle, dim, order, tag):
    z = golden(f"objgrd_orders_{dim}d")
    P = problem_from(z, knl_order=order)
    f, g = oracle.objgrd(P, z["alp"])
    assert abs(f - float(z[f"f_{tag}"])) / abs(float(z[f"f_{tag}"])) < 1e-10
    assert rel(g, z[f"g_{tag}"]) < 1e-11


def test_lbfgs_trace_circle2square(oracle):
    z = golden("circle2square_lbfgs")
    P = problem_from(z)
    itr, tol, w1, w2, m = z["opt"]
    r = oracle.lbfgs(P, np.zeros(P.var_num), itr_max=int(itr), tol=tol, wolfe1=w1, wolfe2=w2,
                     mem_num=int(m))
    assert r["ret"] == int(z["ret"])
    n = len(z["trace_f"])
    assert r["evals"] == n
    assert np.max(np.abs(r["trace_f"] - z["trace_f"]) / np.abs(z["trace_f"])) < 1e-10
    assert rel(r["x"], z["x"]) < 1e-8


def test_lbfgs_trace_sphere2cube_example(oracle):
    z = golden("sphere2cube_example")
    zl = golden("sphere2cube_example_lbfgs")
    P = problem_from(z)
    itr, tol, w1, w2, m = zl["opt"]
    r = oracle.lbfgs(P, np.zeros(P.var_num), itr_max=int(itr), tol=tol, wolfe1=w1, wolfe2=w2,
                     mem_num=int(m))
    assert r["ret"] == int(zl["ret"])
    assert r["evals"] == len(zl["trace_f"])
    assert np.max(np.abs(r["trace_f"] - zl["trace_f"]) / np.abs(zl["trace_f"])) < 1e-10
    assert rel(r["x"], zl["x"]) < 1e-8


def test_oracle_gradient_finite_differences(oracle):
    """The reference's discrete adjoint has no test of its own; check the oracle's
    gradient (identical to the reference's to 1e-12, above) by central differences."""
    from lddmm_b200 import problem

    P = problem.circle_to_square(n_src=40, n_tgt=48, time_num=4)
    rng = np.random.default_rng(1)
    alp = rng.normal(size=P.var_num) * 0.1
    f0, g = oracle.objgrd(P, alp)
    for k in rng.choice(P.var_num, size=8, replace=False):
        h = 1e-6
        e = np.zeros_like(alp)
        e[k] = h
        fp, _ = oracle.objgrd(P, alp + e)
        fm, _ = oracle.objgrd(P, alp - e)
        fd = (fp - fm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k]))


def test_bessel_functions(oracle):
    from scipy.special import k0, k1

    for x in [1e-10, 1e-3, 0.5, 1.0, 1.5, 7.0, 40.0, 300.0]:
        assert abs(oracle.p0(x) - x * x * k0(x)) <= 1e-14 * max(1.0, x * x * k0(x)) + 1e-300
        assert abs(oracle.p1(x) - x * k1(x)) <= 1e-14 * max(1.0, x * k1(x)) + 1e-300
    assert oracle.p0(1e-17) == 0.0 and oracle.p1(1e-17) == 1.0
    assert oracle.p0(701.0) == 0.0 and oracle.p1(701.0) == 0.0
