"""CUDA path (through the C ABI) against the reference's golden vectors and the
CPU oracle.  FP32 kernels with compensated accumulation: objective and gradient
within 1e-5 relative of the FP64 reference, per-kernel sums within 1e-5 relative
(max-norm of the error over the max-norm of the reference)."""
import numpy as np
import pytest

from conftest import golden, problem_from, rel

pytestmark = pytest.mark.gpu

TOL = 1e-5  # FP32 + compensated accumulation vs FP64 reference
ORDERS3 = [(-1, "g"), (0, "m0"), (1, "m1"), (2, "m2"), (3, "m3"), (4, "m4")]


def mrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def api():
    from lddmm_b200 import api as A

    return A


@pytest.mark.parametrize("order,tag", ORDERS3)
def test_multiply_kernel_3d(api, order, tag):
    z = golden("kernels_3d")
    v = api.multiplyKernel(z["q"], z["a"], order, float(z["width"]))
    assert mrel(v, z[f"v_{tag}"]) < TOL


@pytest.mark.parametrize("order,tag", ORDERS3)
def test_dq_kernel_3d(api, order, tag):
    z = golden("kernels_3d")
    dq = api.dqKernel(z["q"], z["l"], z["a"], order, float(z["width"]))
    ref = z[f"dq_{tag}"]
    if np.max(np.abs(ref)) == 0:
        assert np.max(np.abs(dq)) == 0
    else:
        assert mrel(dq, ref) < TOL


@pytest.mark.parametrize("order,tag", ORDERS3)
def test_kernels_2d(api, order, tag):
    """2D: Gaussian and the Bessel-K Matern family (p0 = x^2 K0, p1 = x K1) of every
    order; the order-0 dq sum is zero like the reference's."""
    z = golden("kernels_2d")
    v = api.multiplyKernel(z["q"], z["a"], order, float(z["width"]))
    dq = api.dqKernel(z["q"], z["l"], z["a"], order, float(z["width"]))
    assert mrel(v, z[f"v_{tag}"]) < TOL
    ref = z[f"dq_{tag}"]
    if np.max(np.abs(ref)) == 0:
        assert np.max(np.abs(dq)) == 0
    else:
        assert mrel(dq, ref) < TOL


@pytest.mark.parametrize("dim", [2, 3])
def test_varifold_kernel_types(api, dim):
    z = golden(f"varifold_types_{dim}d")
    for ct in "GC":
        for dt in "BLOU":
            P = problem_from(z, cen_type=ct, dir_type=dt, cen_width=0.3, dir_width=0.8,
                             knl_order=-1)
            v, dq = api.varifold(P, z["q"])
            ref_v, ref_dq = float(z[f"v_{ct}{dt}"]), z[f"dq_{ct}{dt}"]
            # the value is a difference of O(1) sums; compare at the scale of the terms
            scale = abs(ref_v) + 1.0
            assert abs(v - ref_v) < TOL * scale, (ct, dt, v, ref_v)
            assert mrel(dq, ref_dq) < 2 * TOL, (ct, dt)


def test_objgrd_circle2square_golden(api):
    z = golden("circle2square_objgrd")
    P = problem_from(z)
    f, g = api.objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < TOL
    assert rel(g, z["g"]) < TOL


def test_objgrd_circle2square_example_golden(api):
    """The reference's 2D example setting (2D Matern order 3, Cauchy centres)."""
    z = golden("circle2square_example")
    P = problem_from(z)
    f, g = api.objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < TOL
    assert rel(g, z["g"]) < TOL


def test_objgrd_sphere2cube_example_golden(api):
    """The reference's own example data (sphereData.mat / cubeData.mat, Cauchy centre
    kernel, Matern order 3, disWgt 100)."""
    z = golden("sphere2cube_example")
    P = problem_from(z)
    f, g = api.objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < TOL
    assert rel(g, z["g"]) < TOL


@pytest.mark.parametrize("order,tag", ORDERS3)
def test_objgrd_orders_3d_golden(api, order, tag):
    z = golden("objgrd_orders_3d")
    P = problem_from(z, knl_order=order)
    f, g = api.objgrd(P, z["alp"])
    assert abs(f - float(z[f"f_{tag}"])) / abs(float(z[f"f_{tag}"])) < TOL
    assert rel(g, z[f"g_{tag}"]) < TOL


@pytest.mark.parametrize("order,tag", ORDERS3)
def test_objgrd_2d_golden(api, order, tag):
    z = golden("objgrd_orders_2d")
    P = problem_from(z, knl_order=order)
    f, g = api.objgrd(P, z["alp"])
    assert abs(f - float(z[f"f_{tag}"])) / abs(float(z[f"f_{tag}"])) < TOL
    assert rel(g, z[f"g_{tag}"]) < TOL


def test_objgrd_sphere2cube_full_size_vs_oracle(api, oracle):
    """Full benchmark size (2562 vertices, 5120 / 12288 triangles, T = 20) against
    the FP64 oracle at a non-trivial momentum field."""
    from lddmm_b200 import problem

    P = problem.sphere_to_cube()
    rng = np.random.default_rng(2)
    alp = rng.normal(size=P.var_num) * 0.01
    f, g = api.objgrd(P, alp)
    fo, go = oracle.objgrd(P, alp)
    assert abs(f - fo) / abs(fo) < TOL
    assert rel(g, go) < TOL


def test_batch_equals_individual(api):
    """A batch of uneven pairs gives every pair what it gets alone (to FP32 rounding:
    the launch shape, and so the summation order, depends on the batch)."""
    from lddmm_b200 import problem

    probs = [problem.sphere_to_cube(subdiv=s, cube_n=c, time_num=5)
             for s, c in ((1, 3), (3, 8), (2, 5))]
    rng = np.random.default_rng(3)
    alps = [rng.normal(size=P.var_num) * 0.05 for P in probs]
    with api.Context(probs) as ctx:
        f, g = ctx.objgrd(np.concatenate(alps))
        gs = ctx.split(g)
    for k, P in enumerate(probs):
        with api.Context(P) as c1:
            f1, g1 = c1.objgrd(alps[k])
        assert abs(f[k] - f1[0]) <= 1e-7 * abs(f1[0])
        assert rel(gs[k], g1) < 1e-6


def test_deterministic(api):
    from lddmm_b200 import problem

    P = problem.sphere_to_cube(subdiv=3, cube_n=10, time_num=6)
    alp = np.random.default_rng(4).normal(size=P.var_num) * 0.05
    with api.Context(P) as ctx:
        f1, g1 = ctx.objgrd(alp)
        f2, g2 = ctx.objgrd(alp)
    assert f1[0] == f2[0]
    assert np.array_equal(g1, g2)


@pytest.mark.parametrize("S", [1, 2, 4, 8])
def test_cluster_sizes_agree(api, oracle, S):
    from lddmm_b200 import problem

    P = problem.sphere_to_cube(subdiv=3, cube_n=10, time_num=6)
    alp = np.random.default_rng(5).normal(size=P.var_num) * 0.05
    with api.Context(P, cluster=(S, S, S)) as ctx:
        f, g = ctx.objgrd(alp)
    fo, go = oracle.objgrd(P, alp)
    assert abs(f[0] - fo) / abs(fo) < TOL
    assert rel(g, go) < TOL


def test_gradient_finite_differences(api):
    """Directional derivative of the GPU objective against its gradient.  The step is
    large enough that FP32 objective noise (~1e-7 |f| / h) stays below the tolerance;
    the exact gradient check is the parity with the FP64 oracle above."""
    from lddmm_b200 import problem

    P = problem.sphere_to_cube(subdiv=2, cube_n=6, time_num=5)
    rng = np.random.default_rng(6)
    alp = rng.normal(size=P.var_num) * 0.05
    d = rng.normal(size=P.var_num)
    d /= np.linalg.norm(d)
    with api.Context(P) as ctx:
        _, g = ctx.objgrd(alp)
        h = 2e-2
        fp, _ = ctx.objgrd(alp + h * d)
        fm, _ = ctx.objgrd(alp - h * d)
    fd = (fp[0] - fm[0]) / (2 * h)
    assert abs(fd - g @ d) <= 2e-3 * max(abs(g @ d), 1e-3)


def test_shoot_trajectory(api, oracle):
    from lddmm_b200 import problem

    P = problem.sphere_to_cube(subdiv=3, cube_n=4, time_num=6)
    alp = np.random.default_rng(7).normal(size=P.var_num) * 0.1
    with api.Context(P) as ctx:
        (nde, vlc), = ctx.shoot(alp)
    nde_o, vlc_o = oracle.shoot(P.ini_nde, alp, P.knl_order, P.knl_width, P.time_stp,
                                P.time_num)
    assert mrel(nde, nde_o) < TOL
    assert mrel(vlc, vlc_o) < TOL


def test_two_tile_gaussian_shoot_odd_tiles_vs_oracle(api, oracle):
    """Per-step sweeps with the Gaussian kernel: the shooting sweep runs on two-tile
    items, and 642 landmarks give 11 tiles, so the last item holds one tile only.
    Objective and gradient against the FP64 oracle, and the persistent time-loop
    sweeps (single tiles) within the same tolerance."""
    from lddmm_b200 import problem

    P = problem.sphere_to_cube(subdiv=3, cube_n=10, time_num=6, knl_order=-1, knl_width=0.3)
    assert (-(-P.nde_num // 64)) % 2 == 1
    alp = np.random.default_rng(21).normal(size=P.var_num) * 0.05
    with api.Context(P, persistent=-1) as ctx:
        f, g = ctx.objgrd(alp)
    with api.Context(P, persistent=1) as ctx:
        f1, g1 = ctx.objgrd(alp)
    fo, go = oracle.objgrd(P, alp)
    assert abs(f[0] - fo) / abs(fo) < TOL
    assert rel(g, go) < TOL
    assert abs(f1[0] - fo) / abs(fo) < TOL
    assert rel(g1, go) < TOL
