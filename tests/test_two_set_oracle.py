"""Two-landmark-set kernels and the dense kernel matrix (the reference's overloads
Cpp/src/computeKernel.cpp:21 / :246, multiplyKernel.cpp:294, dqKernel.cpp:307): the
oracle against the reference's own outputs (tests/golden/two_set_kernels_{2,3}d.npz,
made by tests/golden/make_golden.py from the compiled reference), the identities
that tie the two-set forms to the one-set ones, and the host-side argument checks of
the C ABI (no GPU work is started for rejected arguments)."""
import numpy as np
import pytest

from conftest import golden

ORDERS = [(-1, "g"), (0, "m0"), (1, "m1"), (2, "m2"), (3, "m3"), (4, "m4")]


def mrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order,tag", ORDERS)
def test_oracle_two_set_golden(oracle, dim, order, tag):
    z = golden(f"two_set_kernels_{dim}d")
    w = float(z["width"])
    assert mrel(oracle.compute_kernel2(z["qi"], z["qj"], order, w), z[f"K_{tag}"]) < 1e-13
    assert mrel(oracle.compute_kernel(z["qi"], order, w), z[f"K1_{tag}"]) < 1e-13
    assert mrel(oracle.multiply_kernel2(z["qi"], z["qj"], z["a"], order, w), z[f"v_{tag}"]) < 1e-13
    dqi, dqj = oracle.dq_kernel2(z["qi"], z["qj"], z["l"], z["r"], order, w)
    for got, key in ((dqi, f"dqi_{tag}"), (dqj, f"dqj_{tag}")):
        ref = z[key]
        if np.max(np.abs(ref)) == 0:  # Matern order 0: no gradient in the reference
            assert np.max(np.abs(got)) == 0
        else:
            assert mrel(got, ref) < 1e-13


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order", [-1, 1, 3])
def test_oracle_two_set_reduces_to_one_set(oracle, dim, order):
    """With qj = qi: K2 = K, multiply2 = multiply, dqi(l, r) + dqj(l, r) = dq(l, r)."""
    rng = np.random.default_rng(5 + dim)
    q = rng.uniform(-1, 1, size=(40, dim))
    a, l, r = (rng.normal(size=(40, dim)) for _ in range(3))
    w = 0.45
    assert mrel(oracle.compute_kernel2(q, q, order, w), oracle.compute_kernel(q, order, w)) < 1e-14
    assert mrel(oracle.multiply_kernel2(q, q, a, order, w),
                oracle.multiply_kernel(q, a, order, w)) < 1e-13
    dqi, dqj = oracle.dq_kernel2(q, q, l, r, order, w)
    assert mrel(dqi + dqj, oracle.dq_kernel(q, l, r, order, w)) < 1e-12


def test_two_set_argument_checks():
    from lddmm_b200 import api
    from lddmm_b200._lib import LddmmError

    q = np.zeros((4, 3))
    with pytest.raises(TypeError):
        api.multiplyKernel(q, q, q, q, -1, 0.5)
    with pytest.raises(TypeError):
        api.dqKernel(q, 0.5)
    with pytest.raises(TypeError):
        api.computeKernel(q)
    with pytest.raises(LddmmError, match="UNSUPPORTED"):
        api.multiplyKernel(q, q, q, 7, 0.5)
    with pytest.raises(LddmmError, match="ARG"):
        api.dqKernel(q, q, q, q, -1, 0.0)
    with pytest.raises(LddmmError, match="ARG"):
        api.computeKernel(np.zeros((0, 3)), -1, 0.5)
    with pytest.raises(LddmmError, match="ARG"):
        api.computeKernel(np.zeros((4, 4)), -1, 0.5)
