"""Two-landmark-set kernel sums and the dense kernel matrix on the GPU, through the C
ABI (lddmm_compute_kernel, lddmm_multiply_kernel2, lddmm_dq_kernel2), against the
reference's golden vectors (every kernel order, 2D and 3D, set sizes that are not
multiples of the 64-row tile) and, at sizes the oracle would take long on, through
size-independent identities with the one-set entry points.  FP32 pair terms with
compensated accumulation: 1e-5 relative (max-norm of the error over the max-norm of
the reference)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

TOL = 1e-5
ORDERS = [(-1, "g"), (0, "m0"), (1, "m1"), (2, "m2"), (3, "m3"), (4, "m4")]


def mrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module")
def api():
    from lddmm_b200 import api as A

    return A


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("order,tag", ORDERS)
def test_two_set_golden(api, dim, order, tag):
    z = golden(f"two_set_kernels_{dim}d")
    w = float(z["width"])
    assert mrel(api.computeKernel(z["qi"], z["qj"], order, w), z[f"K_{tag}"]) < TOL
    assert mrel(api.computeKernel(z["qi"], order, w), z[f"K1_{tag}"]) < TOL
    assert mrel(api.multiplyKernel(z["qi"], z["qj"], z["a"], order, w), z[f"v_{tag}"]) < TOL
    dqi, dqj = api.dqKernel(z["qi"], z["qj"], z["l"], z["r"], order, w)
    for got, key in ((dqi, f"dqi_{tag}"), (dqj, f"dqj_{tag}")):
        ref = z[key]
        if np.max(np.abs(ref)) == 0:
            assert np.max(np.abs(got)) == 0
        else:
            assert mrel(got, ref) < TOL


@pytest.mark.parametrize("dim,order", [(3, -1), (3, 1), (2, 3)])
def test_two_set_identities_large(api, dim, order):
    """3000 + 2200 points: with qj = qi the two-set forms equal the one-set ones
    (multiply2 = multiply, dqi + dqj = dq), and K2 applied to a equals multiply2."""
    rng = np.random.default_rng(40 + dim)
    q = rng.uniform(-1, 1, size=(3000, dim))
    a, l, r = (rng.normal(size=(3000, dim)) for _ in range(3))
    w = 0.35
    assert mrel(api.multiplyKernel(q, q, a, order, w), api.multiplyKernel(q, a, order, w)) < TOL
    dqi, dqj = api.dqKernel(q, q, l, r, order, w)
    assert mrel(dqi + dqj, api.dqKernel(q, l, r, order, w)) < TOL
    qj = rng.uniform(-1, 1, size=(2200, dim))
    aj = rng.normal(size=(2200, dim))
    K = api.computeKernel(q, qj, order, w)
    assert K.shape == (3000, 2200)
    assert mrel(api.multiplyKernel(q, qj, aj, order, w), K @ aj) < TOL


def test_two_set_single_points(api, oracle):
    """One point per set (a single 64-row tile, 63 padding rows on both sides)."""
    rng = np.random.default_rng(3)
    qi, qj = rng.uniform(-0.2, 0.2, size=(1, 3)), rng.uniform(-0.2, 0.2, size=(1, 3))
    a, l, r = (rng.normal(size=(1, 3)) for _ in range(3))
    assert mrel(api.computeKernel(qi, qj, 1, 0.5), oracle.compute_kernel2(qi, qj, 1, 0.5)) < TOL
    assert mrel(api.multiplyKernel(qi, qj, a, 1, 0.5),
                oracle.multiply_kernel2(qi, qj, a, 1, 0.5)) < TOL
    got = api.dqKernel(qi, qj, l, r, -1, 0.5)
    ref = oracle.dq_kernel2(qi, qj, l, r, -1, 0.5)
    assert mrel(got[0], ref[0]) < TOL and mrel(got[1], ref[1]) < TOL
