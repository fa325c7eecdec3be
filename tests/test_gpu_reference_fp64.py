"""The reference's own plain FP64 GPU path (CUDA/src, compiled in place by
``make -C oracle refcu``) as a second pin: it must agree with the reference's C++
path (the golden fixtures) to FP64 rounding, and the FP32 + compensated CUDA path of
this project must agree with it within 1e-5 relative, like it does with the C++
path.  Skipped when the FP64 GPU library has not been built."""
import numpy as np
import pytest

from conftest import golden, problem_from, rel

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9  # two FP64 implementations, different summation orders
TOL = 1e-5       # FP32 kernels with compensated accumulation vs FP64


def _refcu(dim):
    from oracle.oracle import ReferenceCuda

    if not ReferenceCuda.available(dim):
        pytest.skip("oracle/_ref/librefcu*.so not built (make -C oracle refcu)")
    return ReferenceCuda(dim)


@pytest.mark.parametrize("name", ["circle2square_objgrd", "sphere2cube_example"])
def test_fp64_gpu_reference_matches_cpp_reference(name):
    z = golden(name)
    P = problem_from(z)
    f, g = _refcu(P.dim).objgrd(P, z["alp"])
    assert abs(f - float(z["f"])) <= FP64_TOL * abs(float(z["f"]))
    assert rel(g, z["g"]) < FP64_TOL


@pytest.mark.parametrize("dim,tags", [(3, ["g", "m1", "m2", "m3", "m4"]),
                                      (2, ["g", "m1", "m2", "m3", "m4"])])
def test_fp64_gpu_reference_kernel_orders(dim, tags):
    z = golden(f"objgrd_orders_{dim}d")
    R = _refcu(dim)
    for tag in tags:
        order = -1 if tag == "g" else int(tag[1])
        P = problem_from(z, knl_order=order)
        f, g = R.objgrd(P, z["alp"])
        assert abs(f - float(z[f"f_{tag}"])) <= FP64_TOL * abs(float(z[f"f_{tag}"])), tag
        assert rel(g, z[f"g_{tag}"]) < FP64_TOL, tag


def test_fp32_path_matches_fp64_gpu_reference_sphere2cube():
    """Full-size sphere -> cube (2562 vertices, 12288 target triangles, T = 20) at a
    non-trivial momentum: objective and gradient of the CUDA path within 1e-5 of the
    reference's FP64 GPU path."""
    from lddmm_b200 import api
    from lddmm_b200.problem import sphere_to_cube

    P = sphere_to_cube()
    alp = np.random.default_rng(3).normal(scale=0.02, size=P.var_num)
    f_ref, g_ref = _refcu(3).objgrd(P, alp)
    f, g = api.objgrd(P, alp)
    assert abs(f - f_ref) <= TOL * abs(f_ref)
    assert rel(g, g_ref) < TOL
