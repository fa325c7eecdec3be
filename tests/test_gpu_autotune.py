"""The cluster-size autotuner (lddmm_config.autotune): it times every split size of
each per-step sweep on the context's own batch and keeps the fastest.  Checked here:
the chosen sizes are valid, its trial sweeps leave nothing behind (the tuned context
gives bitwise the same objective and gradient as a fresh context created with those
sizes given explicitly -- every reduction has a fixed order for a given launch plan),
and the result agrees with the default context's within the FP32 tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mrel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def test_autotune_valid_and_stateless():
    from lddmm_b200 import api, problem

    P = problem.sphere_to_cube(subdiv=5)  # 10,242 landmarks: per-step sweeps
    x = np.random.default_rng(7).normal(size=P.var_num) * 0.01
    with api.Context(P, autotune=True) as tuned:
        cfg = tuple(int(s) for s in tuned.launch_config())
        f1, g1 = tuned.objgrd(x)
    assert all(s in (1, 2, 4, 8) for s in cfg)
    with api.Context(P, cluster=cfg) as same:
        f2, g2 = same.objgrd(x)
    assert f1[0] == f2[0] and np.array_equal(g1, g2)
    with api.Context(P) as default:
        f3, g3 = default.objgrd(x)
    assert abs(f1[0] - f3[0]) <= 1e-6 * abs(f3[0])
    assert mrel(g1, g3) < 1e-5
