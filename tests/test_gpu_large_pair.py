"""The 163,842-landmark star-surface pair (327,680 source triangles onto 81,920 target
triangles, Gaussian 0.3, varifold 0.1 x Binet, T = 10) at full size.  The FP64 oracle
cannot run here (one objective evaluation is ~6.7e11 pair interactions), so the CUDA
path is checked through properties that do not depend on size: the gradient's
directional derivative against a central difference of the objective along the
gradient direction, and descent along -g."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_large_pair_gradient_directional_derivative():
    from lddmm_b200 import api, problem

    P = problem.star_pair()
    assert P.nde_num == 163842 and P.dfm_elm_num == 327680 and P.tgt_elm_num == 81920
    alp = np.random.default_rng(11).normal(size=P.var_num) * 0.01
    with api.Context(P) as ctx:
        f0, g = ctx.objgrd(alp)
        gn = float(np.linalg.norm(g))
        assert np.isfinite(f0[0]) and np.isfinite(gn) and gn > 0
        d = g / gn
        h = 1e-2 / gn * abs(f0[0])  # a step that moves f by ~1 %
        fp, _ = ctx.objgrd(alp + h * d)
        fm, _ = ctx.objgrd(alp - h * d)
    fd = (fp[0] - fm[0]) / (2 * h)
    # g.d = |g|; second-order error O(h^2) and FP32 noise ~1e-7 |f| / h are both far
    # below 1e-3 of it at this step
    assert abs(fd - gn) <= 1e-3 * gn
    assert fm[0] < f0[0] < fp[0]
