"""The benchmark population's own pairs (problem.population(seed=0) draws its pairs
in order, so its first 12 pairs are the first 12 of the 256-pair batch the bench
registers): the whole group evaluated in one batched context, with the launch shape
the autotuner picks for it, and four of its pairs -- 531 landmarks onto 20,086 target
triangles, 3,714 onto 31,480, 5,443 onto 9,680 and 10,139 onto 1,010 -- checked
against the FP64 oracle: objective and gradient within 1e-5 relative."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-5
CHECKED = (1, 3, 9, 4)


def test_population_pairs_in_one_batch_against_the_oracle(oracle):
    from lddmm_b200 import api, problem

    probs = problem.population(n_pairs=12, seed=0)
    rng = np.random.default_rng(17)
    xs = [rng.normal(size=P.var_num) * 0.01 for P in probs]
    with api.Context(probs) as ctx:
        fb, gb = ctx.objgrd(np.concatenate(xs))
        gbs = ctx.split(gb)
    for k in CHECKED:
        P = probs[k]
        fo, go = oracle.objgrd(P, xs[k])
        ef = abs(fb[k] - fo) / abs(fo)
        eg = rel(gbs[k], go)
        print(f"pair {k}: {P.nde_num} landmarks, {P.tgt_elm_num} target triangles: "
              f"f rel {ef:.1e}, g rel {eg:.1e}")
        assert ef < TOL, (k, ef)
        assert eg < TOL, (k, eg)
