"""The launch-shape autotuner (lddmm_config.autotune, on by default): it times the
candidate shapes of each sweep on the context's own batch (64-row tiles per work
item, cluster splits, persistent or per-step time loops) and keeps the fastest.
Checked here: the chosen sizes are valid, its trial sweeps leave nothing behind (the
tuned context gives bitwise the same objective and gradient as a fresh context created
with those sizes given explicitly -- every reduction has a fixed order for a given
launch plan, and two-tile items give bitwise the sums of one-tile items), the result
agrees with the default context's within the FP32 tolerance, and the tuned shape is
never slower than the built-in rule's on the sphere -> cube pair and the large pair."""
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
    assert cfg[0] in (1, 2, 4, 8) and cfg[1] in (1, 2, 4, 8) and 1 <= cfg[2] <= 8
    with api.Context(P, cluster=cfg) as same:
        f2, g2 = same.objgrd(x)
    assert f1[0] == f2[0] and np.array_equal(g1, g2)
    with api.Context(P) as default:
        f3, g3 = default.objgrd(x)
    assert abs(f1[0] - f3[0]) <= 1e-6 * abs(f3[0])
    assert mrel(g1, g3) < 1e-5


def _eval_ms(ctx, reps, tries=3):
    """Fastest of `tries` measurements of the average evaluation time."""
    return min(ctx.time_sweeps(reps=reps)["eval"] for _ in range(tries))


@pytest.mark.parametrize("which", ["sphere2cube", "large_pair"])
def test_autotuned_shape_is_never_slower_than_the_rule(which):
    """The default context (autotuned: tiles per work item, cluster splits, persistent
    or per-step time loops) against the built-in rule (autotune off), on the 2562-
    landmark sphere -> cube pair and the 163,842-landmark star pair: the tuned shape's
    objective + gradient evaluation is at most 2 % slower (it is chosen by timing, so
    it should not be slower at all beyond noise)."""
    from lddmm_b200 import api, problem

    P = problem.sphere_to_cube() if which == "sphere2cube" else problem.star_pair()
    reps = 20 if which == "sphere2cube" else 2
    with api.Context(P, autotune=False) as rule:
        shape_rule = rule.launch_shape()
        ms_rule = _eval_ms(rule, reps)
    with api.Context(P) as tuned:
        shape_tuned = tuned.launch_shape()
        ms_tuned = _eval_ms(tuned, reps)
    print(f"{which}: rule {shape_rule} {ms_rule:.3f} ms, tuned {shape_tuned} {ms_tuned:.3f} ms")
    assert ms_tuned <= 1.02 * ms_rule, (shape_rule, ms_rule, shape_tuned, ms_tuned)
