"""What the trained warm-start network gains over the plain method, end to end at a
reduced size (642-landmark icosphere onto 1280-triangle perturbed spheres, T = 10):
1024 plain-method registrations train the network (400 epochs), then 32 held-out
pairs are registered from zero (cold) and from the prediction (warm), both run to
convergence (relative objective change below 1e-9, at most 1000 iterations).

Two networks: the configured one (local_k = 0: the target reaches each landmark only
through 64 max-pooled features) and one that also reads every landmark's 24 nearest
target triangles (local_k = 24, lddmm_ws_create_ex).

Measured and asserted, per held-out pair:
  * time to tolerance: objective evaluations (and batch wall time) until the run is
    within 1e-5 relative of the cold start's converged objective; the medians of warm
    and cold are reported.  Measured: configured network 238.5 warm vs 238 cold
    evaluations (no gain; the warm start must not cost more than 5 %); local features
    trained on converged registrations 136.5 vs 235, a median per-pair gain of 1.70x
    (1.43x with the default labels; asserted >= 1.2x).  At full size the same network
    reaches 2.17x;
  * the result is judged by the plain method, not by the network: the warm run's
    converged objective must match the cold start's within 1e-5 relative.
The prediction must also start L-BFGS at a clearly lower objective."""
import functools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-5


@pytest.mark.parametrize("local_k", [0, 24])
def test_warm_start_gain(local_k):
    from lddmm_b200 import warmstart as W

    make = functools.partial(W.pair, src_subdiv=3, tgt_subdiv=3)
    # the local-feature network learns from registrations taken to convergence (the
    # slow eigenmodes it predicts are only settled there); the configured one from the
    # default labels (converged ones measured no gain for it: it fits neither)
    gen = dict(itr_max=1000, rel_obj_tol=1e-9) if local_k else {}
    tri, lab, src, _ = W.generate(list(range(1000, 2024)), batch=64, make=make, **gen)
    scale = float(lab.pow(2).mean().sqrt())
    with W.WarmStart(src, W.T_STEPS, batch_max=64, tri_max=tri.shape[1], label_scale=scale,
                     seed=0, local_k=local_k) as ws:
        hist = W.train(ws, tri, lab, epochs=400, batch=64, lr=1e-3)
        ev = W.evaluate(ws, list(range(50000, 50032)), batch=32, make=make, itr_max=1000,
                        rel_obj_tol=1e-9, rel=REL)
    rows = ev["rows"]
    ratio = np.median([r["f_start_warm"] / r["f_start_cold"] for r in rows])
    dev = np.array([abs(r["f_warm"] - r["f_cold"]) / abs(r["f_cold"]) for r in rows])
    print(f"local_k {local_k}: time to tolerance (median evaluations): cold "
          f"{ev['median_evals_cold']}, warm "
          f"{ev['median_evals_warm']}, median per-pair gain {ev['median_speedup_evals']:.2f}x; "
          f"wall {ev['seconds_cold']:.2f} s cold, {ev['seconds_warm']:.2f} s warm; start "
          f"objective ratio {ratio:.3f}; converged objectives within {REL:g}: "
          f"{int(np.sum(dev <= REL))}/{len(rows)} (median deviation {np.median(dev):.2e})")
    assert hist[-1] < 0.8 * hist[0], hist[::10]
    assert ratio < 0.8, ratio
    assert all(r["f_warm"] == r["f_warm"] for r in rows)
    # judged by the plain method: converged objectives agree within 1e-5
    assert np.median(dev) <= REL, np.median(dev)
    assert np.mean(dev <= REL) >= 0.9, dev
    # time to tolerance: the warm start costs no more than the cold start (5 % margin)
    assert ev["reached"] >= 0.9 * len(rows)
    assert ev["median_evals_warm"] <= 1.05 * ev["median_evals_cold"], ev
    if local_k:
        assert ev["median_speedup_evals"] >= 1.2, ev["median_speedup_evals"]
