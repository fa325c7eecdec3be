"""Times the reference's plain FP64 GPU path (CUDA/src compiled in place, see
``make -C oracle refcu``) on whole registrations, next to this project's CUDA path on
the same problem and options, and prints one JSON line per workload.

    python oracle/fp64_gpu_baseline.py [--workloads sphere2cube,circle2square] [--runs 2]
    python oracle/fp64_gpu_baseline.py --workloads population [--pairs 256] [--samples 8] [--runs 2]

Measurement infrastructure: the FP64 GPU numbers are the baseline the FP32 +
compensated path is compared with; nothing here is part of the product.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from oracle.oracle import ReferenceCuda  # noqa: E402
from lddmm_b200 import api, problem  # noqa: E402

WORKLOADS = {
    # name: (problem factory, L-BFGS options)
    "sphere2cube": (problem.sphere_to_cube, dict(itr_max=500, tol=1e-6)),
    "circle2square": (problem.circle_to_square, dict(itr_max=300, tol=1e-6)),
}


def ours(P, opt, runs):
    with api.Context(P) as ctx:
        x0 = np.zeros(P.var_num)
        ctx.lbfgs(x0, **opt)  # warm-up (first call per context)
        best = None
        for _ in range(runs):
            t = time.perf_counter()
            x, res = ctx.lbfgs(x0, **opt)
            dt = time.perf_counter() - t
            best = dt if best is None else min(best, dt)
        return dict(seconds=best, f=float(res[0]["f"]), evals=int(res[0]["evals"]),
                    iters=int(res[0]["iters"]), status=int(res[0]["status"]))


def population(n_pairs, samples, seed=0, repeats=2):
    """The uneven batch: every pair registered together in one context (stopping at
    1e-5 relative objective change), then the reference's FP64 GPU path on `samples`
    pairs spread over the size range, each run for the iterations that pair took
    here (after one warm-up call; the fastest of `repeats` runs); the reference's
    time for the whole batch is extrapolated from those runs by a two-term model (a
    fixed cost per evaluation plus a cost per pair interaction, fitted to the
    samples)."""
    probs = problem.population(n_pairs=n_pairs, seed=seed)
    x0 = np.zeros(sum(P.var_num for P in probs))
    with api.Context(probs) as ctx:
        ctx.lbfgs(x0, itr_max=1, tol=1e-6)  # warm-up (first call per context)
        t = time.perf_counter()
        x, res = ctx.lbfgs(x0, itr_max=2000, tol=1e-12, rel_obj_tol=1e-5)
        secs = time.perf_counter() - t

    def pairs_per_eval(P):
        return 2 * P.T * P.nde_num ** 2 + P.dfm_elm_num * (P.dfm_elm_num + P.tgt_elm_num)

    order = np.argsort([P.nde_num for P in probs])
    pick = [int(order[int(q * (len(order) - 1))]) for q in np.linspace(0.0, 1.0, samples)]
    R = ReferenceCuda(3)
    P0 = probs[pick[0]]
    R.lbfgs(P0, np.zeros(P0.var_num), itr_max=1, tol=1e-12)  # warm-up: library start-up
    ref = []
    for k in pick:
        P = probs[k]
        it = max(1, int(res[k]["iters"]))
        runs = [R.lbfgs(P, np.zeros(P.var_num), itr_max=it, tol=1e-12)
                for _ in range(max(1, repeats))]
        r = min(runs, key=lambda z: z["ms_total"])
        work = r["evals"] * (pairs_per_eval(P) + P.tgt_elm_num ** 2)  # it recomputes TT
        ref.append(dict(pair=k, landmarks=P.nde_num, targets=P.tgt_elm_num, iters=it,
                        evals=r["evals"], seconds=r["ms_total"] * 1e-3,
                        ns_per_pair=r["ms_total"] * 1e6 / work))
    # time model of the reference per registration: a fixed cost per evaluation (its
    # host-synchronising BLAS calls and launches) plus a cost per pair interaction,
    # least squares over the samples (non-negative)
    Aeq = np.array([[r["evals"], r["evals"] * (pairs_per_eval(probs[r["pair"]]) +
                                               probs[r["pair"]].tgt_elm_num ** 2)]
                    for r in ref], dtype=np.float64)
    tsec = np.array([r["seconds"] for r in ref])
    from scipy.optimize import nnls

    coef, _ = nnls(Aeq, tsec)
    ref_secs = float(sum(coef[0] * res[k]["evals"] + coef[1] * res[k]["evals"] *
                         (pairs_per_eval(P) + P.tgt_elm_num ** 2)
                         for k, P in enumerate(probs)))
    ns = float(coef[1] * 1e9)
    return {"workload": "population", "pairs": n_pairs,
            "landmarks_min_median_max": [int(min(P.nde_num for P in probs)),
                                         int(np.median([P.nde_num for P in probs])),
                                         int(max(P.nde_num for P in probs))],
            "ours": {"seconds": secs, "registrations_per_s": n_pairs / secs,
                     "iters_median": float(np.median([r["iters"] for r in res])),
                     "iters_max": int(max(r["iters"] for r in res)),
                     "status": sorted(set(int(r["status"]) for r in res))},
            "fp64_gpu_sample": ref,
            "fp64_gpu_extrapolated": {"seconds": ref_secs,
                                      "registrations_per_s": n_pairs / ref_secs,
                                      "ms_per_evaluation": float(coef[0] * 1e3),
                                      "ns_per_pair_interaction": ns,
                                      "model": "t = a * evaluations + b * evaluations * pair "
                                               "interactions per evaluation (nnls)"},
            "speedup_extrapolated": ref_secs / secs}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="sphere2cube,circle2square")
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--pairs", type=int, default=256, help="population workload size")
    ap.add_argument("--samples", type=int, default=8, help="population pairs run on FP64")
    a = ap.parse_args()
    for name in a.workloads.split(","):
        if name == "population":
            print(json.dumps(population(a.pairs, a.samples, repeats=a.runs)), flush=True)
            continue
        make, opt = WORKLOADS[name]
        P = make()
        R = ReferenceCuda(P.dim)
        runs = []
        for _ in range(a.runs):
            r = R.lbfgs(P, np.zeros(P.var_num), itr_max=opt["itr_max"], tol=opt["tol"])
            runs.append(r)
        best = min(runs, key=lambda r: r["ms_total"])
        mine = ours(P, opt, a.runs)
        print(json.dumps({
            "workload": name, "nde_num": P.nde_num, "dfm_elm_num": P.dfm_elm_num,
            "tgt_elm_num": P.tgt_elm_num, "T": P.T, "itr_max": opt["itr_max"],
            "fp64_gpu": {"registrations_per_s": 1e3 / best["ms_total"],
                         "ms_total": best["ms_total"], "ms_lbfgs": best["ms_lbfgs"],
                         "evals": best["evals"], "f": best["f"], "status": best["ret"]},
            "ours": {"registrations_per_s": 1.0 / mine["seconds"], **mine},
            "speedup": best["ms_total"] * 1e-3 / mine["seconds"],
            "rel_diff_f": abs(mine["f"] - best["f"]) / abs(best["f"]),
        }), flush=True)


if __name__ == "__main__":
    main()
