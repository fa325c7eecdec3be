"""Times the reference's plain FP64 GPU path (CUDA/src compiled in place, see
``make -C oracle refcu``) on whole registrations, next to this project's CUDA path on
the same problem and options, and prints one JSON line per workload.

    python oracle/fp64_gpu_baseline.py [--workloads sphere2cube,circle2square] [--runs 2]

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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workloads", default="sphere2cube,circle2square")
    ap.add_argument("--runs", type=int, default=2)
    a = ap.parse_args()
    for name in a.workloads.split(","):
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
