"""FP64 reference registration of the benchmark workload (sphere -> cube, 2562
landmarks, 500 L-BFGS iterations) by the CPU oracle; writes
tests/golden/sphere2cube_fp64_500.json.  The oracle matches the compiled reference
to 1e-12 on the golden fixtures; it is used here because the reference's own path
stores an N x N x T kernel stack and runs single-threaded (hours for 545
evaluations).  Takes about 16 minutes on 8 cores:

    make -C oracle && python tests/golden/make_c2_reference.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lddmm_b200 import problem  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

if __name__ == "__main__":
    P = problem.sphere_to_cube()
    O = Oracle(threads=os.cpu_count() or 1)
    t = time.time()
    r = O.lbfgs(P, np.zeros(P.var_num), itr_max=500, tol=1e-6, wolfe1=1e-4, wolfe2=0.9,
                mem_num=5)
    out = dict(workload="sphere2cube subdiv 4 / cube 32, Matern order 1 width 0.4, "
                        "G(0.15) x Binet, T=20, m=5, 500 iterations, tol 1e-6",
               f=r["f"], ret=r["ret"], ls_code=r["ls_code"], iters=r["iters"],
               evals=r["evals"], seconds=time.time() - t)
    with open(os.path.join(HERE, "sphere2cube_fp64_500.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)
