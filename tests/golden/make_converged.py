"""Converged-registration fixtures from the reference's own C++ FP64 path.

    make -C oracle ref
    python tests/golden/make_converged.py circle2square_300    # seconds
    python tests/golden/make_converged.py circle2square_converged  # minutes
    python tests/golden/make_converged.py sphere2cube_500      # ~1 h, one core

circle2square_300: the 2D circle -> square workload (200 landmarks on the unit
circle, 256 target points on the square [-1,1]^2, Gaussian 0.5, varifold G(0.2) x
Binet, T = 20, L-BFGS memory 5, 300 iterations, tolerance 1e-6, Wolfe 1e-4 / 0.9).
sphere2cube_500: the 3D sphere -> cube workload (2562-vertex icosphere onto the cube
surface with 32 x 32 quads per face, Matern nu = 3/2 width 0.4, varifold G(0.15) x
Binet, T = 20, memory 5, 500 iterations).

Both are registered from zero momenta by the compiled reference
(oracle/_ref/libref{2,3}d.so, Cpp/src/LBFGS.cpp with its objgrd), and the final
landmarks are its momenta shot forward by the FP64 oracle's computeNodePosition
restatement (Cpp/src/computeNodePosition.m:1-20; the reference's C++ path has no
trajectory routine of its own).  Each fixture keeps the final objective, the final
landmark positions, the return code and the number of objective evaluations.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lddmm_b200 import problem  # noqa: E402
from oracle.oracle import Oracle, Reference  # noqa: E402


def _run(name, P, itr_max):
    R = Reference(P.dim)
    t = time.time()
    r = R.lbfgs(P, np.zeros(P.var_num), itr_max=itr_max, tol=1e-6, wolfe1=1e-4, wolfe2=0.9,
                mem_num=5)
    secs = time.time() - t
    nde, _ = Oracle().shoot(P.ini_nde, r["x"], P.knl_order, P.knl_width, P.time_stp,
                            P.time_num)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), f=np.array(r["f"]),
                        ret=np.array(r["ret"]), evals=np.array(r["evals"]),
                        nde_final=nde[-1], itr_max=np.array(itr_max),
                        trace_f=r["trace_f"])
    print(name, "f", r["f"], "ret", r["ret"], "evals", r["evals"], f"{secs:.0f} s")


ALL = {
    "circle2square_300": lambda: _run("circle2square_300", problem.circle_to_square(), 300),
    # the same registration run until |g| < 1e-6 (or 20000 iterations)
    "circle2square_converged": lambda: _run("circle2square_converged",
                                            problem.circle_to_square(), 20000),
    "sphere2cube_500": lambda: _run("sphere2cube_500", problem.sphere_to_cube(), 500),
}

if __name__ == "__main__":
    for name in (sys.argv[1:] or list(ALL)):
        ALL[name]()
