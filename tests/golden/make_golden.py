"""Generate the golden parity fixtures from the reference itself.

Run in a container that has the reference tree (it is read at build time only):

    make -C oracle ref          # compiles the reference's Cpp/src into oracle/_ref/
    python tests/golden/make_golden.py

Every output array here comes from the reference's own C++ FP64 code
(oracle/_ref/libref{2,3}d.so, built from Cpp/src unmodified); the inputs are
seeded synthetic shapes or the reference's example data
(Cpp/examples/sphere2cube/sphereData.mat, cubeData.mat; target subsampled 1:10 to
keep the fixture small).  The tests compare the project's oracle and the CUDA path
against these files; nothing at test time reads the reference tree.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from lddmm_b200 import problem  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

# the reference checkout: $LDDMM_REFERENCE, else `reference` beside the repository root
REF_TREE = os.environ.get("LDDMM_REFERENCE",
                          os.path.join(os.path.dirname(ROOT), "reference"))


def save(name, P=None, **arrays):
    out = {}
    if P is not None:
        out.update(ini_nde=P.ini_nde, elm_vtx=P.elm_vtx, tgt_cen=P.tgt_cen, tgt_dir=P.tgt_dir,
                   tgt_vol=P.tgt_vol, elm_ifo=P.elm_ifo,
                   scalars=np.array([P.knl_order, P.knl_width, P.time_num, P.time_stp,
                                     P.cen_width, P.dir_width, P.dis_wgt]),
                   types=np.array([P.cen_type, P.dir_type]))
    out.update(arrays)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print(f"{name}: {os.path.getsize(path) / 1024:.1f} KiB")


def kernels(dim, seed):
    R = Reference(dim)
    rng = np.random.default_rng(seed)
    n = 96
    q = rng.uniform(-1, 1, size=(n, dim))
    a = rng.normal(size=(n, dim))
    l = rng.normal(size=(n, dim))
    arrays = dict(q=q, a=a, l=l, width=np.array(0.6))
    for order in (-1, 0, 1, 2, 3, 4):
        tag = f"m{order}" if order >= 0 else "g"
        arrays[f"v_{tag}"] = R.multiply_kernel(q, a, order, 0.6)
        arrays[f"dq_{tag}"] = R.dq_kernel(q, l, a, order, 0.6)
    save(f"kernels_{dim}d", **arrays)


def two_set_kernels(dim, seed):
    """The two-point-set overloads (computeKernel.cpp:246, multiplyKernel.cpp:294,
    dqKernel.cpp:307) and the one-set kernel matrix (computeKernel.cpp:21)."""
    R = Reference(dim)
    rng = np.random.default_rng(seed)
    ni, nj = 48, 37
    qi = rng.uniform(-1, 1, size=(ni, dim))
    qj = rng.uniform(-1, 1, size=(nj, dim))
    a = rng.normal(size=(nj, dim))
    l = rng.normal(size=(ni, dim))
    r = rng.normal(size=(nj, dim))
    arrays = dict(qi=qi, qj=qj, a=a, l=l, r=r, width=np.array(0.5))
    for order in (-1, 0, 1, 2, 3, 4):
        tag = f"m{order}" if order >= 0 else "g"
        arrays[f"K_{tag}"] = R.compute_kernel2(qi, qj, order, 0.5)
        arrays[f"K1_{tag}"] = R.compute_kernel(qi, order, 0.5)
        arrays[f"v_{tag}"] = R.multiply_kernel2(qi, qj, a, order, 0.5)
        dqi, dqj = R.dq_kernel2(qi, qj, l, r, order, 0.5)
        arrays[f"dqi_{tag}"] = dqi
        arrays[f"dqj_{tag}"] = dqj
    save(f"two_set_kernels_{dim}d", **arrays)


def _sphere2cube_example_problem():
    import scipy.io as sio
    ex = os.path.join(REF_TREE, "Cpp", "examples", "sphere2cube")
    s = sio.loadmat(os.path.join(ex, "sphereData.mat"))
    c = sio.loadmat(os.path.join(ex, "cubeData.mat"))
    sel = np.arange(0, c["tgtCenPosMat"].shape[1], 10)
    # parameters of Cpp/examples/sphere2cube/run_sphere2cube.m:14-24
    return problem.Problem(s["iniNdeMat"].T, s["elmVtxMat"].T.astype(np.int32) - 1,
                           c["tgtCenPosMat"].T[sel], c["tgtUniDirMat"].T[sel],
                           c["tgtElmVolVec"].ravel()[sel], knl_order=3, knl_width=0.25,
                           time_num=21, time_stp=0.05, cen_type="C", cen_width=0.1,
                           dir_type="B", dir_width=0.0, dis_wgt=100.0)


def sphere2cube_example_columns():
    """The reference's example optimiser options as run_sphere2cube.m:27-31 passes them
    (Columns = 10000, Wolfe 0 / 0.5, tolerance 1e-2), for 40 iterations: the history
    grows past 32 pairs.  The reference allocates the whole ring of 10000 (s, y) pairs
    (Cpp/src/LDDMM.cpp:58-60; 5.8 GB here)."""
    P = _sphere2cube_example_problem()
    R = Reference(3)
    r = R.lbfgs(P, np.zeros(P.var_num), itr_max=40, tol=1e-2, wolfe1=0.0, wolfe2=0.5,
                mem_num=10000)
    save("sphere2cube_example_columns", x=r["x"], f=np.array(r["f"]), ret=np.array(r["ret"]),
         trace_f=r["trace_f"], trace_g2=r["trace_g2"],
         opt=np.array([40, 1e-2, 0.0, 0.5, 10000]))


def sphere2cube_example_full():
    """The reference's example exactly as run_sphere2cube.m:27-31 calls it
    (MaxIterations 100000, OptimalityTolerance 1e-2, Wolfe 0 / 0.5, Columns 10000), run
    until its own stopping test; the final landmarks are the returned momenta shot by the
    FP64 oracle (computeNodePosition)."""
    from oracle.oracle import Oracle

    P = _sphere2cube_example_problem()
    R = Reference(3)
    r = R.lbfgs(P, np.zeros(P.var_num), itr_max=100000, tol=1e-2, wolfe1=0.0, wolfe2=0.5,
                mem_num=10000)
    nde, _ = Oracle().shoot(P.ini_nde, r["x"], P.knl_order, P.knl_width, P.time_stp,
                            P.time_num)
    save("sphere2cube_example_full", f=np.array(r["f"]), ret=np.array(r["ret"]),
         evals=np.array(r["evals"]), nde_final=nde[-1], trace_f=r["trace_f"],
         opt=np.array([100000, 1e-2, 0.0, 0.5, 10000]))


def sphere2cube_example():
    P = _sphere2cube_example_problem()
    R = Reference(3)
    rng = np.random.default_rng(11)
    alp = rng.normal(size=P.var_num) * 0.02
    f, g = R.objgrd(P, alp)
    vf, vdq = R.varifold(P, P.ini_nde)
    save("sphere2cube_example", P, alp=alp, f=np.array(f), g=g, vfd=np.array(vf), vfd_dq=vdq)
    r = R.lbfgs(P, np.zeros(P.var_num), itr_max=15, tol=1e-2, wolfe1=0.0, wolfe2=0.5,
                mem_num=10)
    save("sphere2cube_example_lbfgs", x=r["x"], f=np.array(r["f"]), ret=np.array(r["ret"]),
         trace_f=r["trace_f"], trace_g2=r["trace_g2"],
         opt=np.array([15, 1e-2, 0.0, 0.5, 10]))


def circle2square():
    P = problem.circle_to_square()
    R = Reference(2)
    rng = np.random.default_rng(5)
    alp = rng.normal(size=P.var_num) * 0.05
    f, g = R.objgrd(P, alp)
    save("circle2square_objgrd", P, alp=alp, f=np.array(f), g=g)
    r = R.lbfgs(P, np.zeros(P.var_num), itr_max=40, tol=1e-6, wolfe1=1e-4, wolfe2=0.9,
                mem_num=5)
    save("circle2square_lbfgs", P, x=r["x"], f=np.array(r["f"]), ret=np.array(r["ret"]),
         trace_f=r["trace_f"], trace_g2=r["trace_g2"], opt=np.array([40, 1e-6, 1e-4, 0.9, 5]))


def circle2square_example():
    """The reference's 2D example setting (2D Matern order 3, Cauchy centres)."""
    P = problem.circle_to_square_example()
    R = Reference(2)
    rng = np.random.default_rng(11)
    alp = rng.normal(size=P.var_num) * 0.02
    f, g = R.objgrd(P, alp)
    r = R.lbfgs(P, np.zeros(P.var_num), itr_max=15, tol=1e-2, wolfe1=0.0, wolfe2=0.5,
                mem_num=10)
    save("circle2square_example", P, alp=alp, f=np.array(f), g=g, x=r["x"],
         f_lbfgs=np.array(r["f"]), ret=np.array(r["ret"]), trace_f=r["trace_f"],
         trace_g2=r["trace_g2"], opt=np.array([15, 1e-2, 0.0, 0.5, 10]))


def varifold_types():
    R = Reference(3)
    rng = np.random.default_rng(3)
    base = problem.sphere_to_cube(subdiv=2, cube_n=5)
    arrays = {}
    q = base.ini_nde * 0.9 + rng.normal(size=base.ini_nde.shape) * 0.02
    for ct in "GC":
        for dt in "BLOU":
            base.cen_type, base.dir_type = ct, dt
            base.cen_width, base.dir_width = 0.3, 0.8
            v, dq = R.varifold(base, q)
            arrays[f"v_{ct}{dt}"] = np.array(v)
            arrays[f"dq_{ct}{dt}"] = dq
    save("varifold_types_3d", base, q=q, **arrays)
    R2 = Reference(2)
    b2 = problem.circle_to_square(n_src=60, n_tgt=80)
    q2 = b2.ini_nde * 0.8 + rng.normal(size=b2.ini_nde.shape) * 0.02
    arrays = {}
    for ct in "GC":
        for dt in "BLOU":
            b2.cen_type, b2.dir_type = ct, dt
            b2.cen_width, b2.dir_width = 0.3, 0.8
            v, dq = R2.varifold(b2, q2)
            arrays[f"v_{ct}{dt}"] = np.array(v)
            arrays[f"dq_{ct}{dt}"] = dq
    save("varifold_types_2d", b2, q=q2, **arrays)


def objgrd_orders_3d():
    """Small 3D pair for every deformation kernel order (Gaussian, Matern 0..4)."""
    R = Reference(3)
    rng = np.random.default_rng(9)
    arrays = {}
    P = problem.sphere_to_cube(subdiv=2, cube_n=6, time_num=6)
    alp = rng.normal(size=P.var_num) * 0.05
    for order in (-1, 0, 1, 2, 3, 4):
        P.knl_order = order
        f, g = R.objgrd(P, alp)
        tag = f"m{order}" if order >= 0 else "g"
        arrays[f"f_{tag}"] = np.array(f)
        arrays[f"g_{tag}"] = g
    P.knl_order = -1
    save("objgrd_orders_3d", P, alp=alp, **arrays)


def objgrd_orders_2d():
    R = Reference(2)
    rng = np.random.default_rng(10)
    arrays = {}
    P = problem.circle_to_square(n_src=80, n_tgt=96, time_num=6)
    alp = rng.normal(size=P.var_num) * 0.05
    for order in (-1, 0, 1, 2, 3, 4):
        P.knl_order = order
        f, g = R.objgrd(P, alp)
        tag = f"m{order}" if order >= 0 else "g"
        arrays[f"f_{tag}"] = np.array(f)
        arrays[f"g_{tag}"] = g
    P.knl_order = -1
    save("objgrd_orders_2d", P, alp=alp, **arrays)


ALL = {
    "kernels_2d": lambda: kernels(2, 1),
    "kernels_3d": lambda: kernels(3, 2),
    "two_set_kernels_2d": lambda: two_set_kernels(2, 11),
    "two_set_kernels_3d": lambda: two_set_kernels(3, 12),
    "circle2square": circle2square,
    "circle2square_example": circle2square_example,
    "sphere2cube_example": sphere2cube_example,
    "sphere2cube_example_columns": sphere2cube_example_columns,
    "sphere2cube_example_full": sphere2cube_example_full,
    "varifold_types": varifold_types,
    "objgrd_orders_3d": objgrd_orders_3d,
    "objgrd_orders_2d": objgrd_orders_2d,
}

if __name__ == "__main__":
    # python tests/golden/make_golden.py [name ...]   (no names: every fixture)
    for name in (sys.argv[1:] or list(ALL)):
        ALL[name]()
