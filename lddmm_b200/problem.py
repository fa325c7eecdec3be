"""Registration problem description and the synthetic workloads.

``Problem`` carries exactly the arguments of the reference's MEX entry point
``LDDMM3D/LDDMM2D`` (``Cpp/src/LDDMM.cpp:16-37``) in the C++ layout (coordinates
fastest).  The workload builders below create the seeded synthetic shapes the
benchmarks and parity tests run on.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import shapes


@dataclasses.dataclass
class Problem:
    ini_nde: np.ndarray            # (N, D) float64, source landmarks (iniNdeMat)
    elm_vtx: np.ndarray            # (E_d, D) int32, 0-based (dfmElmVtxMat)
    tgt_cen: np.ndarray            # (E_t, D) float64 (tgtCenPosMat)
    tgt_dir: np.ndarray            # (E_t, D) float64 (tgtUniDirMat)
    tgt_vol: np.ndarray            # (E_t,)   float64 (tgtElmVolVec)
    knl_order: int = -1            # -1 Gaussian, 0..4 Matern (knlOrder)
    knl_width: float = 0.5         # knlWidth
    time_num: int = 21             # number of time points, T = time_num - 1 steps
    time_stp: float = 0.05         # timeStp
    cen_type: str = "G"            # cenKnlType: 'G' Gaussian, 'C' Cauchy
    cen_width: float = 0.2         # cenKnlWidth
    dir_type: str = "B"            # dirKnlType: 'B', 'L', 'O', 'U'
    dir_width: float = 0.0         # dirKnlWidth
    dis_wgt: float = 1.0           # disWgt
    elm_ifo: np.ndarray | None = None  # (N, rows) int32 vertex->element table (getElmIfo)
    name: str = ""

    def __post_init__(self):
        self.ini_nde = np.ascontiguousarray(self.ini_nde, dtype=np.float64)
        self.elm_vtx = np.ascontiguousarray(self.elm_vtx, dtype=np.int32)
        self.tgt_cen = np.ascontiguousarray(self.tgt_cen, dtype=np.float64)
        self.tgt_dir = np.ascontiguousarray(self.tgt_dir, dtype=np.float64)
        self.tgt_vol = np.ascontiguousarray(self.tgt_vol, dtype=np.float64).reshape(-1)
        if self.elm_ifo is None:
            self.elm_ifo = elm_ifo(self.elm_vtx, self.ini_nde.shape[0])
        self.elm_ifo = np.ascontiguousarray(self.elm_ifo, dtype=np.int32)

    @property
    def dim(self) -> int:
        return int(self.ini_nde.shape[1])

    @property
    def nde_num(self) -> int:
        return int(self.ini_nde.shape[0])

    @property
    def T(self) -> int:
        return self.time_num - 1

    @property
    def var_num(self) -> int:
        return self.dim * self.nde_num * self.T

    @property
    def dfm_elm_num(self) -> int:
        return int(self.elm_vtx.shape[0])

    @property
    def tgt_elm_num(self) -> int:
        return int(self.tgt_vol.shape[0])

    def pairs_per_eval(self) -> dict:
        """Ordered pair interactions per objective evaluation, as the reference
        evaluates them: shoot T*N^2, adjoint T*N^2, varifold E_d^2 + E_d*E_t
        (the target self-term E_t^2 is constant and computed once)."""
        n, T, ed, et = self.nde_num, self.T, self.dfm_elm_num, self.tgt_elm_num
        return {"shoot": T * n * n, "adjoint": T * n * n, "varifold": ed * ed + ed * et,
                "target_self_once": et * et}

    def diameter(self) -> float:
        q = self.ini_nde
        return float(np.linalg.norm(q.max(axis=0) - q.min(axis=0)))


def elm_ifo(elm_vtx: np.ndarray, nde_num: int) -> np.ndarray:
    """Vertex -> adjacent element table, the semantics of ``Cpp/src/getElmIfo.m:1-59``
    (0-based).  Row 0 of each vertex column is its element count; then per adjacent
    element (in increasing element order) either (element, sign) in 2D, sign -1 when
    the vertex is the element's first vertex, or (element, a, b) in 3D with (a, b)
    the two other vertices ordered so that dd x (q_a - q_b) is the derivative of the
    element's normal with respect to this vertex.  Returned as (N, rows)."""
    ev = np.asarray(elm_vtx, dtype=np.int64)
    E, V = ev.shape
    if V not in (2, 3):
        raise ValueError("elements must have 2 or 3 vertices")
    flat = ev.ravel()
    cnt = np.bincount(flat, minlength=nde_num)
    rows = 1 + int(cnt.max() if cnt.size else 0) * V
    out = np.zeros((nde_num, rows), dtype=np.int32)
    # entry (e, k) of vertex v = ev[e, k]; a vertex's entries in increasing element order
    # (a stable sort of the element-major list by vertex), a = rank within the vertex
    order = np.argsort(flat, kind="stable")
    v_sorted = flat[order]
    start = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    a = np.arange(flat.size) - start[v_sorted]
    e, k = order // V, order % V
    if V == 2:
        out[v_sorted, 1 + 2 * a] = e
        out[v_sorted, 2 + 2 * a] = np.where(k == 0, -1, 1)
    else:
        o1 = np.array([2, 0, 1])[k]  # the other two vertices: (2, 1), (0, 2), (1, 0)
        o2 = np.array([1, 2, 0])[k]
        out[v_sorted, 1 + 3 * a] = e
        out[v_sorted, 2 + 3 * a] = ev[e, o1]
        out[v_sorted, 3 + 3 * a] = ev[e, o2]
    out[:, 0] = cnt
    return out


# --------------------------------------------------------------------- workloads

def circle_to_square(n_src: int = 200, n_tgt: int = 256, sigma_v: float = 0.5,
                     sigma_w: float = 0.2, time_num: int = 21, dis_wgt: float = 1.0) -> Problem:
    """2D circle -> square: source n_src points on the unit circle, target n_tgt
    points on the boundary of [-1,1]^2, both closed polylines.  Gaussian deformation
    kernel, varifold Gaussian on segment centres x Binet on tangents."""
    src, se = shapes.circle(n_src)
    tv, te = shapes.square_boundary(n_tgt, 1.0)
    cen, dr, vol = shapes.varifold_of(tv, te)
    T = time_num - 1
    return Problem(src, se, cen, dr, vol, knl_order=-1, knl_width=sigma_v, time_num=time_num,
                   time_stp=1.0 / T, cen_type="G", cen_width=sigma_w, dir_type="B",
                   dir_width=0.0, dis_wgt=dis_wgt, name="circle2square")


def circle_to_square_example(n_src: int = 500, n_tgt: int = 1000, half: float = 0.8) -> Problem:
    """The reference's own 2D example (Cpp/examples/circle2square/run_circle2square.m:3-45),
    restated: n_src points on the unit circle onto the boundary of [-half, half]^2
    (n_tgt points, counter-clockwise from a corner), both closed polylines.  2D Matern
    order 3 (Bessel K form) of width 0.025, varifold Cauchy(0.1) on segment centres x
    Binet, weight 100, dt = 0.05 over 20 steps."""
    src, se = shapes.circle(n_src)
    tv, te = shapes.square_boundary(n_tgt, half)
    cen, dr, vol = shapes.varifold_of(tv, te)
    return Problem(src, se, cen, dr, vol, knl_order=3, knl_width=0.025, time_num=21,
                   time_stp=0.05, cen_type="C", cen_width=0.1, dir_type="B", dir_width=0.0,
                   dis_wgt=100.0, name="circle2square_example")


def sphere_to_cube(subdiv: int = 4, cube_n: int = 32, knl_width: float = 0.4,
                   sigma_w: float = 0.15, time_num: int = 21, dis_wgt: float = 1.0,
                   knl_order: int = 1) -> Problem:
    """3D sphere -> cube: icosphere (2562 v / 5120 t at subdiv 4) onto the surface of
    [-1,1]^3 with cube_n x cube_n quads per face (12288 t at 32).  Matern nu=3/2
    (order 1) deformation kernel, varifold Gaussian x Binet."""
    V, F = shapes.icosphere(subdiv)
    cv, cf = shapes.cube_surface(cube_n, 1.0)
    cen, dr, vol = shapes.varifold_of(cv, cf)
    T = time_num - 1
    return Problem(V, F, cen, dr, vol, knl_order=knl_order, knl_width=knl_width,
                   time_num=time_num, time_stp=1.0 / T, cen_type="G", cen_width=sigma_w,
                   dir_type="B", dis_wgt=dis_wgt, name="sphere2cube")


def star_pair(src_subdiv: int = 7, tgt_subdiv: int = 6, lmax: int = 8, sigma: float = 0.05,
              seed_src: int = 0, seed_tgt: int = 1, sigma_v: float = 0.3, sigma_w: float = 0.1,
              time_num: int = 11, dis_wgt: float = 1.0) -> Problem:
    """Star-shaped source (icosphere ``src_subdiv``) onto a star-shaped target
    (icosphere ``tgt_subdiv``), r = 1 + sum_{l<=lmax} c_lm Y_lm, c_lm ~ N(0, sigma^2).
    Gaussian deformation kernel and varifold Gaussian x Binet."""
    V, F = shapes.star_surface(src_subdiv, lmax, sigma, seed_src)
    tv, tf = shapes.star_surface(tgt_subdiv, lmax, sigma, seed_tgt)
    cen, dr, vol = shapes.varifold_of(tv, tf)
    T = time_num - 1
    return Problem(V, F, cen, dr, vol, knl_order=-1, knl_width=sigma_v, time_num=time_num,
                   time_stp=1.0 / T, cen_type="G", cen_width=sigma_w, dir_type="B",
                   dis_wgt=dis_wgt, name="star_pair")


def _population_pair(args) -> Problem:
    k, nv, nt, ps, lmax, sigma, sigma_v, sigma_w, time_num = args
    V, F = shapes.decimated_star(nv, lmax, sigma, ps)
    # a closed triangulation of the sphere with nt triangles has nt/2 + 2 vertices
    tv, tf = shapes.decimated_star(max(nt // 2 + 2, 12), lmax, sigma, ps + 1)
    cen, dr, vol = shapes.varifold_of(tv, tf)
    T = time_num - 1
    return Problem(V, F, cen, dr, vol, knl_order=-1, knl_width=sigma_v, time_num=time_num,
                   time_stp=1.0 / T, cen_type="G", cen_width=sigma_w, dir_type="B",
                   dis_wgt=1.0, name=f"pop{k}")


def population(n_pairs: int = 256, seed: int = 0, n_min: int = 500, n_max: int = 20000,
               t_min: int = 1000, t_max: int = 40000, lmax: int = 8, sigma: float = 0.05,
               sigma_v: float = 0.3, sigma_w: float = 0.1, time_num: int = 11,
               workers: int = 1):
    """Batch of independent star-shaped pairs with log-uniform vertex counts in
    [n_min, n_max] (random vertex decimation) and log-uniform target triangle counts
    in [t_min, t_max].  workers > 1 builds the meshes in that many spawned processes
    (same pairs: every random draw of the sizes and seeds happens here, in order)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_pairs):
        nv = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        nt = int(round(math.exp(rng.uniform(math.log(t_min), math.log(t_max)))))
        ps = int(rng.integers(0, 2**31 - 1))
        jobs.append((k, nv, nt, ps, lmax, sigma, sigma_v, sigma_w, time_num))
    if workers <= 1:
        return [_population_pair(j) for j in jobs]
    import concurrent.futures as cf
    import multiprocessing as mp

    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_population_pair, jobs, chunksize=4))
