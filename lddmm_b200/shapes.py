"""Seeded synthetic shapes for registration problems (host-side, numpy).

Every array uses the reference's C++ layout: coordinates fastest, then node/element
(``Cpp/src/objgrd.cpp:47-50``).  A mesh is ``(verts (N, D) float64, elems (E, D) int32)``
with 0-based vertex indices; triangles are oriented so that their normals point
outward, segments run counter-clockwise.

The varifold representation of a target (centres, unit normals/tangents, areas/
lengths) follows ``landmarksToVarifoldKernel`` (``Cpp/src/varifold3D.cpp:8-39``,
``Cpp/src/varifold2D.cpp:8-32``) and the square target of
``Cpp/examples/circle2square/run_circle2square.m:63-66``.
"""
from __future__ import annotations

import functools
import math

import numpy as np


# ----------------------------------------------------------------------- 2D curves

def circle(n: int, radius: float = 1.0):
    """n points at angles 2*pi*k/n on a circle, closed polyline (k, k+1 mod n)."""
    th = 2.0 * np.pi * np.arange(n) / n
    verts = np.stack([radius * np.cos(th), radius * np.sin(th)], axis=1)
    elems = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int32)
    return verts, elems


def square_boundary(n: int, half: float = 1.0):
    """n points (a multiple of 4) equally spaced on the boundary of [-half, half]^2,
    starting at the corner (-half, -half) and running counter-clockwise, closed."""
    assert n % 4 == 0
    s = n // 4
    side = np.linspace(-half, half, s + 1)[:s]
    x = np.concatenate([side, np.full(s, half), -side, np.full(s, -half)])
    y = np.concatenate([np.full(s, -half), side, np.full(s, half), -side])
    verts = np.stack([x, y], axis=1)
    elems = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1).astype(np.int32)
    return verts, elems


# ---------------------------------------------------------------------- 3D meshes

def icosphere(subdiv: int, radius: float = 1.0):
    """Icosahedron subdivided ``subdiv`` times, vertices projected to the sphere.
    10*4^k + 2 vertices, 20*4^k triangles (k = 4: 2562 / 5120).  Returns new arrays
    (the unit mesh of each subdivision level is built once per process)."""
    v, f = _unit_icosphere(subdiv)
    return v * radius, f.copy()


@functools.lru_cache(maxsize=None)
def _unit_icosphere(subdiv: int):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    verts = [tuple(x) for x in v]
    for _ in range(subdiv):
        cache: dict = {}
        vl = verts

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                p = (np.asarray(vl[a]) + np.asarray(vl[b])) / 2.0
                p /= np.linalg.norm(p)
                cache[key] = len(vl)
                vl.append(tuple(p))
            return cache[key]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = np.array(nf, dtype=np.int64)
        verts = vl
    V = np.array(verts, dtype=np.float64)
    F = _orient_outward(V, f).astype(np.int32)
    V.setflags(write=False)
    F.setflags(write=False)
    return V, F


def cube_surface(n: int, half: float = 1.0):
    """Surface of [-half, half]^3, each face an n x n grid of quads, two triangles
    per quad, outward normals.  6n^2 + 2 vertices, 12n^2 triangles."""
    g = np.linspace(-half, half, n + 1)
    pts = {}
    verts = []
    faces = []

    def vid(p, key):
        if key not in pts:
            pts[key] = len(verts)
            verts.append(p)
        return pts[key]

    for axis in range(3):
        for side in (-half, half):
            u_ax, v_ax = [a for a in range(3) if a != axis]
            for a in range(n):
                for b in range(n):
                    quad = []
                    for da, db in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        p = [0.0, 0.0, 0.0]
                        k = [0, 0, 0]
                        p[axis], k[axis] = side, (0 if side < 0 else n)
                        p[u_ax], k[u_ax] = g[a + da], a + da
                        p[v_ax], k[v_ax] = g[b + db], b + db
                        quad.append(vid(p, tuple(k)))
                    faces.append([quad[0], quad[1], quad[2]])
                    faces.append([quad[0], quad[2], quad[3]])
    V = np.array(verts, dtype=np.float64)
    F = _orient_outward(V, np.array(faces, dtype=np.int64))
    return V, F.astype(np.int32)


def _orient_outward(V, F):
    """Flip triangles whose normal points toward the origin (star-shaped surfaces)."""
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    n = np.cross(b - a, c - a)
    ctr = (a + b + c) / 3.0
    flip = np.einsum("ij,ij->i", n, ctr) < 0
    F = F.copy()
    F[flip, 1], F[flip, 2] = F[flip, 2].copy(), F[flip, 1].copy()
    return F


# ------------------------------------------------------- real spherical harmonics

def real_sph_harm(lmax: int, dirs: np.ndarray) -> np.ndarray:
    """Orthonormal real spherical harmonics Y_lm(dirs) for 0 <= l <= lmax,
    columns ordered (l, m) with m = -l..l.  dirs: (K, 3) unit vectors."""
    x, y, z = dirs[:, 0], dirs[:, 1], np.clip(dirs[:, 2], -1.0, 1.0)
    phi = np.arctan2(y, x)
    ct = z
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    K = dirs.shape[0]
    # associated Legendre P_l^m(cos theta) without Condon-Shortley phase
    P = {}
    P[(0, 0)] = np.ones(K)
    for m in range(1, lmax + 1):
        P[(m, m)] = P[(m - 1, m - 1)] * (2 * m - 1) * st
    for m in range(0, lmax):
        P[(m + 1, m)] = (2 * m + 1) * ct * P[(m, m)]
    for m in range(0, lmax + 1):
        for l in range(m + 2, lmax + 1):
            P[(l, m)] = ((2 * l - 1) * ct * P[(l - 1, m)] - (l + m - 1) * P[(l - 2, m)]) / (l - m)
    cols = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
            if m == 0:
                cols.append(norm * P[(l, 0)])
            elif m > 0:
                cols.append(math.sqrt(2.0) * norm * P[(l, am)] * np.cos(am * phi))
            else:
                cols.append(math.sqrt(2.0) * norm * P[(l, am)] * np.sin(am * phi))
    return np.stack(cols, axis=1)


def star_radius(dirs: np.ndarray, lmax: int, sigma: float, seed: int) -> np.ndarray:
    """r = 1 + sum_{l<=lmax} c_lm Y_lm(dir), c_lm ~ N(0, sigma^2) drawn with ``seed``."""
    rng = np.random.default_rng(seed)
    Y = real_sph_harm(lmax, dirs)
    c = rng.normal(0.0, sigma, size=Y.shape[1])
    return 1.0 + Y @ c


def star_surface(subdiv: int, lmax: int, sigma: float, seed: int):
    """Star-shaped surface r(dir) = 1 + sum c_lm Y_lm on an icosphere."""
    V, F = icosphere(subdiv)
    r = star_radius(V, lmax, sigma, seed)
    return V * r[:, None], F


def decimated_star(n_verts: int, lmax: int, sigma: float, seed: int, base_subdiv: int = 6):
    """Icosphere resampled by random vertex decimation to ``n_verts`` vertices,
    re-triangulated as the convex hull of the kept unit directions, then lifted to
    the star surface of ``seed``."""
    from scipy.spatial import ConvexHull  # host-side data preparation only

    V, _ = icosphere(base_subdiv)
    rng = np.random.default_rng(seed + 7919)
    keep = np.sort(rng.choice(V.shape[0], size=min(n_verts, V.shape[0]), replace=False))
    D = V[keep]
    hull = ConvexHull(D)
    F = _orient_outward(D, hull.simplices.astype(np.int64))
    r = star_radius(D, lmax, sigma, seed)
    return D * r[:, None], F.astype(np.int32)


# --------------------------------------------------------- varifold representation

def varifold_of(verts: np.ndarray, elems: np.ndarray):
    """(centres (E, D), unit normals/tangents (E, D), areas/lengths (E,)) of a mesh,
    as ``landmarksToVarifoldKernel`` computes them."""
    D = verts.shape[1]
    if D == 3:
        q0, q1, q2 = verts[elems[:, 0]], verts[elems[:, 1]], verts[elems[:, 2]]
        cen = (q0 + q1 + q2) / 3.0
        n = np.cross(q1 - q0, q2 - q0)
        ln = np.linalg.norm(n, axis=1)
        return cen, n / ln[:, None], 0.5 * ln
    q0, q1 = verts[elems[:, 0]], verts[elems[:, 1]]
    cen = 0.5 * (q0 + q1)
    t = q1 - q0
    ln = np.linalg.norm(t, axis=1)
    return cen, t / ln[:, None], ln
