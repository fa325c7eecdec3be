"""Host-side statistics of the varifold sweep's distance culling.

The varifold sweep (Gaussian centre kernel, k = 2^-|x|^2 in scaled centre
coordinates x = c sqrt(log2 e) / cenKnlWidth) tests every (64-row tile, aligned
32-column block) pair of a problem once: the block is skipped when the bounding box
of its scaled centres lies farther than squared distance 64 from the box of the
tile's 64 rows.  Which blocks survive depends only on the geometry and on the
elements' storage order (which the library may change to a Morton order, see
``spatial_order``), not on the launch shape, so the share of pair interactions that
the sweep evaluates can be restated here exactly (up to the FP32 rounding of the
boxes) for rooflines and tests.
"""
from __future__ import annotations

import numpy as np

CULL_R2 = 64.0  # squared scaled distance of the cut-off (centre factors below 2^-64)
TILE = 64       # rows per tile
BLOCK = 32      # columns per block


def _pad(n: int) -> int:
    return -(-n // TILE) * TILE


def _block_boxes(cen: np.ndarray, ok: np.ndarray, scale: float, D: int):
    """(lo, hi) per 32-element block of the padded element list; padding is left out
    (an all-padding block has an empty box) and an element whose centre, direction or
    weight is not finite (``ok`` false) widens its block's box to all of space, as the
    device does."""
    n = cen.shape[0]
    npad = _pad(n)
    c = np.zeros((npad, 3), np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        c[:n, :D] = (cen * scale).astype(np.float32)
    real = (np.arange(npad) < n)[:, None]
    fin = np.isfinite(c).all(axis=1, keepdims=True)
    fin[:n, 0] &= ok
    lo = np.where(real, np.where(fin, c, -np.inf), np.inf).reshape(-1, BLOCK, 3).min(axis=1)
    hi = np.where(real, np.where(fin, c, np.inf), -np.inf).reshape(-1, BLOCK, 3).max(axis=1)
    return lo, hi


def spatial_order(cen: np.ndarray):
    """The library's storage order of a 3D surface's elements (``spatial_order`` in
    lddmm_b200.cu): the elements sorted along a Morton curve of their centres (10 bits
    per axis over the set's bounding cube, stable) when that shrinks the summed extent
    of the 32-element blocks' boxes below 0.8 of the given order's, else None (keep
    the given order)."""
    n = cen.shape[0]
    if n < 64:
        return None
    with np.errstate(invalid="ignore"):
        lo, hi = cen.min(axis=0), cen.max(axis=0)
        span = float((hi - lo).max())
    if not (span > 0.0) or not np.isfinite(span):
        return None
    with np.errstate(invalid="ignore"):
        u = (cen - lo) / span * 1023.0
    u = np.where(u > 0.0, u, 0.0)
    m = np.minimum(u, 1023.0).astype(np.uint32)
    code = np.zeros(n, np.uint64)
    for b in range(10):
        for d in range(3):
            code |= ((m[:, d].astype(np.uint64) >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + d)
    perm = np.argsort(code, kind="stable")

    def extent(c):
        tot = 0.0
        for b0 in range(0, n, BLOCK):
            blk = c[b0:b0 + BLOCK]
            tot += float((blk.max(axis=0) - blk.min(axis=0)).sum())
        return tot

    with np.errstate(invalid="ignore"):
        return perm if extent(cen[perm]) < 0.8 * extent(cen) else None


def varifold_kept_fraction(P, nde: np.ndarray | None = None) -> float | None:
    """Share of the varifold sweep's padded Ed x (Ed + Et) pair interactions that it
    evaluates with the deformed surface at landmark positions ``nde`` (default: the
    source, i.e. zero momenta).  None for a centre kernel without culling."""
    if P.cen_type != "G":
        return None
    D = P.ini_nde.shape[1]
    q = P.ini_nde if nde is None else np.asarray(nde, dtype=np.float64)
    scale = float(np.float32(np.sqrt(np.log2(np.e)) / P.cen_width))
    Ed, Et = P.elm_vtx.shape[0], P.tgt_cen.shape[0]
    elm = np.asarray(P.elm_vtx)
    tcen = np.asarray(P.tgt_cen, dtype=np.float64)
    tdir, tvol = np.asarray(P.tgt_dir), np.asarray(P.tgt_vol).reshape(-1)
    if D == 3:  # the device's storage order, chosen at the source geometry
        dp = spatial_order(P.ini_nde[elm].mean(axis=1))
        tp = spatial_order(tcen)
        if dp is not None:
            elm = elm[dp]
        if tp is not None:
            tcen, tdir, tvol = tcen[tp], tdir[tp], tvol[tp]
    v = q[elm]
    with np.errstate(invalid="ignore", divide="ignore"):
        if D == 3:
            nrm = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
        else:
            nrm = v[:, 1] - v[:, 0]
        nrm = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    dok = np.isfinite(nrm).all(axis=1)
    tok = np.isfinite(tdir).all(axis=1) & np.isfinite(tvol)
    dlo, dhi = _block_boxes(v.mean(axis=1), dok, scale, D)
    tlo, thi = _block_boxes(tcen, tok, scale, D)
    clo, chi = np.concatenate([dlo, tlo]), np.concatenate([dhi, thi])
    rlo = np.fmin(dlo[0::2], dlo[1::2])
    rhi = np.fmax(dhi[0::2], dhi[1::2])
    kept = 0
    with np.errstate(invalid="ignore"):
        for t0 in range(0, rlo.shape[0], 256):
            a, b = rlo[t0:t0 + 256, None, :], rhi[t0:t0 + 256, None, :]
            # fmax ignores a NaN operand (inf - inf), as the device's fmaxf does
            gap = np.fmax(np.float32(0.0), np.fmax(clo[None] - b, a - chi[None]))
            kept += int(((gap * gap).sum(axis=2) <= CULL_R2).sum())
    return kept * TILE * BLOCK / (_pad(Ed) * (_pad(Ed) + _pad(Et)))
