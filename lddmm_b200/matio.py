"""MATLAB .mat data in the reference's variable names and layouts (scipy.io).

The reference's MATLAB examples keep a source surface and a target varifold in .mat
files and pass them to ``LDDMM`` (MATLAB/examples/sphere2cube/run_sphere2cube.m:4-13):
``sphereData.mat`` holds ``iniNdeMat`` (dim x N) and ``elmVtxMat`` ((2|3) x E,
1-based), ``cubeData.mat`` holds ``tgtCenPosMat`` and ``tgtUniDirMat`` (dim x E_t)
and ``tgtElmVolVec`` (1 x E_t).  ``LDDMM`` returns ``ndeStk`` (dim x N x timeNum) and
``vlcStk`` (dim x N x (timeNum - 1)) (Cpp/src/LDDMM.m).  This module reads such files
into the arguments of :func:`lddmm_b200.api.LDDMM`, builds a target varifold from a
target mesh (run_circle2square.m:21-24 computes it inline), and writes results back
under the same names.
"""
from __future__ import annotations

import numpy as np

from .shapes import varifold_of


def load(path: str) -> dict:
    """The variables of one .mat file (MATLAB's ``load``), header entries dropped."""
    import scipy.io as sio

    return {k: v for k, v in sio.loadmat(path).items() if not k.startswith("__")}


def target_varifold(tgtNdeMat, tgtElmVtxMat) -> dict:
    """tgtCenPosMat, tgtUniDirMat (dim x E_t) and tgtElmVolVec (1 x E_t) of a target
    mesh given as tgtNdeMat (dim x N_t) and tgtElmVtxMat ((2|3) x E_t, 1-based):
    element centres, unit normals (3D) / unit tangents (2D) and areas / lengths."""
    v = np.asarray(tgtNdeMat, dtype=np.float64).T
    e = np.asarray(tgtElmVtxMat).T.astype(np.int64) - 1
    cen, drc, vol = varifold_of(v, e)
    return {"tgtCenPosMat": cen.T, "tgtUniDirMat": drc.T, "tgtElmVolVec": vol[None, :]}


def dis_obj(source: dict, target: dict, cenKnlType: str, cenKnlWidth: float,
            dirKnlType: str, dirKnlWidth: float, disWgt: float) -> dict:
    """The ``disObj`` of run_sphere2cube.m:9-18 from a loaded source (``elmVtxMat``)
    and target (``tgtCenPosMat``, ``tgtUniDirMat``, ``tgtElmVolVec``)."""
    return {"dfmElmVtxMat": source["elmVtxMat"], "tgtCenPosMat": target["tgtCenPosMat"],
            "tgtElmVolVec": target["tgtElmVolVec"], "tgtUniDirMat": target["tgtUniDirMat"],
            "cenKnlType": cenKnlType, "cenKnlWidth": cenKnlWidth, "dirKnlType": dirKnlType,
            "dirKnlWidth": dirKnlWidth, "disWgt": disWgt}


def save_result(path: str, result, **extra) -> None:
    """Write ``ndeStk``, ``vlcStk`` and ``alpStk`` of an :func:`lddmm_b200.api.LDDMM`
    result (MATLAB layouts: dim x N x timeNum, dim x N x (timeNum - 1)), plus any
    ``extra`` variables, to a .mat file."""
    import scipy.io as sio

    out = {"ndeStk": np.asarray(result.ndeStk), "vlcStk": np.asarray(result.vlcStk),
           "alpStk": np.asarray(result.alpStk)}
    out.update(extra)
    sio.savemat(path, out)
