""".mat input and output in the reference's variable names (CPU): the example data
layout of MATLAB/examples/sphere2cube/run_sphere2cube.m round-trips through a .mat
file into the problem that LDDMM solves, and results are written back under the
reference's names and shapes."""
from types import SimpleNamespace

import numpy as np
import pytest
import scipy.io as sio

from conftest import golden


def write_example(tmp_path, z):
    """sphereData.mat / cubeData.mat as the reference's example keeps them."""
    src = tmp_path / "sphereData.mat"
    tgt = tmp_path / "cubeData.mat"
    sio.savemat(src, {"iniNdeMat": z["ini_nde"].T, "elmVtxMat": (z["elm_vtx"] + 1).T})
    sio.savemat(tgt, {"tgtCenPosMat": z["tgt_cen"].T, "tgtUniDirMat": z["tgt_dir"].T,
                      "tgtElmVolVec": z["tgt_vol"][None, :]})
    return src, tgt


def test_mat_example_gives_the_fixture_problem(tmp_path):
    from lddmm_b200 import api, matio

    z = golden("sphere2cube_example")
    src, tgt = write_example(tmp_path, z)
    s, t = matio.load(src), matio.load(tgt)
    sc = z["scalars"]
    ct, dt = (str(x) for x in z["types"])
    d = matio.dis_obj(s, t, ct, float(sc[4]), dt, float(sc[5]), float(sc[6]))
    # timeEnd / timeStp as run_sphere2cube.m sets them; 1 x 1 arrays as loadmat gives
    P = api.problem_from_matlab(s["iniNdeMat"], d, np.array([[sc[0]]]), np.array([[sc[1]]]),
                                np.array([[1.0]]), np.array([[sc[3]]]))
    assert np.array_equal(P.ini_nde, z["ini_nde"])
    assert np.array_equal(P.elm_vtx, z["elm_vtx"])
    assert np.array_equal(P.tgt_cen, z["tgt_cen"])
    assert np.array_equal(P.tgt_dir, z["tgt_dir"])
    assert np.array_equal(P.tgt_vol, z["tgt_vol"])
    assert (P.knl_order, P.knl_width, P.time_num, P.time_stp) == (3, 0.25, int(sc[2]), 0.05)
    assert (P.cen_type, P.dir_type) == (ct, dt)
    assert (P.cen_width, P.dir_width, P.dis_wgt) == (float(sc[4]), float(sc[5]), float(sc[6]))


def test_target_varifold_from_mesh():
    from lddmm_b200 import matio, problem, shapes

    cv, cf = shapes.cube_surface(6, 1.0)
    t = matio.target_varifold(cv.T, (cf + 1).T)
    P = problem.sphere_to_cube(subdiv=1, cube_n=6, time_num=3)
    assert t["tgtCenPosMat"].shape == (3, cf.shape[0])
    assert t["tgtElmVolVec"].shape == (1, cf.shape[0])
    assert np.allclose(t["tgtCenPosMat"].T, P.tgt_cen, rtol=0, atol=1e-15)
    assert np.allclose(t["tgtUniDirMat"].T, P.tgt_dir, rtol=0, atol=1e-15)
    assert np.allclose(t["tgtElmVolVec"].ravel(), P.tgt_vol, rtol=0, atol=1e-15)


def test_save_result_names_and_shapes(tmp_path):
    from lddmm_b200 import matio

    rng = np.random.default_rng(0)
    r = SimpleNamespace(ndeStk=rng.normal(size=(3, 7, 5)), vlcStk=rng.normal(size=(3, 7, 4)),
                        alpStk=rng.normal(size=(3, 7, 4)))
    out = tmp_path / "result.mat"
    matio.save_result(out, r, knlWidth=0.25)
    back = matio.load(out)
    assert np.array_equal(back["ndeStk"], r.ndeStk)
    assert np.array_equal(back["vlcStk"], r.vlcStk)
    assert np.array_equal(back["alpStk"], r.alpStk)
    assert float(back["knlWidth"].ravel()[0]) == 0.25


@pytest.mark.gpu
def test_lddmm_from_mat_files(tmp_path):
    """The reference example's flow on .mat files: load the source and the target,
    LDDMM with loadmat-style (1 x 1 array) parameters, save the result; the same run
    as with plain Python values."""
    from lddmm_b200 import api, matio

    z = golden("sphere2cube_example")
    src, tgt = write_example(tmp_path, z)
    s, t = matio.load(src), matio.load(tgt)
    d = matio.dis_obj(s, t, "C", 0.1, "B", 0.0, 100.0)
    sio.savemat(tmp_path / "opt.mat", {"MaxIterations": 3.0, "OptimalityTolerance": 1e-2,
                                       "Wolfe1": 0.0, "Wolfe2": 0.5, "Columns": 10.0})
    opt = matio.load(tmp_path / "opt.mat")
    out = api.LDDMM(s["iniNdeMat"], None, d, np.array([[3.0]]), np.array([[0.25]]),
                    np.array([[1.0]]), np.array([[0.05]]), opt)
    ref = api.LDDMM(z["ini_nde"].T, None, dict(d, dfmElmVtxMat=(z["elm_vtx"] + 1).T), 3, 0.25,
                    1.0, 0.05, dict(MaxIterations=3, OptimalityTolerance=1e-2, Wolfe1=0.0,
                                    Wolfe2=0.5, Columns=10))
    assert np.array_equal(out.alpStk, ref.alpStk)
    matio.save_result(tmp_path / "result.mat", out)
    back = matio.load(tmp_path / "result.mat")
    assert back["ndeStk"].shape == (3, 600, 21)
    assert np.array_equal(back["ndeStk"], out.ndeStk)
