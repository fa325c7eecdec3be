import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    so = os.path.join(ROOT, "oracle", "liblddmm_oracle.so")
    src = os.path.join(ROOT, "oracle", "lddmm_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    from oracle.oracle import Oracle

    return Oracle()


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def problem_from(z, **over):
    from lddmm_b200.problem import Problem

    s = z["scalars"]
    ct, dt = (str(x) for x in z["types"])
    kw = dict(knl_order=int(s[0]), knl_width=float(s[1]), time_num=int(s[2]),
              time_stp=float(s[3]), cen_type=ct, cen_width=float(s[4]), dir_type=dt,
              dir_width=float(s[5]), dis_wgt=float(s[6]))
    kw.update(over)
    return Problem(z["ini_nde"], z["elm_vtx"], z["tgt_cen"], z["tgt_dir"], z["tgt_vol"],
                   elm_ifo=z["elm_ifo"], **kw)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
