"""The allocation-free kernel sum, lddmm_multiply_kernel_noalloc, against the existing
entry point lddmm_multiply_kernel and against the compiled reference's kernel sums.

The allocation-free variant exists for callers that cannot let the library call
cudaMalloc/cudaFree: a MEX function operating on MATLAB gpuArray data owned by
MATLAB's allocator, a framework whose caching allocator owns the GPU, or a host loop
that cannot take the device-wide synchronisation of cudaFree.  Its buffers are the
caller's (allocated here by torch, in the test); its working set is a fixed array in
the library, limited to LDDMM_NOALLOC_MAX_POINTS landmarks.

Calls in a row of growing and shrinking sizes: a call must see neither the previous
call's leftovers in the shared array nor a work list that is not yet written (the
first call of a process starts from a zeroed array; a call with more tiles than every
earlier one reads list entries no earlier call wrote).  This file is collected last
and passes alone or after the others.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

TOL = 1e-5  # FP32 kernel sums vs the existing entry point, as in the parity tests
MAX_POINTS = 32768  # LDDMM_NOALLOC_MAX_POINTS in include/lddmm_b200.h


def _call(L, dim, n, q, a, order, width, v):
    return L.lddmm_multiply_kernel_noalloc(dim, n, C.c_void_p(q.data_ptr()),
                                           C.c_void_p(a.data_ptr()), order, width,
                                           C.c_void_p(v.data_ptr()), None)


def _noalloc(q, a, order, width):
    import torch

    from lddmm_b200 import _lib

    n, dim = q.shape
    dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    da = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dv = torch.full_like(dq, float("nan"))
    rc = _call(_lib.lib, dim, n, dq, da, order, width, dv)
    assert rc == 0, _lib.lib.lddmm_last_error()
    torch.cuda.synchronize()
    return dv.cpu().numpy()


def _relmax(v, ref):
    return float(np.max(np.abs(v - ref)) / np.max(np.abs(ref)))


# sizes rise and fall: 5000 then 300 (fewer tiles), then 20000 (more tiles than any
# earlier call), 2D Matern, and the largest size allowed
CASES = ((5000, 3, 1, 0.4), (300, 3, -1, 0.5), (257, 2, -1, 0.3), (20000, 3, -1, 0.3),
         (900, 2, 3, 0.25), (1200, 2, 0, 0.3), (MAX_POINTS, 3, -1, 0.3))


def test_noalloc_matches_existing_entry_point_in_a_row():
    from lddmm_b200 import api

    rng = np.random.default_rng(0)
    for n, dim, order, width in CASES:
        q = rng.uniform(-1.0, 1.0, size=(n, dim))
        a = rng.normal(size=(n, dim))
        ref = api.multiplyKernel(q, a, order, width)  # existing entry point
        for _ in range(2):  # the same call twice: the second sees the first's leftovers
            err = _relmax(_noalloc(q, a, order, width), ref)
            assert err < TOL, (n, dim, order, err)


def test_noalloc_matches_reference_kernel_sums():
    """Against the compiled reference's multiplyKernel (tests/golden/kernels_3d.npz),
    every 3D kernel order."""
    z = golden("kernels_3d")
    w = float(z["width"])
    for key, order in (("v_g", -1), ("v_m0", 0), ("v_m1", 1), ("v_m2", 2), ("v_m3", 3),
                       ("v_m4", 4)):
        err = _relmax(_noalloc(z["q"], z["a"], order, w), z[key])
        assert err < TOL, (key, err)


_FIRST_CALL = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch
from tests.test_zz_no_alloc import _noalloc
from lddmm_b200 import api
rng = np.random.default_rng(7)
q = rng.uniform(-1.0, 1.0, size=(6000, 3))
a = rng.normal(size=(6000, 3))
v = _noalloc(q, a, -1, 0.4)          # the first library call of this process
ref = api.multiplyKernel(q, a, -1, 0.4)
err = float(np.max(np.abs(v - ref)) / np.max(np.abs(ref)))
print("ERR", err)
sys.exit(0 if err < 1e-5 else 1)
"""


def test_noalloc_first_call_of_a_process():
    """The first call in a fresh process, with many tiles, before any other library
    call: the shared array is still all zeros, so a work list read before it is
    written would show."""
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([ROOT, os.path.join(ROOT, "tests")] +
                                        ([env["PYTHONPATH"]] if env.get("PYTHONPATH") else []))
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, ROOT], capture_output=True,
                       text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch

    from lddmm_b200 import _lib

    L = _lib.lib
    buf = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    rc = _call(L, 3, MAX_POINTS + 1, buf, buf, -1, 0.5, buf)
    assert rc == -1  # LDDMM_ERR_ARG
    assert b"LDDMM_NOALLOC_MAX_POINTS" in L.lddmm_last_error()
