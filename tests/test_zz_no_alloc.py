"""The allocation-free kernel sum, lddmm_multiply_kernel_noalloc, against the existing
entry point lddmm_multiply_kernel.

The allocation-free variant exists for callers that cannot let the library call
cudaMalloc/cudaFree: a MEX function operating on MATLAB gpuArray data owned by
MATLAB's allocator, a framework whose caching allocator owns the GPU, or a host loop
that cannot take the device-wide synchronisation of cudaFree.  Its buffers are the
caller's (allocated here by torch, in the test); its working set is a fixed array in
the library, limited to LDDMM_NOALLOC_MAX_POINTS landmarks.

Two calls in a row: the second, smaller one must not see the first call's leftovers in
the shared array.  This file is collected last and passes alone or after the others.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5  # FP32 kernel sums vs the existing entry point, as in the parity tests
MAX_POINTS = 32768  # LDDMM_NOALLOC_MAX_POINTS in include/lddmm_b200.h


def _call(L, dim, n, q, a, order, width, v):
    return L.lddmm_multiply_kernel_noalloc(dim, n, C.c_void_p(q.data_ptr()),
                                           C.c_void_p(a.data_ptr()), order, width,
                                           C.c_void_p(v.data_ptr()), None)


def test_noalloc_matches_existing_entry_point_twice():
    import torch

    from lddmm_b200 import _lib, api

    L = _lib.lib
    rng = np.random.default_rng(0)
    for n, dim, order, width in ((700, 3, 1, 0.4), (300, 3, -1, 0.5), (257, 2, -1, 0.3)):
        q = rng.uniform(-1.0, 1.0, size=(n, dim))
        a = rng.normal(size=(n, dim))
        ref = api.multiplyKernel(q, a, order, width)  # existing entry point
        dq = torch.from_numpy(q).cuda()
        da = torch.from_numpy(a).cuda()
        dv = torch.full_like(dq, float("nan"))
        rc = _call(L, dim, n, dq, da, order, width, dv)
        assert rc == 0, _lib.lib.lddmm_last_error()
        torch.cuda.synchronize()
        v = dv.cpu().numpy()
        err = np.max(np.abs(v - ref)) / np.max(np.abs(ref))
        assert err < TOL, (n, order, err)


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch

    from lddmm_b200 import _lib

    L = _lib.lib
    buf = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    rc = _call(L, 3, MAX_POINTS + 1, buf, buf, -1, 0.5, buf)
    assert rc == -1  # LDDMM_ERR_ARG
    assert b"LDDMM_NOALLOC_MAX_POINTS" in L.lddmm_last_error()
