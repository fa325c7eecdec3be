"""Probe kernels that give the rooflines their denominators (lddmm_pipe_peaks): the
FP32 FMA, packed FP32x2 FMA and ex2 (MUFU) throughput of the GPU."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_pipe_peaks_are_plausible():
    from lddmm_b200 import _lib

    out = (C.c_double * 3)()
    _lib.check(_lib.lib.lddmm_pipe_peaks(0, out))
    one = C.c_double()
    _lib.check(_lib.lib.lddmm_fp32_peak(0, C.byref(one)))
    fp32, fp32x2, ex2 = out[0], out[1], out[2]
    assert 10.0 < fp32 < 300.0 and 10.0 < fp32x2 < 600.0  # TFLOP/s
    assert 100.0 < ex2 < 1e5  # G results/s
    assert abs(fp32 - one.value) < 0.1 * one.value  # the same probe as lddmm_fp32_peak
