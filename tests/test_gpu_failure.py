"""Failure detection without a GPU fault: a device wait that nothing can complete
gives up after its bound, the host reads the error status, and the device stays
usable (the same bounded grid barrier guards the persistent sweeps and the L-BFGS
cycle)."""
import ctypes as C

import pytest

from conftest import golden, problem_from, rel

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_device_stays_usable():
    from lddmm_b200 import _lib, api

    ms = C.c_double()
    rc = _lib.lib.lddmm_wait_selftest(0, 1, C.byref(ms))
    assert rc == -4, _lib.lib.lddmm_last_error()          # LDDMM_ERR_TIMEOUT
    assert 1.0 < ms.value < 30000.0, ms.value
    assert b"gave up" in _lib.lib.lddmm_last_error()
    rc = _lib.lib.lddmm_wait_selftest(0, 0, C.byref(ms))
    assert rc == 0 and ms.value < 1000.0
    # the device still computes correctly after the timed-out kernel
    z = golden("circle2square_objgrd")
    f, g = api.objgrd(problem_from(z), z["alp"])
    assert abs(f - float(z["f"])) / abs(float(z["f"])) < 1e-5
    assert rel(g, z["g"]) < 1e-5
