"""The device's bounded waits.  The staged line solve waits on an mbarrier for its bulk
copy with a limit; here a wait that no copy completes must run out, report
JR_ETIMEOUT / JR_STATUS_WAIT_LIMIT, and leave the context usable -- no fault, no hang
(the failure is made by arming a barrier that nothing completes)."""

from __future__ import annotations

import ctypes as C

import pytest

from test_gpu_parity import device_plan, row_rel

pytestmark = pytest.mark.gpu


def test_a_wait_that_nothing_completes_runs_out(cuda):
    from jaxrans_b200.native import JR_EINVAL, JR_ETIMEOUT, JR_STATUS_WAIT_LIMIT, load_library
    lib = load_library()
    status = C.c_int32(-1)
    assert lib.jr_wait_limit_check(1000, C.byref(status)) == JR_ETIMEOUT
    assert status.value == JR_STATUS_WAIT_LIMIT
    assert b"ran out" in lib.jr_last_error()
    assert lib.jr_wait_limit_check(0, None) == JR_EINVAL
    # the context still answers: the residual of a reference state through a plan
    z, case, plan, dev = device_plan("c_sa")
    assert row_rel(dev.residual(z["sin_U"]), z["sin_R2"]) < 1e-12
