"""The mixed form (FP32 line factor and solve, FP32 Krylov basis; FP64 residual, J.v,
state update, Hessenberg least squares and forces) against FP64, on the device.

The reference has only FP64 (its float32 path was removed), so its FP64 outputs are the
only pin the mixed form has.  Three checks, each with its error bound stated:

* the FP32 line solve against the reference's FP64 solve: within 1e-4 relative;
* one Newton step of the mixed form from the reference's state: its update within
  1e-4 relative of the reference's FP64 update (GMRES stops at krylov_tol = 1e-2 of the
  initial residual either way; the FP32 basis moves the iterates, not the tolerance);
* a converging case run to convergence in the mixed form: CL, CD and CM within 1e-5 of
  the reference's converged FP64 run (|dCD| < 1e-5 is a tenth of a drag count), as the
  fixed point R = 0 is the FP64 residual's whatever the preconditioner's precision.
"""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from goldens import CASES, converged, load, rel

pytestmark = pytest.mark.gpu


def mixed_plan(name):
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load(name)
    imp = replace(case.implicit, precision="mixed")
    return z, case, plan, DevicePlan(plan, case.flow, case.numerics, imp), imp


@pytest.mark.parametrize("name", CASES)
def test_fp32_line_solve_against_the_fp64_solve(cuda, name):
    z, case, plan, dev, _ = mixed_plan(name)
    try:
        out = dev.precondition(z["rand0_U"], 25.0, z["rand0_prec_r"])
    finally:
        dev.close()
    err = rel(out, z["rand0_prec_z"])
    assert 0.0 < err < 1e-4


@pytest.mark.parametrize("name", ["o_euler", "c_laminar", "c_sa"])
def test_mixed_newton_update_against_the_fp64_update(cuda, name):
    z, case, plan, dev, _ = mixed_plan(name)
    try:
        dev.set_state(z["rand0_U"], 25.0, float("inf"))
        dev.newton_steps(1)
        U = dev.get_state()[0]
    finally:
        dev.close()
    dU, ref = U - z["rand0_U"], z["newton0_U"] - z["rand0_U"]
    assert rel(dU, ref) < 1e-4


@pytest.mark.parametrize("name", ["o_euler", "c_laminar"])
def test_mixed_form_converges_to_the_fp64_forces(cuda, name):
    from jaxrans_b200.solver import march
    z, case, plan = load(name)
    ref = converged(name)
    case = replace(case, implicit=replace(case.implicit, precision="mixed"))
    result = march(case, plan)
    assert result.history.reason == "converged"
    cl, cd, cm = ref["forces"][:3]
    assert abs(result.forces.cl - cl) < 1e-5
    assert abs(result.forces.cd - cd) < 1e-5
    assert abs(result.forces.cm - cm) < 1e-5
