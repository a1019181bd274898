"""Parity of the device path (through the C ABI) with the reference's own outputs.

Every comparison is against a golden array the reference produced
(``tests/golden/make_golden.py``), or the oracle where the golden holds none.
Tolerances (FP64): residuals 1e-12 relative to each row's largest entry (the
plain-path target); J.v 1e-12 on the mean-flow rows and 1e-10 on the SA row, whose
tangent in a near-uniform state is a difference of source terms O(1e3) larger than
itself (fused multiply-adds move it by 4e-11, plain multiplies by 1e-12); wave speeds 1e-13; the line solve 1e-10 (block cyclic reduction on the
device against the reference's: the same solve to round-off, amplified by the blocks'
conditioning); forces 1e-12.
"""

from __future__ import annotations

import numpy as np
import pytest

from goldens import CASES, converged, load, oracle_model, rel
from oracle import numerics as nm

pytestmark = pytest.mark.gpu


def device_plan(name, **implicit):
    from dataclasses import replace
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load(name)
    imp = replace(case.implicit, **implicit) if implicit else case.implicit
    return z, case, plan, DevicePlan(plan, case.flow, case.numerics, imp)


def row_rel(a, b):
    return max(float(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300)) for v in range(b.shape[0]))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_residual_matches_reference(cuda, name, state):
    z, case, plan, dev = device_plan(name)
    U = z[f"{state}_U"]
    assert row_rel(dev.residual(U), z[f"{state}_R2"]) < 1e-12
    assert row_rel(dev.residual(U, first_order=True), z[f"{state}_R1"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_jvp_matches_reference(cuda, name, state):
    z, case, plan, dev = device_plan(name)
    Jv, ref = dev.jvp(z[f"{state}_U"], z[f"{state}_v"]), z[f"{state}_Jv"]
    assert row_rel(Jv[:4], ref[:4]) < 1e-12
    if ref.shape[0] > 4:
        assert row_rel(Jv[4:], ref[4:]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_wave_speeds_match_reference(cuda, name):
    z, case, plan, dev = device_plan(name)
    li, lj = dev.wave_speeds(z["rand0_U"])
    interior = plan.interior
    # faces adjacent to a block cell
    live_i = np.zeros(li.shape, bool)
    live_i[:-1] |= interior
    live_i[1:] |= interior
    live_j = np.zeros(lj.shape, bool)
    live_j[:, :-1] |= interior
    live_j[:, 1:] |= interior
    assert rel(li[live_i], z["rand0_lam_i"][live_i]) < 1e-13
    assert rel(lj[live_j], z["rand0_lam_j"][live_j]) < 1e-13


@pytest.mark.parametrize("name", CASES)
def test_line_preconditioner_matches_reference(cuda, name):
    z, case, plan, dev = device_plan(name)
    out = dev.precondition(z["rand0_U"], 25.0, z["rand0_prec_r"])
    assert rel(out, z["rand0_prec_z"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_forces_match_reference(cuda, name):
    z, case, plan, dev = device_plan(name)
    f = dev.forces(z["rand0_U"])
    assert np.abs(f - z["rand0_forces"]).max() < 1e-12


@pytest.mark.parametrize("name", ["o_euler", "c_laminar", "c_sa"])
def test_newton_steps_track_reference(cuda, name):
    """Three steps from one state: the same updates to round-off (a restart decision
    could flip on round-off; these states are far from the tolerance).  Measured on a
    B200: norms within 1.5e-13, the state within 2.6e-14."""
    z, case, plan, dev = device_plan(name)
    dev.set_state(z["rand0_U"], 25.0, float("inf"))
    norms = dev.newton_steps(3)
    U, cfl, _, status = dev.get_state()
    for k in range(3):
        assert abs(norms[k] - float(z[f"newton{k}_norm"])) <= 1e-12 * float(z[f"newton{k}_norm"])
    assert rel(U, z["newton2_U"]) < 1e-12
    assert cfl == pytest.approx(float(z["newton2_cfl"]), rel=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_freestream_preserved_on_device(cuda, name):
    """|R| < 1e-12 away from the wall for the uniform freestream
    (the reference's tests/verification/test_freestream.py:49-113)."""
    z, case, plan, dev = device_plan(name)
    model = oracle_model(case, plan)
    U0 = nm.initial_state(model)
    for first in (False, True):
        R = dev.residual(U0, first_order=first)
        g = plan.g
        block = R[:4, g:plan.NI - g, g:plan.NJ - g]   # the mean flow (the SA source is not zero)
        away = block[:, :, 2:]                        # two cells off the wall (the MUSCL stencil)
        scale = max(1.0, float(np.abs(plan.faces_j).max()) * case.flow.mach)
        assert np.abs(away).max() < 1e-12 * scale
        assert np.abs(block[:, :, 0]).max() > 1e-8     # the wall does disturb a uniform flow


@pytest.mark.parametrize("name", ["o_euler", "c_sa", "c_laminar"])
def test_converged_forces_match_reference(cuda, name):
    """Run to the reference's convergence test and compare CL, CD, CM with the
    reference's converged run on the same grid (1e-6)."""
    ref = converged(name)
    if ref is None:
        pytest.skip("no converged golden")
    from jaxrans_b200.solver import march
    z, case, plan, dev = device_plan(name)
    result = march(case, plan, device=dev)
    assert result.history.reason in ("converged", "settled")
    f = result.forces
    assert abs(f.cl - ref["forces"][0]) < 1e-6
    assert abs(f.cd - ref["forces"][1]) < 1e-6
    assert abs(f.cm - ref["forces"][2]) < 1e-6


@pytest.mark.parametrize("name", CASES)
def test_wall_loads_match_oracle(cuda, name):
    """Per wall face: gauge pressure, area vector into the fluid and viscous force against
    the oracle's wall loads (the arithmetic the golden forces pin), 1e-12 of each column's
    largest entry."""
    import oracle
    z, case, plan, dev = device_plan(name)
    U = z["rand0_U"]
    got = dev.wall_loads(U)
    p, S, shear = oracle.wall_loads(U, oracle_model(case, plan))
    ref = np.column_stack([p, S[0], S[1], shear[0], shear[1]])
    for k in range(5):
        scale = max(np.abs(ref[:, k]).max(), 1e-300)
        assert np.abs(got[:, k] - ref[:, k]).max() <= 1e-12 * scale


@pytest.mark.parametrize("name", ["c_sa", "o_sa_qcr"])
def test_coupled_line_preconditioner_matches_oracle(cuda, name):
    """The coupled (5x5) line blocks -- jaxrans_b200's 5x5 form; the reference has the split
    form only -- against the oracle's coupled solve (itself checked against dense block
    solves), 1e-10 as the split solve."""
    from oracle import implicit as im
    z, case, plan, dev = device_plan(name, preconditioner="line_j_coupled")
    U, r = z["rand0_U"], z["rand0_prec_r"]
    model = oracle_model(case, plan)
    ref = im.precondition_coupled(U, nm.wave_speeds(U, model), 25.0, model)(r)
    out = dev.precondition(U, 25.0, r)
    assert rel(out, ref) < 1e-10


def test_coupled_form_converges_to_the_same_forces(cuda):
    """A preconditioner does not move the fixed point: the coupled form's converged
    forces are the split form's (the reference's converged run) to 1e-6."""
    from jaxrans_b200.solver import march
    ref = converged("c_sa")
    if ref is None:
        pytest.skip("no converged golden")
    z, case, plan, dev = device_plan("c_sa", preconditioner="line_j_coupled")
    result = march(case, plan, device=dev)
    assert result.history.reason in ("converged", "settled")
    assert abs(result.forces.cl - ref["forces"][0]) < 1e-6
    assert abs(result.forces.cd - ref["forces"][1]) < 1e-6


@pytest.mark.parametrize("name", CASES)
def test_norm_on_the_device_matches_reference(cuda, name):
    """ResidualOperator.norm on the device (jr_norm) against the reference's norm of its
    own residual (src/jaxrans/numerics/residual.py:237-240)."""
    from jaxrans_b200.residual import make_residual
    z, case, plan = load(name)
    op = make_residual(plan, case.flow, case.numerics)
    for state in ("sin", "rand0"):
        assert op.norm(z[f"{state}_R2"]) == pytest.approx(float(z[f"{state}_norm"]), rel=1e-13)
