"""The 3D device path (jr_residual3d, jr_jvp3d, the line solve, the Newton step, the
forces and the wall distance) against the reference's own 3D outputs on the C-H wing
fixture (tests/golden/ch_sa3d.npz) and the multi-block fixtures (tests/golden/blocks3d.npz)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from jaxrans_b200.case import flow_conditions
from jaxrans_b200.geometry import section_source
from jaxrans_b200.grid3d import wing_block
from jaxrans_b200.plan3d import build_plan3d

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ch_sa3d.npz"
KINDS = {"wall": "no_slip_wall", "farfield": "far_field", "root": "symmetry", "tip": "symmetry"}


@pytest.fixture(scope="module")
def device3d():
    from jaxrans_b200.native3d import DevicePlan3
    z = np.load(GOLDEN)
    w = json.loads(str(z["wing_json"]))
    doc = json.loads(str(z["case_json"]))
    plan = build_plan3d([wing_block(section_source(w.pop("section")), **w).with_kinds(KINDS)])
    flow = flow_conditions(doc["case"])
    a = flow.alpha_rad
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma,
                      flow.nu_tilde_ratio])
    cv = doc["numerical"]["convective_fluxes"]
    from jaxrans_b200.case import implicit_config
    imp = implicit_config(doc["numerical"])
    dev = DevicePlan3(plan, q_inf, flow.gamma, cv["riemann_solver"], cv["limiter"], 0.0, flow.mu_inf,
                      flow.sutherland_ratio, imp)
    yield z, dev
    dev.close()


def rows_rel(a, b):
    return max(float(np.abs(a[k] - b[k]).max() / max(np.abs(b[k]).max(), 1e-300)) for k in range(a.shape[0]))


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_residual3d_matches_the_reference(cuda, device3d, state):
    z, dev = device3d
    U = z[f"{state}_U"]
    assert rows_rel(dev.residual(U), z[f"{state}_R2"]) < 1e-12
    assert rows_rel(dev.residual(U, first_order=True), z[f"{state}_R1"]) < 1e-12


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_jvp3d_matches_the_reference(cuda, device3d, state):
    z, dev = device3d
    Jv, ref = dev.jvp(z[f"{state}_U"], z[f"{state}_v"]), z[f"{state}_Jv"]
    assert rows_rel(Jv[:5], ref[:5]) < 1e-12
    assert rows_rel(Jv[5:], ref[5:]) < 1e-10


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_wave_speeds3d_and_line_solve_match_the_reference(cuda, device3d, state):
    z, dev = device3d
    U = z[f"{state}_U"]
    for a, lam in enumerate(dev.wave_speeds(U)):
        assert np.allclose(lam, z[f"{state}_lam{a}"], rtol=1e-13, atol=0.0)
    zz = dev.precondition(U, 25.0, z[f"{state}_prec_r"])
    assert rows_rel(zz, z[f"{state}_prec_z"]) < 1e-10


def test_newton_steps3d_match_the_reference(cuda, device3d):
    z, dev = device3d
    U, cfl, res, hist = dev.newton_steps(z["rand0_U"], 3, 25.0)
    for k in range(3):
        assert np.isclose(hist[k], float(z[f"newton{k}_norm"]), rtol=1e-10, atol=0.0)
    assert rows_rel(U, z["newton2_U"]) < 1e-8
    assert np.isclose(cfl, float(z["newton2_cfl"]), rtol=1e-12)


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_forces3d_match_the_reference(cuda, device3d, state):
    z, dev = device3d
    area = json.loads(str(z["case_json"]))["case"]["domain"]["reference_area"]
    assert np.allclose(dev.forces(z[f"{state}_U"], area, 0.8, (0.25, 0.0, 0.0)), z[f"{state}_forces"],
                       rtol=1e-11, atol=1e-16)


BLOCKS = Path(__file__).resolve().parent / "golden" / "blocks3d.npz"


@pytest.fixture(scope="module")
def blocks3d(tmp_path_factory):
    """The multi-block and pole cases of tests/golden/blocks3d.npz loaded as case directories."""
    from jaxrans_b200.case import load_case
    from jaxrans_b200.grid3d import write_plot3d
    z = np.load(BLOCKS)
    out = {}
    for name in ("split", "wing4", "pole", "split_laminar", "wing4_euler", "split_qcr"):
        d = tmp_path_factory.mktemp(name)
        doc = json.loads(str(z[f"{name}_case_json"]))
        write_plot3d(d / "grid.x", [z[f"{name}_raw{b}"] for b in range(int(z[f"{name}_n_blocks"]))])
        (d / "case.json").write_text(json.dumps(doc["case"]))
        (d / "numerical.json").write_text(json.dumps(doc["numerical"]))
        case = load_case(d)
        out[name] = (case, case.grid())
    return z, out


@pytest.mark.parametrize("name", ["split", "wing4", "pole", "split_laminar", "wing4_euler", "split_qcr"])
def test_blocks3d_residual_and_jvp_on_the_device(cuda, blocks3d, name):
    from jaxrans_b200.solver3d import device3_for
    z, cases = blocks3d
    case, plan = cases[name]
    dev = device3_for(case, plan)
    try:
        inside = plan.interior
        U = z[f"{name}_U"]
        for got, ref, tol in ((dev.residual(U), z[f"{name}_R2"], 1e-12),
                              (dev.residual(U, first_order=True), z[f"{name}_R1"], 1e-12),
                              (dev.jvp(U, z[f"{name}_v"]), z[f"{name}_Jv"], 1e-10)):
            for k in range(got.shape[0]):
                err = np.abs(got[k][inside] - ref[k][inside]).max() / max(np.abs(ref[k][inside]).max(), 1e-300)
                assert err < tol, (k, err)
    finally:
        dev.close()


def test_run_marches_a_3d_grid_file(cuda, blocks3d):
    from dataclasses import replace
    from jaxrans_b200.solver import run
    _, cases = blocks3d
    case, plan = cases["pole"]
    result = run(replace(case, block_iters=2, numerics=replace(case.numerics, max_iters=4)), plan)
    assert 2 <= result.history.n_iters <= 4 and np.all(np.isfinite(result.history.residual))
    assert result.U.shape == (5,) + plan.shape


def test_wall_distance_on_the_device(cuda, blocks3d):
    """jr_wall_distance3d against the reference's distance and the plan's NumPy distance."""
    from jaxrans_b200.native3d import wall_distance_device
    z, cases = blocks3d
    for name in ("split", "wing4"):
        _, plan = cases[name]
        points = np.moveaxis(plan.centres[:, 1:-1, 1:-1, 1:-1], 0, -1)[plan.interior]
        got = wall_distance_device(points, plan.walls.quads.corners)
        assert np.allclose(got, z[f"{name}_distance"][plan.interior], rtol=1e-12, atol=1e-15)


def test_mixed_line_solve3d_on_the_device(cuda, device3d):
    """The FP32 line factor and apply (implicit.precision = mixed) within FP32 of FP64."""
    from dataclasses import replace
    from jaxrans_b200.native3d import DevicePlan3
    z, dev = device3d
    imp = replace(dev.implicit, precision="mixed")
    U, r = z["rand0_U"], z["rand0_prec_r"]
    exact = dev.precondition(U, 25.0, r)
    mixed_dev = DevicePlan3(dev.plan, dev.q_inf, dev.gamma, dev.flux, dev.limiter, 0.0, dev.mu_inf, dev.sutherland,
                            imp)
    try:
        mixed = mixed_dev.precondition(U, 25.0, r)
    finally:
        mixed_dev.close()
    err = max(float(np.abs(mixed[k] - exact[k]).max() / np.abs(exact[k]).max()) for k in range(exact.shape[0]))
    assert 0.0 < err < 1e-4


def test_make_residual_on_a_3d_plan(cuda, blocks3d):
    """``make_residual`` on a 3D plan: the reference's operator surface over the 3D kernels."""
    from jaxrans_b200.residual import make_residual
    z, cases = blocks3d
    case, plan = cases["wing4"]
    op = make_residual(plan, case.flow, case.numerics)
    inside = plan.interior
    R = op.residual(z["wing4_U"])
    for k in range(R.shape[0]):
        ref = z["wing4_R2"][k][inside]
        assert np.abs(R[k][inside] - ref).max() <= 1e-12 * np.abs(ref).max()
    U0 = op.initial_state()
    assert U0.shape == (6,) + plan.shape and np.isfinite(op.norm(op.residual(U0)))


def test_time_kernels3d_leaves_the_results_alone(cuda, device3d):
    """jr_time_kernels3d times the residual, J.v and line preconditioner on its own work
    vectors: every time is positive, and the residual at the same state is unchanged."""
    z, dev = device3d
    U = z["sin_U"]
    before = dev.residual(U)
    ms = dev.time_kernels(U, 2)
    assert set(ms) == {"residual3d", "jvp3d", "line_precondition3d"}
    assert all(v > 0.0 for v in ms.values())
    assert np.array_equal(dev.residual(U), before)
