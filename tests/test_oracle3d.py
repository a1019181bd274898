"""The 3D oracle (oracle.numerics3d) against the reference's own 3D residual, exact
first-order JVP, wave speeds and norm on the C-H wing fixture (tests/golden/ch_sa3d.npz,
made by tests/golden/make_golden3d.py from the reference's sources)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from jaxrans_b200.case import flow_conditions
from jaxrans_b200.geometry import section_source
from jaxrans_b200.grid3d import wing_block
from jaxrans_b200.plan3d import build_plan3d
from oracle import numerics3d as n3

GOLDEN = Path(__file__).resolve().parent / "golden" / "ch_sa3d.npz"
KINDS = {"wall": "no_slip_wall", "farfield": "far_field", "root": "symmetry", "tip": "symmetry"}


@pytest.fixture(scope="module")
def setup():
    z = np.load(GOLDEN)
    w = json.loads(str(z["wing_json"]))
    doc = json.loads(str(z["case_json"]))
    plan = build_plan3d([wing_block(section_source(w.pop("section")), **w).with_kinds(KINDS)])
    flow = flow_conditions(doc["case"])
    a = flow.alpha_rad
    # x-z incidence, y along the span (core/state.py:107-140)
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma,
                      flow.nu_tilde_ratio])
    cv = doc["numerical"]["convective_fluxes"]
    model = n3.Model3(plan, q_inf, flow.gamma, cv["riemann_solver"], cv["limiter"], 0.0, flow.mu_inf,
                      flow.sutherland_ratio, True, plan.distance)
    return z, model


def rows_rel(a, b):
    return max(float(np.abs(a[k] - b[k]).max() / max(np.abs(b[k]).max(), 1e-300)) for k in range(a.shape[0]))


def test_freestream_canvas(setup):
    z, model = setup
    assert np.array_equal(n3.initial_state(model), z["U0"])


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_residuals_and_jvp_match_the_reference(setup, state):
    z, model = setup
    U = z[f"{state}_U"]
    R2 = n3.residual(U, model)
    assert rows_rel(R2, z[f"{state}_R2"]) < 1e-14
    assert rows_rel(n3.residual(U, model, first_order=True), z[f"{state}_R1"]) < 1e-14
    assert rows_rel(n3.jvp(U, z[f"{state}_v"], model), z[f"{state}_Jv"]) < 1e-13
    assert np.isclose(n3.norm(R2, model), float(z[f"{state}_norm"]), rtol=1e-14, atol=0.0)


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_wave_speeds_match_the_reference(setup, state):
    z, model = setup
    lam = n3.wave_speeds(z[f"{state}_U"], model)
    for a in range(3):
        assert np.allclose(lam[a], z[f"{state}_lam{a}"], rtol=1e-14, atol=0.0)
    assert np.allclose(n3.cell_sum(lam) / 25.0, z[f"{state}_vdt"], rtol=1e-14, atol=0.0)


def test_freestream_is_preserved_off_the_wall(setup):
    """A uniform state leaves no residual away from the wall and its ghosts (the face
    vectors of every cell close)."""
    z, model = setup
    R = n3.residual(n3.initial_state(model), model)
    plan = model.plan
    off = plan.interior & (plan.distance > 0.5)
    assert np.abs(R[:5][:, off]).max() < 1e-12


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_chain_blocks_and_preconditioner_match_the_reference(setup, state):
    """5x5 mean-flow chain blocks, scalar SA chain blocks and the line_j solve at CFL
    25 (src/jaxrans/solvers/preconditioners.py:209-306)."""
    from oracle import implicit3d as i3
    z, model = setup
    U = z[f"{state}_U"]
    lam = n3.wave_speeds(U, model)
    for name, blocks in (("flow", i3.chain_blocks_flow(U, lam, 25.0, model)),
                         ("sa", i3.chain_blocks_sa(U, lam, 25.0, model))):
        for part, ref in zip(blocks, ("lower", "diag", "upper")):
            assert np.allclose(part, z[f"{state}_{name}_{ref}"], rtol=1e-13, atol=0.0), (name, ref)
    zz = i3.precondition(U, lam, 25.0, model)(z[f"{state}_prec_r"])
    assert rows_rel(zz, z[f"{state}_prec_z"]) < 1e-13
    # cyclic reduction and block Thomas agree
    zt = i3.precondition(U, lam, 25.0, model, solver="thomas")(z[f"{state}_prec_r"])
    assert rows_rel(zt, zz) < 1e-10


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_forces_match_the_reference(setup, state):
    from oracle import forces3d as f3
    z, model = setup
    area = json.loads(str(z["case_json"]))["case"]["domain"]["reference_area"]
    f = f3.forces(z[f"{state}_U"], model, area, 0.8, (0.25, 0.0, 0.0))
    assert np.allclose(f, z[f"{state}_forces"], rtol=1e-12, atol=1e-17)


def _implicit_config(doc):
    from jaxrans_b200.case import implicit_config
    return implicit_config(doc["numerical"])


def test_gmres_and_newton_steps_match_the_reference(setup):
    """One right-preconditioned GMRES solve of the Newton system and three Newton steps
    from the 'rand0' state at CFL 25 (src/jaxrans/solvers/implicit.py:84-168)."""
    from oracle import implicit3d as i3
    from oracle.implicit import NewtonState, gmres_right
    z, model = setup
    config = _implicit_config(json.loads(str(z["case_json"])))
    U = z["rand0_U"]
    R = n3.residual(U, model)
    lam = n3.wave_speeds(U, model)
    vdt = n3.cell_sum(lam) / 25.0
    dU, action = gmres_right(lambda d: vdt[None] * d + n3.jvp(U, d, model), -R,
                             i3.precondition(U, lam, 25.0, model), config.krylov_subspace,
                             config.krylov_restarts, config.krylov_tol)
    assert rows_rel(dU, z["gmres_dU"]) < 1e-9
    assert rows_rel(action, z["gmres_action"]) < 1e-9
    state = NewtonState(U, 25.0, np.inf)
    for k in range(3):
        state, norm = i3.newton_step(state, model, config)
        assert np.isclose(norm, float(z[f"newton{k}_norm"]), rtol=1e-12, atol=0.0)
        assert rows_rel(state.U, z[f"newton{k}_U"]) < 1e-13
        assert np.isclose(state.cfl, float(z[f"newton{k}_cfl"]), rtol=1e-12)


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_coupled_line_solve_is_the_dense_6x6_block_solve(setup, state):
    """The coupled (6x6) line blocks -- the SA row also coupled to the neighbours' mean
    flow -- solved by mean flow first, then the SA chains with r_sa - C z_flow, against a
    dense solve of each chain's assembled block-tridiagonal matrix (CPU)."""
    from oracle import implicit3d as i3
    z, model = setup
    U, r = z[f"{state}_U"], z[f"{state}_prec_r"]
    lam = n3.wave_speeds(U, model)
    fl, fd, fu = i3.chain_blocks_flow(U, lam, 25.0, model)
    sl, sd, su = i3.chain_blocks_sa(U, lam, 25.0, model)
    cl, cu = i3.chain_coupling_sa(U, model)
    assert np.abs(cl).max() > 0.0 and np.abs(cu).max() > 0.0
    got = i3.precondition_coupled(U, lam, 25.0, model)(r)
    lines = model.plan.lines
    flat_r = r.reshape(6, -1)
    flat_got = got.reshape(6, -1)
    for line in range(lines.cells.shape[0]):
        cells = lines.cells[line][lines.cells[line] >= 0]
        L = len(cells)
        M = np.zeros((6 * L, 6 * L))
        for k in range(L):
            def put(col, flow, cpl, sa):
                M[6 * k:6 * k + 5, 6 * col:6 * col + 5] = flow
                if cpl is not None:
                    M[6 * k + 5, 6 * col:6 * col + 5] = cpl
                M[6 * k + 5, 6 * col + 5] = sa
            put(k, fd[k, line], None, sd[k, line, 0, 0])
            if k > 0:
                put(k - 1, fl[k, line], cl[k, line], sl[k, line, 0, 0])
            if k + 1 < L:
                put(k + 1, fu[k, line], cu[k, line], su[k, line, 0, 0])
        x = np.linalg.solve(M, flat_r[:, cells].T.reshape(-1)).reshape(L, 6).T
        assert np.allclose(flat_got[:, cells], x, rtol=1e-9, atol=1e-12 * np.abs(x).max())
