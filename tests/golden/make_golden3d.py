#!/usr/bin/env python3
"""Generate the 3D golden fixture by running the reference solver itself.

The grid is this package's C-H wing block (``jaxrans_b200.grid3d.wing_block``: a swept,
tapered NACA 0012 wing spanning root to tip plane), written as a Plot3D file; the
reference reads it through its own 3D loader (``grid: file`` with box patch rules), so
its assembly, atlas, residual, linearisation, chain blocks, preconditioner and forces
all run on the reference's sources, unmodified, on top of the NumPy stand-in in
``tests/golden/jaxshim`` (as ``make_golden.py`` does for the 2D cases).

    python tests/golden/make_golden3d.py

writes ``tests/golden/ch_sa3d.npz``.  The reference source tree is read from
``$JAXRANS_REFERENCE`` (required).
"""

from __future__ import annotations

import json
import os
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
if "JAXRANS_REFERENCE" not in os.environ:
    raise SystemExit("set JAXRANS_REFERENCE to the reference source checkout (the directory holding src/jaxrans)")
REFERENCE = Path(os.environ["JAXRANS_REFERENCE"])
sys.path.insert(0, str(HERE / "jaxshim"))
sys.path.insert(1, str(REFERENCE / "src"))
sys.path.insert(2, str(ROOT / "jax-rans_b200"))

import numpy as np  # noqa: E402

import jax  # noqa: E402  (the stand-in)
import jax.numpy as jnp  # noqa: E402
from jaxrans.case.loader import load_case  # noqa: E402
from jaxrans.mesh.block3d import SIDES_3D, InterfaceRect  # noqa: E402
from jaxrans.numerics.residual import cell_wave_speed_sum, make_residual  # noqa: E402
from jaxrans.post.forces import integrate_forces  # noqa: E402
from jaxrans.solvers import implicit  # noqa: E402
from jaxrans.solvers import preconditioners as pre  # noqa: E402
from jaxrans.solvers.krylov import gmres_right  # noqa: E402

from jaxrans_b200.geometry import section_source  # noqa: E402
from jaxrans_b200.grid3d import wing_block, write_plot3d  # noqa: E402

# The wing (config 5's section, taper and sweep; a coarse grid) and its case.
WING = {"section": "naca0012", "cells_airfoil": 24, "cells_wake": 6, "cells_normal": 10, "cells_span": 4,
        "wall_spacing": 1e-3, "far_field": 20.0, "semispan": 2.0, "taper": 0.6, "sweep_deg": 25.0}
CASE = {"general": {"case_name": "ch_sa3d"},
        "domain": {"grid": "file", "file": "wing.x",
                   "patches": [{"name": "root", "y_max": 1e-9}, {"name": "tip", "y_min": 2.0 - 1e-9},
                               {"name": "wall", "x_min": -0.5, "x_max": 3.0, "z_min": -0.5, "z_max": 0.5},
                               {"name": "farfield"}],
                   "reference_area": 1.6, "reference_length": 0.8, "moment_centre": [0.25, 0.0, 0.0]},
        "boundary_conditions": {"wall": {"type": "no_slip_wall"}, "farfield": {"type": "far_field"},
                                "root": {"type": "symmetry"}, "tip": {"type": "symmetry"}},
        "freestream": {"mach": 0.8, "alpha_deg": 2.5, "reynolds": 1e7},
        "turbulence": {"model": "sa_noft2"}}
NUMERICAL = {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "van_albada_smooth"},
             "time_integration": {"solver": "implicit"}, "implicit": {"max_relative_update": 0.2},
             "convergence": {"max_iters": 100, "tol": 1e-10, "block_iters": 20}}


def sides_record(block) -> dict:
    out = {}
    for side in SIDES_3D:
        rects = []
        for r in block.sides.side(side):
            if isinstance(r, InterfaceRect):
                rects.append(["interface", list(r.start), list(r.stop), r.block, r.side, list(r.origin),
                              list(r.axes), [bool(f) for f in r.flip], list(r.period)])
            else:
                rects.append(["boundary", list(r.start), list(r.stop), r.patch, r.kind])
        out[side] = rects
    return out


def perturbed(U0, seed: int, amplitude: float):
    rng = np.random.default_rng(seed)
    return jnp.asarray(np.asarray(U0) * (1.0 + amplitude * rng.uniform(-1.0, 1.0, U0.shape)))


def main() -> int:
    w = dict(WING)
    block = wing_block(section_source(w.pop("section")), **w)
    out: dict[str, np.ndarray] = {}
    with tempfile.TemporaryDirectory() as tmp:
        d = Path(tmp)
        write_plot3d(d / "wing.x", [block.nodes])
        (d / "case.json").write_text(json.dumps(CASE))
        (d / "numerical.json").write_text(json.dumps(NUMERICAL))
        case = load_case(str(d))
        atlas = case.grid()
    flow, numerics = case.flow, case.numerics
    op = make_residual(atlas, flow, numerics)
    jop = make_residual(atlas, flow, numerics, first_order=True, distance=op.distance)
    out["wing_json"] = np.array(json.dumps(WING))
    out["case_json"] = np.array(json.dumps({"case": CASE, "numerical": NUMERICAL}))
    out["nodes"] = np.asarray(atlas.mesh[0].nodes)
    out["sides"] = np.array(json.dumps(sides_record(atlas.mesh[0])))
    out["interior"] = np.asarray(atlas.interior)
    out["volume"] = np.asarray(atlas.grid.volume)
    for a in range(3):
        out[f"faces{a}"] = np.asarray(atlas.grid.faces[a])
    out["centres"] = np.asarray(atlas.centres)
    out["neighbours"] = np.asarray(atlas.neighbours)
    out["n_stages"] = np.array(len(atlas.stages))
    for s, stage in enumerate(atlas.stages):
        out[f"stage{s}_index"] = np.asarray(stage.index)
        out[f"stage{s}_kinds"] = np.array(json.dumps([c[0] for c in stage.conditions]))
        for k, (kind, source, normal, midpoint) in enumerate(stage.conditions):
            out[f"stage{s}_cond{k}_source"] = np.asarray(source)
            out[f"stage{s}_cond{k}_normal"] = np.asarray(normal)
            out[f"stage{s}_cond{k}_midpoint"] = np.asarray(midpoint)
    for key in ("cells", "up_face", "up_sign", "down_face", "down_sign"):
        out[f"lines_{key}"] = np.asarray(getattr(atlas.lines, key))
    W = atlas.walls
    out["walls_cell"], out["walls_family"] = W.cell, W.family
    out["walls_face"], out["walls_into_fluid"] = W.face, W.into_fluid
    out["distance"] = np.asarray(op.distance)

    U0 = op.initial_state()
    out["U0"] = np.asarray(U0)
    states = {"sin": U0 * (1.0 + 1e-3 * jnp.sin(jnp.arange(U0.size).reshape(U0.shape))),
              "rand0": perturbed(U0, 0, 1e-2)}
    rng = np.random.default_rng(7)
    cfl = jnp.asarray(25.0)
    prepare = pre.get_preconditioner("line_j")(atlas, flow.gamma, op.viscosity, op.model, op.distance)
    reference = case.grid_spec.force_reference()
    for label, U in states.items():
        U = jnp.asarray(U)
        out[f"{label}_U"] = np.asarray(U)
        out[f"{label}_R2"] = np.asarray(op.residual(U))
        R1, jvp = jax.linearize(jop.residual, U)
        out[f"{label}_R1"] = np.asarray(R1)
        v = np.where(atlas.interior, rng.standard_normal(U.shape), 0.0)
        out[f"{label}_v"] = v
        out[f"{label}_Jv"] = np.asarray(jvp(jnp.asarray(v)))
        out[f"{label}_norm"] = np.asarray(op.norm(op.residual(U)))
        lam = op.wave_speeds(U)
        for a in range(3):
            out[f"{label}_lam{a}"] = np.asarray(lam[a])
        out[f"{label}_vdt"] = np.asarray(cell_wave_speed_sum(lam) / cfl)
        layout = pre.ChainLayout(atlas)
        n_flow = 2 + atlas.components
        lo, di, up = pre.flow_chain_blocks(U[:n_flow], lam, cfl, atlas, flow.gamma, layout)
        out[f"{label}_flow_lower"], out[f"{label}_flow_diag"], out[f"{label}_flow_upper"] = \
            np.asarray(lo), np.asarray(di), np.asarray(up)
        lo, di, up = pre.sa_chain_blocks(U, lam, cfl, atlas, flow.gamma, op.viscosity, op.model,
                                         op.distance, layout)
        out[f"{label}_sa_lower"], out[f"{label}_sa_diag"], out[f"{label}_sa_upper"] = \
            np.asarray(lo), np.asarray(di), np.asarray(up)
        r = np.where(atlas.interior, rng.standard_normal(U.shape), 0.0)
        out[f"{label}_prec_r"] = r
        out[f"{label}_prec_z"] = np.asarray(prepare(U, lam, cfl)(jnp.asarray(r)))
        f = integrate_forces(U, atlas, flow, reference)
        out[f"{label}_forces"] = np.array([f.cl, f.cd, f.cm, f.cd_friction])
    # One GMRES solve of the Newton system, and three Newton steps, at "rand0"
    config = case.implicit
    U = jnp.asarray(states["rand0"])
    residual = op.residual(U)
    _, jvp = jax.linearize(jop.residual, U)
    lam = op.wave_speeds(U)
    vdt = cell_wave_speed_sum(lam) / cfl
    dU, action = gmres_right(lambda d: vdt[None] * d + jvp(d), -residual, prepare(U, lam, cfl),
                             restart=config.krylov_subspace, maxiter=config.krylov_restarts,
                             tol=config.krylov_tol, return_action=True, action_from_arnoldi=True)
    out["gmres_dU"], out["gmres_action"] = np.asarray(dU), np.asarray(action)
    step = implicit.make_newton_step(op, config, jop)
    state = implicit.ImplicitState(U=U, cfl=cfl, residual_norm=jnp.asarray(np.inf))
    for k in range(3):
        state, norm = step(state)
        out[f"newton{k}_U"], out[f"newton{k}_cfl"] = np.asarray(state.U), np.asarray(state.cfl)
        out[f"newton{k}_norm"] = np.asarray(norm)
    np.savez_compressed(HERE / "ch_sa3d.npz", **out)
    print(f"ch_sa3d: {atlas.shape} canvas, {atlas.cells} cells -> ch_sa3d.npz")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
