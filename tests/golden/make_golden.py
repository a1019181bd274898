#!/usr/bin/env python3
"""Generate the golden fixtures by running the reference solver itself.

The reference (giovannicatalani/jax-rans) is pure Python on JAX.  JAX is not
installed where the fixtures are made, so its sources run unmodified on top of
the NumPy stand-in in ``tests/golden/jaxshim`` (complex-step derivatives with
JAX's JVP rules).  Every array below is the reference's own output on small
generated grids; nothing here is used at run time by the library.

    PYTHONPATH=tests/golden/jaxshim:<reference>/src python tests/golden/make_golden.py [--converge]

writes ``tests/golden/<case>.npz`` (+ ``<case>_converged.npz`` with ``--converge``).
The reference source tree is read from ``$JAXRANS_REFERENCE`` (required).
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
if "JAXRANS_REFERENCE" not in os.environ:
    raise SystemExit("set JAXRANS_REFERENCE to the reference source checkout (the directory holding src/jaxrans)")
REFERENCE = Path(os.environ["JAXRANS_REFERENCE"])
sys.path.insert(0, str(HERE / "jaxshim"))
sys.path.insert(1, str(REFERENCE / "src"))

import numpy as np  # noqa: E402

import jax  # noqa: E402  (the stand-in)
import jax.numpy as jnp  # noqa: E402
from jaxrans.case.loader import parse_case  # noqa: E402
from jaxrans.mesh.block import Boundary, Interface, SIDES  # noqa: E402
from jaxrans.numerics.residual import cell_wave_speed_sum, make_residual  # noqa: E402
from jaxrans.post.forces import integrate_forces  # noqa: E402
from jaxrans.solvers import implicit  # noqa: E402
from jaxrans.solvers import preconditioners as pre  # noqa: E402
from jaxrans.solvers.krylov import gmres_right  # noqa: E402
from jaxrans import simulation  # noqa: E402

# The small cases: one per flow model, O- and C-grid topologies.
CASES = {
    "o_euler": (
        {"general": {"case_name": "o_euler"},
         "domain": {"grid": "o_grid", "airfoil": "naca0012", "cells_airfoil": 48, "cells_normal": 32,
                    "wall_spacing": 1e-3, "far_field": 20.0},
         "freestream": {"mach": 0.8, "alpha_deg": 1.25}},
        {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "van_albada"},
         "time_integration": {"solver": "implicit"},
         "convergence": {"max_iters": 3000, "tol": 1e-10, "forces_tol": None, "block_iters": 20}},
    ),
    "c_sa": (
        {"general": {"case_name": "c_sa"},
         "domain": {"grid": "c_grid", "airfoil": "naca4412", "cells_airfoil": 32, "cells_wake": 8,
                    "cells_normal": 16, "wall_spacing": 1e-4, "far_field": 20.0},
         "freestream": {"mach": 0.2, "alpha_deg": 8.0, "reynolds": 6e6},
         "turbulence": {"model": "sa_noft2"}},
        {"convective_fluxes": {"riemann_solver": "roe", "limiter": "minmod"},
         "time_integration": {"solver": "implicit"},
         "implicit": {"max_relative_update": 0.2, "krylov_subspace": 12},
         "convergence": {"max_iters": 4000, "tol": 1e-10, "forces_tol": None, "block_iters": 20}},
    ),
    "c_laminar": (
        {"general": {"case_name": "c_laminar"},
         "domain": {"grid": "c_grid", "airfoil": "naca0012", "cells_airfoil": 32, "cells_wake": 8,
                    "cells_normal": 16, "wall_spacing": 2e-3, "far_field": 20.0},
         "freestream": {"mach": 0.5, "alpha_deg": 2.0, "reynolds": 5000.0, "temperature": 288.0},
         "material_properties": {"dynamic_viscosity": "sutherland", "sutherland_temperature": 110.3}},
        {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "none"},
         "time_integration": {"solver": "implicit"},
         "convergence": {"max_iters": 3000, "tol": 1e-10, "forces_tol": None, "block_iters": 20}},
    ),
    "o_sa_qcr": (
        {"general": {"case_name": "o_sa_qcr"},
         "domain": {"grid": "o_grid", "airfoil": "naca2412", "cells_airfoil": 48, "cells_normal": 32,
                    "wall_spacing": 1e-4, "far_field": 20.0},
         "boundary_conditions": {"farfield": {"type": "far_field", "model": "point_vortex"}},
         "freestream": {"mach": 0.3, "alpha_deg": 4.0, "reynolds": 3e6},
         "turbulence": {"model": "sa_noft2_qcr"}},
        {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "van_albada_smooth"},
         "time_integration": {"solver": "implicit"},
         "implicit": {"max_relative_update": 0.2},
         "convergence": {"max_iters": 3000, "tol": 1e-10, "forces_tol": None, "block_iters": 20}},
    ),
}


def sides_record(block) -> list:
    """A block's side segments as plain lists (JSON)."""
    out = {}
    for side in SIDES:
        segs = []
        for seg in block.sides.side(side):
            if isinstance(seg, Interface):
                segs.append(["interface", seg.start, seg.stop, seg.block, seg.side, seg.partner_start,
                             bool(seg.reversed)])
            else:
                segs.append(["boundary", seg.start, seg.stop, seg.patch, seg.kind])
        out[side] = segs
    return out


def perturbed(U0, seed: int, amplitude: float):
    rng = np.random.default_rng(seed)
    return jnp.asarray(np.asarray(U0) * (1.0 + amplitude * rng.uniform(-1.0, 1.0, U0.shape)))


def generate(name: str, converge: bool) -> None:
    case_doc, num_doc = CASES[name]
    case = parse_case(json.loads(json.dumps(case_doc)), json.loads(json.dumps(num_doc)))
    atlas = case.grid()
    flow, numerics, config = case.flow, case.numerics, case.implicit
    op = make_residual(atlas, flow, numerics)
    jop = make_residual(atlas, flow, numerics, first_order=True, distance=op.distance)
    out: dict[str, np.ndarray] = {}
    out["case_json"] = np.array(json.dumps({"case": case_doc, "numerical": num_doc}))
    mesh = atlas.mesh
    out["n_blocks"] = np.array(len(mesh))
    for b, block in enumerate(mesh):
        out[f"block{b}_x"] = np.asarray(block.x_node)
        out[f"block{b}_y"] = np.asarray(block.y_node)
        out[f"block{b}_sides"] = np.array(json.dumps(sides_record(block)))
    # The reference's atlas (static plans)
    out["interior"] = np.asarray(atlas.interior)
    out["volume"] = np.asarray(atlas.grid.volume)
    out["faces_i"] = np.asarray(atlas.grid.faces[0])
    out["faces_j"] = np.asarray(atlas.grid.faces[1])
    out["centres"] = np.asarray(atlas.centres)
    out["neighbours"] = np.asarray(atlas.neighbours)
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
    out["walls_body"], out["walls_a"], out["walls_b"] = W.faces.body, W.faces.a, W.faces.b
    out["quarter_chord"] = np.asarray(atlas.quarter_chord)
    if op.distance is not None:
        out["distance"] = np.asarray(op.distance)

    U0 = op.initial_state()
    out["U0"] = np.asarray(U0)
    states = {"sin": U0 * (1.0 + 1e-3 * jnp.sin(jnp.arange(U0.size).reshape(U0.shape))),
              "rand0": perturbed(U0, 0, 1e-2)}
    rng = np.random.default_rng(7)
    cfl = jnp.asarray(25.0)
    prepare = pre.get_preconditioner("line_j")(atlas, flow.gamma, op.viscosity, op.model, op.distance)
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
        out[f"{label}_lam_i"], out[f"{label}_lam_j"] = np.asarray(lam[0]), np.asarray(lam[1])
        out[f"{label}_vdt"] = np.asarray(cell_wave_speed_sum(lam) / cfl)
        layout = pre.ChainLayout(atlas)
        n_flow = 2 + atlas.components
        lo, di, up = pre.flow_chain_blocks(U[:n_flow], lam, cfl, atlas, flow.gamma, layout)
        out[f"{label}_flow_lower"], out[f"{label}_flow_diag"], out[f"{label}_flow_upper"] = \
            np.asarray(lo), np.asarray(di), np.asarray(up)
        if op.model is not None:
            lo, di, up = pre.sa_chain_blocks(U, lam, cfl, atlas, flow.gamma, op.viscosity, op.model,
                                             op.distance, layout)
            out[f"{label}_sa_lower"], out[f"{label}_sa_diag"], out[f"{label}_sa_upper"] = \
                np.asarray(lo), np.asarray(di), np.asarray(up)
        r = np.where(atlas.interior, rng.standard_normal(U.shape), 0.0)
        out[f"{label}_prec_r"] = r
        out[f"{label}_prec_z"] = np.asarray(prepare(U, lam, cfl)(jnp.asarray(r)))
        forces = integrate_forces(U, atlas, flow, case.grid_spec.force_reference())
        out[f"{label}_forces"] = np.array([forces.cl, forces.cd, forces.cm, forces.cd_friction,
                                           forces.fx, forces.fy])

    # One GMRES solve of the Newton system, and three Newton steps, at "rand0"
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
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(f"{name}: {atlas.shape} canvas, {atlas.cells} cells -> {name}.npz")

    if converge:
        started = time.time()
        result = simulation.run(case, grid=atlas)
        f = result.forces
        conv = {"U": np.asarray(result.U), "residual": result.history.residual,
                "reason": np.array(result.history.reason), "iterations": np.array(result.history.n_iters),
                "forces": np.array([f.cl, f.cd, f.cm, f.cd_friction, f.fx, f.fy])}
        np.savez_compressed(HERE / f"{name}_converged.npz", **conv)
        print(f"{name}: {result.history.summary()}; CL {f.cl:.10f} CD {f.cd:.10f} CM {f.cm:.10f} "
              f"({time.time() - started:.0f} s)")


def main() -> int:
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("cases", nargs="*", default=list(CASES))
    p.add_argument("--converge", action="store_true", help="also run each case to convergence")
    args = p.parse_args()
    for name in args.cases:
        generate(name, args.converge)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
