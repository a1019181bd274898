#!/usr/bin/env python3
"""Generate the multi-block and pole 3D fixtures by running the reference solver itself.

Three grids (six cases), written as unformatted Plot3D files and read by the reference through its own
3D loader (``grid: file``, box patch rules), under the NumPy stand-in in
``tests/golden/jaxshim`` (as ``make_golden3d.py`` does):

* ``split``: the C-H wing block of ``ch_sa3d`` (``jaxrans_b200.grid3d.wing_block``) cut at
  two ``i`` stations into three blocks; the second stored with ``i`` and ``k`` reversed,
  the third with ``i`` and ``k`` swapped (left-handed as stored, so the loader reverses
  it).  The wake cut becomes an interface between the first and third blocks; SA RANS.
* ``wing4``: the four-block C-H grid of the swept, tapered wing with its tip region
  (``jaxrans_b200.grid3d.wing_ch_blocks``: wing and beyond-tip blocks, lower and upper
  halves; past the tip an elliptic cap, then a sheet facing itself), coarse; SA RANS.
* ``split_laminar``: the split grid, laminar with Sutherland's law, Roe with minmod;
  ``split_qcr``: the split grid with SA-noft2-QCR2000;
  ``wing4_euler``: the four-block wing inviscid, HLLC with unlimited MUSCL, kappa 1/3.
* ``pole``: a cylinder of cells round the z axis -- ``i`` the azimuth (an O seam), ``j``
  the radius from the axis (``j_min`` collapsed to a line: a pole), ``k`` along the
  axis -- with far field all round; inviscid.

For each: the assembled sides, the canvas, the reference's residual, first-order J.v and
wave speeds, and for the wings the line preconditioner, the forces and the surface
distributions.

    python tests/golden/make_golden_blocks3d.py

writes ``tests/golden/blocks3d.npz``.  The reference source tree is read from
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
from jaxrans.numerics.residual import make_residual  # noqa: E402
from jaxrans.post.forces import integrate_forces, surface  # noqa: E402
from jaxrans.solvers import preconditioners as pre  # noqa: E402

from jaxrans_b200.geometry import section_source  # noqa: E402
from jaxrans_b200.grid3d import wing_block, wing_ch_blocks, write_plot3d  # noqa: E402

sys.path.insert(0, str(HERE))
from make_golden3d import CASE, NUMERICAL, WING, perturbed, sides_record  # noqa: E402


def split_blocks() -> list[np.ndarray]:
    w = dict(WING)
    nodes = wing_block(section_source(w.pop("section")), **w).nodes
    a, b, c = nodes[:, :13], nodes[:, 12:25], nodes[:, 24:]
    return [a.copy(), b[:, ::-1, :, ::-1].copy(), c.transpose(0, 3, 2, 1).copy()]


def pole_blocks() -> list[np.ndarray]:
    theta = np.linspace(0.0, 2.0 * np.pi, 9)
    theta[-1] = 0.0
    r = np.array([0.0, 0.4, 0.9, 1.6, 2.5])
    z = np.linspace(-1.5, 1.5, 7)
    T, R, Z = np.meshgrid(theta, r, z, indexing="ij")
    return [np.stack([R * np.cos(T), R * np.sin(T), Z])]


POLE_CASE = {"general": {"case_name": "pole3d"},
             "domain": {"grid": "file", "file": "grid.x", "patches": [{"name": "farfield"}],
                        "reference_area": 1.0},
             "boundary_conditions": {"farfield": {"type": "far_field"}},
             "freestream": {"mach": 0.5, "alpha_deg": 10.0}}
POLE_NUMERICAL = {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "van_albada_smooth"},
                  "time_integration": {"solver": "implicit"}}


def split_case() -> dict:
    doc = json.loads(json.dumps(CASE))
    doc["general"]["case_name"] = "split3d"
    doc["domain"]["file"] = "grid.x"
    return doc


WING4 = {"section": "naca0012", "cells_airfoil": 24, "cells_wake": 6, "cells_normal": 10, "cells_span": 6,
         "cells_tip": 6, "wall_spacing": 1e-3, "far_field": 20.0, "semispan": 1.6, "taper": 0.6, "sweep_deg": 25.0,
         "cap_cells": 2, "span_far": 3.0}


def wing4_grid():
    w = dict(WING4)
    return wing_ch_blocks(section_source(w.pop("section")), **w)


def wing4_case() -> dict:
    g = wing4_grid()
    doc = json.loads(json.dumps(CASE))
    doc["general"]["case_name"] = "wing4"
    doc["domain"] = {"grid": "file", "file": "grid.x", "patches": g.patches, "reference_area": g.reference_area,
                     "reference_length": g.reference_length, "moment_centre": list(g.moment_centre)}
    doc["boundary_conditions"] = {"wall": {"type": "no_slip_wall"}, "farfield": {"type": "far_field"},
                                  "symmetry": {"type": "symmetry"}}
    return doc


def laminar_case() -> dict:
    """The split grid, laminar (Re 1e4, Sutherland's law at 540 R): 5 variables, viscous, no SA."""
    doc = split_case()
    doc["general"]["case_name"] = "split_laminar"
    doc.pop("turbulence")
    doc["freestream"] = {"mach": 0.5, "alpha_deg": 4.0, "reynolds": 1e4, "temperature": 540.0}
    doc["material_properties"] = {"dynamic_viscosity": "sutherland", "sutherland_temperature": 198.6}
    return doc


LAMINAR_NUMERICAL = {"convective_fluxes": {"riemann_solver": "roe", "limiter": "minmod"},
                     "time_integration": {"solver": "implicit"}}


def euler_case() -> dict:
    """The four-block wing, inviscid (slip walls), unlimited MUSCL with kappa = 1/3."""
    doc = wing4_case()
    doc["general"]["case_name"] = "wing4_euler"
    doc.pop("turbulence")
    doc["freestream"] = {"mach": 0.8, "alpha_deg": 2.5}
    doc["boundary_conditions"]["wall"] = {"type": "slip_wall"}
    return doc


def qcr_case() -> dict:
    """The split grid with SA-noft2-QCR2000 (the quadratic constitutive relation)."""
    doc = split_case()
    doc["general"]["case_name"] = "split_qcr"
    doc["turbulence"] = {"model": "sa_noft2_qcr"}
    return doc


EULER_NUMERICAL = {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "none", "muscl_kappa": 1.0 / 3.0},
                   "time_integration": {"solver": "implicit"}}

GRIDS = {"split": (split_blocks, split_case(), NUMERICAL), "pole": (pole_blocks, POLE_CASE, POLE_NUMERICAL),
         "wing4": (lambda: wing4_grid().blocks, wing4_case(), NUMERICAL),
         "split_laminar": (split_blocks, laminar_case(), LAMINAR_NUMERICAL),
         "wing4_euler": (lambda: wing4_grid().blocks, euler_case(), EULER_NUMERICAL),
         "split_qcr": (split_blocks, qcr_case(), NUMERICAL)}
WALLED = ("split", "wing4", "split_laminar", "wing4_euler", "split_qcr")


def main() -> int:
    out: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(11)
    for name, (make, case_doc, numerical) in GRIDS.items():
        blocks = make()
        with tempfile.TemporaryDirectory() as tmp:
            d = Path(tmp)
            write_plot3d(d / "grid.x", blocks)
            (d / "case.json").write_text(json.dumps(case_doc))
            (d / "numerical.json").write_text(json.dumps(numerical))
            case = load_case(str(d))
            atlas = case.grid()
        flow = case.flow
        op = make_residual(atlas, flow, case.numerics)
        jop = make_residual(atlas, flow, case.numerics, first_order=True, distance=op.distance)
        out[f"{name}_case_json"] = np.array(json.dumps({"case": case_doc, "numerical": numerical}))
        out[f"{name}_n_blocks"] = np.array(len(blocks))
        for b, nodes in enumerate(blocks):
            out[f"{name}_raw{b}"] = nodes
            out[f"{name}_sides{b}"] = np.array(json.dumps(sides_record(atlas.mesh[b])))
            out[f"{name}_nodes{b}"] = np.asarray(atlas.mesh[b].nodes)
        out[f"{name}_interior"] = np.asarray(atlas.interior)
        out[f"{name}_volume"] = np.asarray(atlas.grid.volume)
        if op.distance is not None:
            out[f"{name}_distance"] = np.asarray(op.distance)
        U = perturbed(op.initial_state(), 5, 1e-2)
        if numerical["convective_fluxes"]["riemann_solver"] == "roe":
            # a spanwise velocity everywhere: with none, V.n is zero to round-off on the faces
            # normal to the span, where Roe's |V.n| has its kink, and the tangent there is
            # decided by the sign of round-off
            U = np.asarray(U).copy()
            U[2] = U[2] + 2e-2 * U[0] * np.random.default_rng(9).uniform(-1.0, 1.0, U[0].shape)
            U = jnp.asarray(U)
        out[f"{name}_U"] = np.asarray(U)
        out[f"{name}_R2"] = np.asarray(op.residual(U))
        R1, jvp = jax.linearize(jop.residual, U)
        out[f"{name}_R1"] = np.asarray(R1)
        v = np.where(atlas.interior, rng.standard_normal(U.shape), 0.0)
        out[f"{name}_v"] = v
        out[f"{name}_Jv"] = np.asarray(jvp(jnp.asarray(v)))
        lam = op.wave_speeds(U)
        for a in range(3):
            out[f"{name}_lam{a}"] = np.asarray(lam[a])
        if name in WALLED:
            cfl = jnp.asarray(25.0)
            prepare = pre.get_preconditioner("line_j")(atlas, flow.gamma, op.viscosity, op.model, op.distance)
            r = np.where(atlas.interior, rng.standard_normal(U.shape), 0.0)
            out[f"{name}_prec_r"] = r
            out[f"{name}_prec_z"] = np.asarray(prepare(U, lam, cfl)(jnp.asarray(r)))
            f = integrate_forces(U, atlas, flow, case.grid_spec.force_reference())
            out[f"{name}_forces"] = np.array([f.cl, f.cd, f.cm, f.cd_friction])
            for key, values in surface(U, atlas, flow).items():
                out[f"{name}_surface_{key}"] = np.asarray(values)
        print(f"{name}: {len(blocks)} blocks, {atlas.shape} canvas, {atlas.cells} cells")
    np.savez_compressed(HERE / "blocks3d.npz", **out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
