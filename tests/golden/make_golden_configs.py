#!/usr/bin/env python3
"""Generate golden fixtures on the benchmark workloads' own grids by running the
reference solver itself.

The grids are this package's workloads (``jaxrans_b200.workloads``): the 2D Euler O-grid
of 257 x 65 nodes (``o_euler_257``), the SA C-grid of 385 x 97 nodes (``c_sa_385``) and the
uneven SA C-grid of 513 x 129 nodes of the batched polar (``c_sa_513``).  Each grid is
written as a formatted Plot3D file and read by the reference through ``"grid": "file"``
(its own reader, assembly, loop naming and atlas), with the workload's case documents,
under the NumPy stand-in for JAX in ``tests/golden/jaxshim``.  Saved per workload: the
reference's blocks and sides, its freestream state, and its outputs on two states --

* ``sin``: U0 (1 + 1e-3 sin(k)) (the state ``scripts/benchmark.py`` times);
* ``rand0``: U0 (1 + 1e-2 u), u uniform on [-1, 1) from ``np.random.default_rng(0)``;

R2, R1, the exact J.v, the wave speeds and the line_j solve (the vectors v and r are
standard normals from fixed seeds, zero off the interior; the tests draw them again).
With ``--converge NAME`` the workload is also run to convergence by the reference and its
forces saved (``<name>_converged.npz``).

    JAXRANS_REFERENCE=<reference checkout> python tests/golden/make_golden_configs.py [names]

writes ``tests/golden/<name>.npz``.
"""

from __future__ import annotations

import argparse
import copy
import json
import os
import sys
import tempfile
import time
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
from jaxrans.post.forces import integrate_forces  # noqa: E402
from jaxrans.solvers import preconditioners as pre  # noqa: E402
from jaxrans import simulation  # noqa: E402

from jaxrans_b200.gridfile import write_plot3d_2d  # noqa: E402
from jaxrans_b200.workloads import WORKLOADS, workload  # noqa: E402

NAMES = ("o_euler_257", "c_sa_385", "c_sa_513")
# the arrays kept per workload and state (the fixtures stay a few MB each)
KEEP = {
    "o_euler_257": {"sin": ("R2", "R1", "Jv", "lam", "prec_z"), "rand0": ("R2", "Jv")},
    "c_sa_385": {"sin": ("R2", "R1", "Jv", "lam", "prec_z"), "rand0": ("R2", "Jv")},
    "c_sa_513": {"sin": ("R2", "prec_z")},
}
# seeds of the vectors the tests draw again: (state, what) -> seed
SEEDS = {("sin", "v"): 11, ("sin", "r"): 12, ("rand0", "v"): 13, ("rand0", "r"): 14}
CFL = 25.0


def masked_normal(seed: int, shape, interior) -> np.ndarray:
    return np.where(interior, np.random.default_rng(seed).standard_normal(shape), 0.0)


def sides_record(block) -> dict:
    from jaxrans.mesh.block import Interface, SIDES
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


def reference_case(name: str, directory: Path):
    """The workload's grid as a Plot3D file and its documents, loaded by the reference."""
    case_doc, num_doc = copy.deepcopy(WORKLOADS[name])
    ours = workload(name)
    blocks = ours.grid_spec.build(Path("."))
    write_plot3d_2d(directory / "grid.p2dfmt", [(b.x, b.y) for b in blocks])
    case_doc["domain"] = {"grid": "file", "file": "grid.p2dfmt", "patches": []}
    (directory / "case.json").write_text(json.dumps(case_doc))
    (directory / "numerical.json").write_text(json.dumps(num_doc))
    return load_case(str(directory)), case_doc, num_doc


def generate(name: str, converge: bool) -> None:
    started = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        case, case_doc, num_doc = reference_case(name, Path(tmp))
        atlas = case.grid()
    flow, numerics = case.flow, case.numerics
    op = make_residual(atlas, flow, numerics)
    jop = make_residual(atlas, flow, numerics, first_order=True, distance=op.distance)
    out: dict[str, np.ndarray] = {"case_json": np.array(json.dumps({"case": case_doc, "numerical": num_doc}))}
    mesh = atlas.mesh
    out["n_blocks"] = np.array(len(mesh))
    for b, block in enumerate(mesh):
        out[f"block{b}_x"] = np.asarray(block.x_node)
        out[f"block{b}_y"] = np.asarray(block.y_node)
        out[f"block{b}_sides"] = np.array(json.dumps(sides_record(block)))
    interior = np.asarray(atlas.interior)
    U0 = op.initial_state()
    out["U_inf"] = np.asarray(U0)[(slice(None),) + (0,) * (U0.ndim - 1)]
    assert np.all(np.asarray(U0) == out["U_inf"].reshape((-1,) + (1,) * (U0.ndim - 1)))
    rng = np.random.default_rng(0)
    states = {"sin": U0 * (1.0 + 1e-3 * jnp.sin(jnp.arange(U0.size).reshape(U0.shape))),
              "rand0": jnp.asarray(np.asarray(U0) * (1.0 + 1e-2 * rng.uniform(-1.0, 1.0, U0.shape)))}
    prepare = pre.get_preconditioner("line_j")(atlas, flow.gamma, op.viscosity, op.model, op.distance)
    for label, keep in KEEP[name].items():
        U = jnp.asarray(states[label])
        if "R2" in keep:
            out[f"{label}_R2"] = np.asarray(op.residual(U))
            out[f"{label}_norm"] = np.asarray(op.norm(op.residual(U)))
        if "R1" in keep or "Jv" in keep:
            R1, jvp = jax.linearize(jop.residual, U)
            if "R1" in keep:
                out[f"{label}_R1"] = np.asarray(R1)
            if "Jv" in keep:
                v = masked_normal(SEEDS[(label, "v")], U.shape, interior)
                out[f"{label}_Jv"] = np.asarray(jvp(jnp.asarray(v)))
        if "lam" in keep or "prec_z" in keep:
            lam = op.wave_speeds(U)
            if "lam" in keep:
                out[f"{label}_lam_i"], out[f"{label}_lam_j"] = np.asarray(lam[0]), np.asarray(lam[1])
            if "prec_z" in keep:
                r = masked_normal(SEEDS[(label, "r")], U.shape, interior)
                out[f"{label}_prec_z"] = np.asarray(prepare(U, lam, jnp.asarray(CFL))(jnp.asarray(r)))
        forces = integrate_forces(U, atlas, flow, case.grid_spec.force_reference())
        out[f"{label}_forces"] = np.array([forces.cl, forces.cd, forces.cm, forces.cd_friction, forces.fx, forces.fy])
        print(f"{name} {label}: {', '.join(keep)} ({time.time() - started:.0f} s)", flush=True)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(f"{name}: {atlas.shape} canvas, {atlas.cells} cells -> {name}.npz ({time.time() - started:.0f} s)")

    if converge:
        started = time.time()
        result = simulation.run(case, grid=atlas)
        f = result.forces
        conv = {"residual": result.history.residual, "reason": np.array(result.history.reason),
                "iterations": np.array(result.history.n_iters),
                "forces": np.array([f.cl, f.cd, f.cm, f.cd_friction, f.fx, f.fy])}
        np.savez_compressed(HERE / f"{name}_converged.npz", **conv)
        print(f"{name}: {result.history.summary()}; CL {f.cl:.10f} CD {f.cd:.10f} CM {f.cm:.10f} "
              f"({time.time() - started:.0f} s)")


def main() -> int:
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("names", nargs="*", default=list(NAMES))
    p.add_argument("--converge", action="store_true", help="also run each workload to convergence")
    args = p.parse_args()
    for name in args.names:
        generate(name, args.converge)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
