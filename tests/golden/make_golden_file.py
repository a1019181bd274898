#!/usr/bin/env python3
"""Generate the grid-file fixtures by running the reference's own loader.

The grids are C- and O-grids of the 2D fixtures (tests/golden/<case>.npz), written as
formatted Plot3D files by this package's writer (``jaxrans_b200.gridfile``): one case as a
single block, one split into two blocks at mid-i with the second stored in reversed i
order.  The reference reads them through ``"grid": "file"`` (its Plot3D reader and
assembly: right-handedness, face matching, loop naming, patch rules) and its atlas
and residual are saved, under the NumPy stand-in in ``tests/golden/jaxshim``.

    python tests/golden/make_golden_file.py

writes ``tests/golden/file_grids.npz``.
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

import jax.numpy as jnp  # noqa: E402  (the stand-in)
from jaxrans.case.loader import load_case  # noqa: E402
from jaxrans.numerics.residual import make_residual  # noqa: E402

from jaxrans_b200.gridfile import write_plot3d_2d  # noqa: E402

# name: (source fixture, split, patch rules)
GRIDS = {
    "c_single": ("c_sa", False, []),
    "c_split": ("c_sa", True, []),
    "o_rules": ("o_euler", False, [{"name": "body", "x_min": -0.5, "x_max": 1.5, "y_min": -0.5, "y_max": 0.5},
                                   {"name": "outer"}]),
}


def blocks_of(z, split: bool):
    x, y = z["block0_x"], z["block0_y"]
    if not split:
        return [(x, y)]
    m = (x.shape[0] - 1) // 2
    return [(x[:m + 1], y[:m + 1]), (x[m:][::-1].copy(), y[m:][::-1].copy())]


def main() -> int:
    out = {}
    for name, (source, split, rules) in GRIDS.items():
        z = np.load(HERE / f"{source}.npz")
        doc = json.loads(str(z["case_json"]))
        case_doc = json.loads(json.dumps(doc["case"]))
        keep = {k: v for k, v in case_doc["domain"].items() if k in ("reference_length", "moment_centre")}
        case_doc["domain"] = {"grid": "file", "file": "grid.p2dfmt", "patches": rules, **keep}
        if rules:
            bc = case_doc.setdefault("boundary_conditions", {})
            bc["body"] = {"type": "slip_wall" if "reynolds" not in case_doc["freestream"] else "no_slip_wall"}
            bc["outer"] = {"type": "far_field"}
        blocks = blocks_of(z, split)
        with tempfile.TemporaryDirectory() as tmp:
            d = Path(tmp)
            write_plot3d_2d(d / "grid.p2dfmt", blocks)
            (d / "case.json").write_text(json.dumps(case_doc))
            (d / "numerical.json").write_text(json.dumps(doc["numerical"]))
            case = load_case(str(d))
            atlas = case.grid()
        op = make_residual(atlas, case.flow, case.numerics)
        out[f"{name}_case_json"] = np.array(json.dumps({"case": case_doc, "numerical": doc["numerical"]}))
        out[f"{name}_n_blocks"] = np.array(len(blocks))
        for b, (x, y) in enumerate(blocks):
            out[f"{name}_block{b}_x"], out[f"{name}_block{b}_y"] = x, y
        out[f"{name}_interior"] = np.asarray(atlas.interior)
        out[f"{name}_volume"] = np.asarray(atlas.grid.volume)
        out[f"{name}_faces_i"] = np.asarray(atlas.grid.faces[0])
        out[f"{name}_faces_j"] = np.asarray(atlas.grid.faces[1])
        out[f"{name}_centres"] = np.asarray(atlas.centres)
        out[f"{name}_neighbours"] = np.asarray(atlas.neighbours)
        for key in ("cells", "up_face", "up_sign", "down_face", "down_sign"):
            out[f"{name}_lines_{key}"] = np.asarray(getattr(atlas.lines, key))
        out[f"{name}_walls_cell"] = atlas.walls.cell
        U0 = op.initial_state()
        U = U0 * (1.0 + 1e-3 * jnp.sin(jnp.arange(U0.size).reshape(U0.shape)))
        out[f"{name}_U"] = np.asarray(U)
        out[f"{name}_R2"] = np.asarray(op.residual(U))
        print(f"{name}: {len(blocks)} block(s), canvas {atlas.shape}")
    np.savez_compressed(HERE / "file_grids.npz", **out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
