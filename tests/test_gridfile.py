"""Grid files through the case loader (``"grid": "file"``): Plot3D read and assembled
(right-handedness, face matching into cuts, loop naming, patch rules) to the same plan
as the reference's own loader builds (tests/golden/file_grids.npz, made by
tests/golden/make_golden_file.py), and the oracle residual on it equal to the
reference's."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from goldens import oracle_model
from jaxrans_b200.case import parse_case
from jaxrans_b200.gridfile import read_plot3d_2d, write_plot3d_2d
from oracle import numerics as nm

GOLDEN = Path(__file__).resolve().parent / "golden" / "file_grids.npz"
NAMES = ("c_single", "c_split", "o_rules")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def load(golden, name, tmp_path):
    doc = json.loads(str(golden[f"{name}_case_json"]))
    blocks = [(golden[f"{name}_block{b}_x"], golden[f"{name}_block{b}_y"])
              for b in range(int(golden[f"{name}_n_blocks"]))]
    write_plot3d_2d(tmp_path / "grid.p2dfmt", blocks)
    case = parse_case(doc["case"], doc["numerical"], tmp_path)
    return case, case.grid()


@pytest.mark.parametrize("name", NAMES)
def test_file_grid_plan_matches_the_reference(golden, name, tmp_path):
    case, plan = load(golden, name, tmp_path)
    assert np.array_equal(plan.interior, golden[f"{name}_interior"])
    assert np.array_equal(plan.volume, golden[f"{name}_volume"])
    assert np.array_equal(plan.faces_i, golden[f"{name}_faces_i"])
    assert np.array_equal(plan.faces_j, golden[f"{name}_faces_j"])
    assert np.array_equal(plan.centres, golden[f"{name}_centres"])
    assert np.array_equal(plan.neighbours, golden[f"{name}_neighbours"])
    for key in ("cells", "up_face", "up_sign", "down_face", "down_sign"):
        assert np.array_equal(getattr(plan.chains, key), golden[f"{name}_lines_{key}"]), key
    assert np.array_equal(plan.walls.cell, golden[f"{name}_walls_cell"])


@pytest.mark.parametrize("name", NAMES)
def test_residual_on_a_file_grid_matches_the_reference(golden, name, tmp_path):
    case, plan = load(golden, name, tmp_path)
    R = nm.residual(golden[f"{name}_U"], oracle_model(case, plan))
    ref = golden[f"{name}_R2"]
    for k in range(R.shape[0]):
        assert np.abs(R[k] - ref[k]).max() <= 1e-13 * max(np.abs(ref[k]).max(), 1e-300)


def test_plot3d_formats_round_trip(tmp_path):
    """Formatted and unformatted, single and multi-block, and a thin 3D extrusion."""
    from jaxrans_b200.grid3d import write_plot3d
    rng = np.random.default_rng(3)
    a = (rng.random((5, 4)), rng.random((5, 4)))
    b = (rng.random((3, 6)), rng.random((3, 6)))
    write_plot3d_2d(tmp_path / "g.p2dfmt", [a, b])
    back = read_plot3d_2d(tmp_path / "g.p2dfmt")
    assert all(np.array_equal(p, q) for blk, ref in zip(back, [a, b]) for p, q in zip(blk, ref))
    # a 2D grid extruded one cell along z, unformatted
    x, y = a
    nodes = np.stack([np.stack([x, x], -1), np.stack([y, y], -1), np.stack([0 * x, 0 * x + 1.0], -1)])
    write_plot3d(tmp_path / "g.x", [nodes])
    (xx, yy), = read_plot3d_2d(tmp_path / "g.x")
    assert np.array_equal(xx, x) and np.array_equal(yy, y)


def test_a_tangled_3d_grid_file_is_a_case_error(tmp_path):
    """A 3D file goes to the 3D assembly; cells of both volume signs are refused."""
    from jaxrans_b200.case import CaseError
    from jaxrans_b200.grid3d import write_plot3d
    nodes = np.random.default_rng(0).random((3, 4, 5, 6))
    write_plot3d(tmp_path / "w.x", [nodes])
    doc = {"case": {"general": {"case_name": "w"},
                    "domain": {"grid": "file", "file": "w.x", "reference_area": 1.0},
                    "freestream": {"mach": 0.5}},
           "numerical": {"time_integration": {"solver": "implicit"}}}
    case = parse_case(doc["case"], doc["numerical"], tmp_path)
    with pytest.raises(CaseError, match="non-positive volume"):
        case.grid()
