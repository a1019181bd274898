"""The 3D plan (canvas, ghost stages, chains, walls, wall distance) of a C-H wing block,
against the reference's own 3D atlas of the same grid (tests/golden/ch_sa3d.npz, made by
tests/golden/make_golden3d.py: the reference read the block as a Plot3D file and
assembled it from the coordinates and box patch rules)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from jaxrans_b200.geometry import section_source
from jaxrans_b200.grid3d import SIDES_3D, Cut3, read_plot3d, wing_block, write_plot3d
from jaxrans_b200.plan3d import build_plan3d, metrics3d

GOLDEN = Path(__file__).resolve().parent / "golden" / "ch_sa3d.npz"
KINDS = {"wall": "no_slip_wall", "farfield": "far_field", "root": "symmetry", "tip": "symmetry"}


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="module")
def block(golden):
    w = json.loads(str(golden["wing_json"]))
    return wing_block(section_source(w.pop("section")), **w).with_kinds(KINDS)


@pytest.fixture(scope="module")
def plan(block):
    return build_plan3d([block])


def test_generated_block_is_the_reference_grid(golden, block):
    assert np.array_equal(block.nodes, golden["nodes"])
    sides = json.loads(str(golden["sides"]))
    for side in SIDES_3D:
        mine = []
        for r in block.sides[side]:
            if isinstance(r, Cut3):
                mine.append(["interface", list(r.start), list(r.stop), r.block, r.side, list(r.origin),
                             list(r.axes), list(r.flip), list(r.period)])
            else:
                mine.append(["boundary", list(r.start), list(r.stop), r.name, r.kind])
        assert mine == sides[side], side


def test_plot3d_round_trip(tmp_path, block):
    write_plot3d(tmp_path / "w.x", [block.nodes, block.nodes[:, ::-1]])
    back = read_plot3d(tmp_path / "w.x")
    assert len(back) == 2 and np.array_equal(back[0], block.nodes) and np.array_equal(back[1], block.nodes[:, ::-1])


def test_face_vectors_of_every_cell_close(block):
    """S of a warped quadrilateral is half the cross product of its diagonals, so the
    six outward vectors of a cell sum to zero to round-off."""
    _, volume, faces = metrics3d(block.nodes)
    total = sum(np.diff(f, axis=1 + a) for a, f in enumerate(faces))
    scale = max(np.abs(f).max() for f in faces)
    assert np.abs(total).max() < 1e-14 * scale
    assert np.all(volume > 0.0)


def test_canvas_geometry_matches_the_reference(golden, plan):
    assert plan.shape == golden["interior"].shape
    assert np.array_equal(plan.interior, golden["interior"])
    assert np.array_equal(plan.volume, golden["volume"])
    for a in range(3):
        assert np.array_equal(plan.faces[a], golden[f"faces{a}"])
    assert np.array_equal(plan.centres, golden["centres"])
    assert np.array_equal(plan.neighbours, golden["neighbours"])


def test_ghost_stages_match_the_reference(golden, plan):
    assert len(plan.stages) == int(golden["n_stages"])
    for s, st in enumerate(plan.stages):
        assert np.array_equal(st.index, golden[f"stage{s}_index"])
        assert [c[0] for c in st.conditions] == json.loads(str(golden[f"stage{s}_kinds"]))
        for k, (kind, source, normal, mid) in enumerate(st.conditions):
            assert np.array_equal(source, golden[f"stage{s}_cond{k}_source"])
            assert np.array_equal(normal, golden[f"stage{s}_cond{k}_normal"])
            assert np.array_equal(mid, golden[f"stage{s}_cond{k}_midpoint"])


def test_chains_walls_and_distance_match_the_reference(golden, plan):
    for key in ("cells", "up_face", "up_sign", "down_face", "down_sign"):
        assert np.array_equal(getattr(plan.lines, key), golden[f"lines_{key}"]), key
    assert np.array_equal(plan.walls.cell, golden["walls_cell"])
    assert np.array_equal(plan.walls.family, golden["walls_family"])
    assert np.array_equal(plan.walls.face, golden["walls_face"])
    assert np.array_equal(plan.walls.into_fluid, golden["walls_into_fluid"])
    assert np.allclose(plan.distance, golden["distance"], rtol=1e-14, atol=0.0)


def test_ghost_records_reproduce_the_gather_fill(golden, plan):
    """The device runs each ghost stage as records (one per ghost the stage writes); run
    on the host with the oracle's conditions, they give the reference's gather fill."""
    import json as _json
    from jaxrans_b200.case import flow_conditions
    from jaxrans_b200.native3d import KIND3, records_of
    from oracle import numerics3d as n3
    flow = flow_conditions(_json.loads(str(golden["case_json"]))["case"])
    a = flow.alpha_rad
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma, flow.nu_tilde_ratio])
    model = n3.Model3(plan, q_inf, flow.gamma, "hllc", "van_albada_smooth", 0.0, flow.mu_inf,
                      flow.sutherland_ratio, True, plan.distance)
    q = n3.prim(golden["rand0_U"], flow.gamma)
    rec = records_of(plan)
    assert rec.counts.sum() == len(rec.ghost) and np.all(rec.ghost < plan.n_canvas)
    names = {code: name for name, code in KIND3.items()}
    flat = q.reshape(q.shape[0], -1).copy()
    at = 0
    for count in rec.counts:
        g, s, k, nrm = (x[at:at + count] for x in (rec.ghost, rec.source, rec.kind, rec.normal))
        new = flat.copy()
        for code in np.unique(k):
            m = k == code
            vals = flat[:, s[m]]
            new[:, g[m]] = vals if code == 0 else n3._condition(names[int(code)], vals, nrm[m].T, model)
        flat = new
        at += count
    assert np.array_equal(flat.reshape(q.shape), n3.fill_ghosts(q, model))
