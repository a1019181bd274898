"""3D grid files with several blocks and with a pole, against the reference's own loader
and solver (tests/golden/blocks3d.npz, made by tests/golden/make_golden_blocks3d.py):

* the assembly (``jaxrans_b200.gridfile3d``) gives the reference's blocks and sides;
* a case directory on such a file loads (``load_case``) to a 3D plan on the reference's
  canvas;
* the 3D kernels' bodies, run on the host by the test harness, give the reference's
  residual, J.v, wave speeds, line preconditioner, forces and surface distributions
  across interfaces of every orientation and across a pole, for SA RANS (HLLC, smooth
  van Albada; with and without QCR2000), laminar flow with Sutherland's law (Roe, minmod) and inviscid flow
  (HLLC, unlimited MUSCL with kappa 1/3);
* ``solver3d.march3d`` drives blocks of Newton steps and the exit test over a device
  stand-in built on the same harness."""

from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from jaxrans_b200.case import CaseError, load_case
from jaxrans_b200.grid3d import SIDES_3D, Cut3, Rect3, write_plot3d
from jaxrans_b200.gridfile import PatchRule
from jaxrans_b200.gridfile3d import assemble3d, is_3d

GOLDEN = Path(__file__).resolve().parent / "golden" / "blocks3d.npz"
NAMES = ("split", "wing4", "pole", "split_laminar", "wing4_euler", "split_qcr")
WALLED = ("split", "wing4", "split_laminar", "wing4_euler", "split_qcr")


@pytest.fixture(scope="module")
def z():
    return np.load(GOLDEN)


def raw_blocks(z, name):
    return [z[f"{name}_raw{b}"] for b in range(int(z[f"{name}_n_blocks"]))]


def docs(z, name):
    d = json.loads(str(z[f"{name}_case_json"]))
    return d["case"], d["numerical"]


def face_labels(rects, extent) -> dict:
    """Per face of a side: its patch name, or the partner block, side and running position
    (independent of how the side is cut into rectangles)."""
    out = {}
    for r in rects:
        for a in ((x, y) for x in range(r.start[0], r.stop[0]) for y in range(r.start[1], r.stop[1])):
            out[a] = r.name if isinstance(r, Rect3) else (r.block, r.side, r.partner(a))
    assert len(out) == extent[0] * extent[1]
    return out


def from_record(r):
    if r[0] == "boundary":
        return Rect3(r[3], tuple(r[1]), tuple(r[2]))
    return Cut3(tuple(r[1]), tuple(r[2]), r[3], r[4], tuple(r[5]), tuple(r[6]), tuple(r[7]), tuple(r[8]))


@pytest.mark.parametrize("name", NAMES)
def test_assembly_matches_the_reference(z, name):
    case_doc, _ = docs(z, name)
    asm = assemble3d(raw_blocks(z, name), [PatchRule(**r) for r in case_doc["domain"]["patches"]])
    assert asm.mismatch < 1e-12
    for b, block in enumerate(asm.blocks):
        assert np.array_equal(block.nodes, z[f"{name}_nodes{b}"])     # the left-handed block reversed
        ref = json.loads(str(z[f"{name}_sides{b}"]))
        for side in SIDES_3D:
            n = block.extent(side)
            assert face_labels(block.sides[side], n) == face_labels([from_record(r) for r in ref[side]], n), \
                (b, side)


def test_the_four_block_wing_generator(z):
    """``wing_ch_blocks`` reproduces the fixture's blocks; its tip region closes the wing:
    past the cap the sheet's two sides face each other, so the wall is the wing and the
    cap only."""
    from jaxrans_b200.geometry import section_source
    from jaxrans_b200.grid3d import wing_ch_blocks
    w = json.loads(str(z["wing4_case_json"]))["case"]["domain"]
    g = wing_ch_blocks(section_source("naca0012"), 24, 6, 10, 6, 6, 1e-3, 20.0, 1.6, 0.6, 25.0, cap_cells=2,
                       span_far=3.0)
    assert g.patches == w["patches"] and np.isclose(g.reference_area, w["reference_area"])
    for b, nodes in enumerate(g.blocks):
        assert np.array_equal(nodes, z[f"wing4_raw{b}"])
    asm = assemble3d(g.blocks, [PatchRule(**r) for r in g.patches])
    assert asm.patches["wall"] == 2 * 12 * 6 + 2 * 12 * 2      # both halves of the wing, then of the cap
    with pytest.raises(ValueError, match="symmetric section"):
        wing_ch_blocks(section_source("naca4412"), 64, 16, 24, 6, 6, 1e-3, 20.0, 1.6, span_far=3.0)


def test_assembly_errors():
    theta = np.linspace(0.0, 2.0 * np.pi, 8)              # 7 cells round: a pole needs an even count
    theta[-1] = 0.0
    T, R, Zc = np.meshgrid(theta, [0.0, 1.0, 2.0], [0.0, 1.0, 2.0], indexing="ij")
    odd = np.stack([R * np.cos(T), R * np.sin(T), Zc])
    with pytest.raises(ValueError, match="collapsed"):
        assemble3d([odd], [PatchRule("farfield")])
    box = np.stack(np.meshgrid(*(np.arange(4.0),) * 3, indexing="ij"))
    with pytest.raises(ValueError, match="no patch rule"):
        assemble3d([box], [PatchRule("wall", x_max=0.5)])
    mixed = box.copy()
    mixed[0, 3] = 1.5                                     # folds the last layer of cells over
    with pytest.raises(ValueError, match="non-positive"):
        assemble3d([mixed], [PatchRule("farfield")])


def case_dir(tmp_path: Path, z, name) -> Path:
    case_doc, numerical = docs(z, name)
    write_plot3d(tmp_path / "grid.x", raw_blocks(z, name))
    (tmp_path / "case.json").write_text(json.dumps(case_doc))
    (tmp_path / "numerical.json").write_text(json.dumps(numerical))
    return tmp_path


@pytest.fixture(scope="module")
def cases(z, tmp_path_factory):
    out = {}
    for name in NAMES:
        case = load_case(case_dir(tmp_path_factory.mktemp(name), z, name))
        out[name] = (case, case.grid())
    return out


@pytest.mark.parametrize("name", NAMES)
def test_case_loads_the_file_to_the_reference_canvas(z, cases, name):
    case, plan = cases[name]
    assert plan.dim == 3 and is_3d(case.directory / "grid.x")
    assert plan.shape == z[f"{name}_interior"].shape
    assert np.array_equal(plan.interior, z[f"{name}_interior"])
    inside = plan.interior
    assert np.allclose(plan.volume[inside], z[f"{name}_volume"][inside], rtol=1e-13, atol=0.0)
    if f"{name}_distance" in z:
        assert np.allclose(plan.distance[inside], z[f"{name}_distance"][inside], rtol=1e-10, atol=1e-14)


def test_case_loader_refuses_what_the_3d_path_lacks(z, tmp_path):
    d = case_dir(tmp_path, z, "pole")
    doc = json.loads((d / "case.json").read_text())
    doc["domain"].pop("reference_area")
    (d / "case.json").write_text(json.dumps(doc))
    with pytest.raises(CaseError, match="reference_area"):
        load_case(d).grid()
    doc["domain"]["reference_area"] = 1.0
    doc["boundary_conditions"]["farfield"] = {"type": "outflow_static"}
    (d / "case.json").write_text(json.dumps(doc))
    with pytest.raises(CaseError, match="3D path"):
        load_case(d).grid()
    doc["boundary_conditions"]["farfield"] = {"type": "far_field", "model": "point_vortex"}
    (d / "case.json").write_text(json.dumps(doc))
    with pytest.raises(CaseError, match="2D model"):
        load_case(d).grid()


def rows_rel(a, b, inside):
    return max(float(np.abs(a[k][inside] - b[k][inside]).max() / max(np.abs(b[k][inside]).max(), 1e-300))
               for k in range(a.shape[0]))


@pytest.fixture(scope="module")
def described(cases):
    from jaxrans_b200.solver3d import describe_case
    return {name: describe_case(case, plan) for name, (case, plan) in cases.items()}


def host_eval(harness, desc, U, v=None, first_order=False):
    U = np.ascontiguousarray(U, dtype=np.float64)
    R = np.zeros_like(U)
    dU = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
    assert harness.jr3_host_eval(C.addressof(desc), U.ctypes.data, None if dU is None else dU.ctypes.data,
                                 R.ctypes.data, int(first_order)) == 0
    return R


@pytest.mark.parametrize("name", NAMES)
def test_kernel_bodies_give_the_reference_residual_and_jvp(harness, z, cases, described, name):
    _, plan = cases[name]
    desc, _ = described[name]
    inside = plan.interior
    U = z[f"{name}_U"]
    assert rows_rel(host_eval(harness, desc, U), z[f"{name}_R2"], inside) < 1e-12
    assert rows_rel(host_eval(harness, desc, U, first_order=True), z[f"{name}_R1"], inside) < 1e-12
    Jv, ref = host_eval(harness, desc, U, z[f"{name}_v"]), z[f"{name}_Jv"]
    assert rows_rel(Jv[:5], ref[:5], inside) < 1e-11
    if Jv.shape[0] > 5:
        assert rows_rel(Jv[5:], ref[5:], inside) < 1e-10


@pytest.mark.parametrize("name", NAMES)
def test_kernel_bodies_give_the_reference_wave_speeds(harness, z, cases, described, name):
    _, plan = cases[name]
    desc, _ = described[name]
    U = np.ascontiguousarray(z[f"{name}_U"])
    shapes = [tuple(n + (a == x) for x, n in enumerate(plan.shape)) for a in range(3)]
    lam = np.zeros(sum(int(np.prod(s)) for s in shapes))
    assert harness.jr3_host_wave_speeds(C.addressof(desc), U.ctypes.data, lam.ctypes.data) == 0
    at = 0
    for a, s in enumerate(shapes):
        part = lam[at:at + int(np.prod(s))].reshape(s)
        at += int(np.prod(s))
        # faces of block cells (the rest of the canvas is never read)
        ref = z[f"{name}_lam{a}"]
        used = np.zeros(s, dtype=bool)
        lo = [slice(None)] * 3
        lo[a] = slice(0, s[a] - 1)
        hi = [slice(None)] * 3
        hi[a] = slice(1, s[a])
        used[tuple(lo)] |= plan.interior
        used[tuple(hi)] |= plan.interior
        assert np.allclose(part[used], ref[used], rtol=1e-13, atol=0.0)


@pytest.mark.parametrize("name", WALLED)
def test_kernel_bodies_give_the_reference_line_solve_and_forces(harness, z, cases, described, name):
    case, plan = cases[name]
    desc, _ = described[name]
    U = np.ascontiguousarray(z[f"{name}_U"])
    r = np.ascontiguousarray(z[f"{name}_prec_r"])
    out = np.zeros_like(r)
    assert harness.jr3_host_precondition(C.addressof(desc), U.ctypes.data, 25.0, r.ctypes.data, out.ctypes.data) == 0
    assert rows_rel(out, z[f"{name}_prec_z"], plan.interior) < 1e-10
    spec = case.grid_spec
    centre = np.ascontiguousarray(spec.moment_centre, dtype=np.float64)
    f = np.zeros(4)
    assert harness.jr3_host_forces(C.addressof(desc), U.ctypes.data, spec.reference_area, spec.reference_length,
                                   centre.ctypes.data, f.ctypes.data) == 0
    assert np.allclose(f, z[f"{name}_forces"], rtol=1e-11, atol=1e-16)


class HostDevice3:
    """The ``DevicePlan3`` state methods ``march3d`` uses, over the host harness."""

    def __init__(self, harness, case, desc):
        cfg = case.implicit
        self.lib, self.desc = harness, desc
        self.config = np.array([cfg.krylov_tol, cfg.krylov_success,
                                cfg.max_relative_update if cfg.max_relative_update is not None else -1.0,
                                cfg.cfl_min, cfg.cfl_max, cfg.cfl_growth, cfg.cfl_cutback])
        self.iconfig = np.array([cfg.krylov_subspace, cfg.krylov_restarts, 1], dtype=np.int32)
        self.calls = 0

    def newton_steps(self, U, n, cfl, res):
        U = np.ascontiguousarray(U, dtype=np.float64).copy()
        c, r = C.c_double(cfl), C.c_double(res)
        hist = np.zeros(n)
        assert self.lib.jr3_host_newton_steps(C.addressof(self.desc), self.config.ctypes.data,
                                              self.iconfig.ctypes.data, U.ctypes.data, C.byref(c), C.byref(r), n,
                                              hist.ctypes.data) == 0
        self.calls += 1
        return U, c.value, r.value, hist

    def set_state(self, U, cfl, res):
        self.state = (np.ascontiguousarray(U, dtype=np.float64).copy(), cfl, res)

    def get_state(self):
        return self.state

    def newton_block(self, n):
        U, cfl, res, hist = self.newton_steps(*self.state[:1], n, *self.state[1:])
        self.state = (U, cfl, res)
        return hist

    def state_wall_loads(self):
        out = np.zeros((self.desc.n_walls, 7))
        assert self.lib.jr3_host_wall_loads(C.addressof(self.desc), self.state[0].ctypes.data, out.ctypes.data) == 0
        return out

    def state_forces(self, area, length, centre):
        return self.forces(self.state[0], area, length, centre)

    def forces(self, U, area, length, centre):
        U = np.ascontiguousarray(U, dtype=np.float64)
        c = np.ascontiguousarray(centre, dtype=np.float64)
        out = np.zeros(4)
        assert self.lib.jr3_host_forces(C.addressof(self.desc), U.ctypes.data, area, length, c.ctypes.data,
                                        out.ctypes.data) == 0
        return out


def test_march3d_runs_blocks_to_the_iteration_limit(harness, z, cases, described, tmp_path):
    from dataclasses import replace
    from jaxrans_b200.solver3d import freestream_state3, march3d
    case, plan = cases["pole"]
    case = replace(case, block_iters=2)
    desc, _ = described["pole"]
    dev = HostDevice3(harness, case, desc)
    seen = []
    result = march3d(case, plan, device=dev, max_iters=6, progress=lambda *a: seen.append(a[0]))
    assert dev.calls == 3 and seen == [2, 4, 6]
    assert result.history.reason == "max_iters" and result.history.n_iters == 6
    assert np.all(np.isfinite(result.history.residual)) and result.cl_history.shape == (3,)
    # the state the blocks left is the one six steps from the freestream give in one call
    U, _, _, hist = HostDevice3(harness, case, desc).newton_steps(freestream_state3(case, plan), 6,
                                                                  case.implicit.cfl, float("inf"))
    assert np.array_equal(result.U, U) and np.array_equal(result.history.residual, hist)
    out = result.write(tmp_path / "out")
    fields = np.load(out / f"{case.name}_fields.npz")
    assert fields["U_0"].shape == (5, 8, 4, 6) and "z_node_0" in fields
    assert (out / f"{case.name}_block0.vts").read_bytes().startswith(b"<?xml")
    assert not (out / f"{case.name}_surface.dat").exists()      # the pole case has no wall


@pytest.mark.parametrize("name", ["split", "wing4"])
def test_wall_distance_kernel_body_gives_the_reference_distance(harness, z, cases, name):
    """The device wall distance's arithmetic (csrc/walldist3d.cuh: the stable 16-candidate
    ranking and the patch distance), run on the host, against the reference's distance
    and the plan's NumPy distance."""
    _, plan = cases[name]
    points = np.ascontiguousarray(np.moveaxis(plan.centres[:, 1:-1, 1:-1, 1:-1], 0, -1)[plan.interior])
    faces = np.ascontiguousarray(plan.walls.quads.corners)
    out, every = np.zeros(len(points)), np.zeros(len(points))
    assert harness.jr3_host_wall_distance(points.ctypes.data, len(points), faces.ctypes.data, len(faces),
                                          out.ctypes.data, 1) == 0
    assert harness.jr3_host_wall_distance(points.ctypes.data, len(points), faces.ctypes.data, len(faces),
                                          every.ctypes.data, 0) == 0
    assert np.array_equal(out, every)          # the sphere bound skips only faces the ranking refuses
    assert np.allclose(out, z[f"{name}_distance"][plan.interior], rtol=1e-12, atol=1e-15)
    assert np.allclose(out, plan.distance[plan.interior], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", WALLED)
def test_surface_distributions_match_the_reference(harness, z, cases, described, name):
    """Per wall face: block, running position, centre, cp and the skin-friction vector
    (``solver3d.surface3`` on the kernels' wall loads), face by face in the reference's order."""
    from jaxrans_b200.solver3d import surface3
    case, plan = cases[name]
    desc, _ = described[name]
    U = np.ascontiguousarray(z[f"{name}_U"])
    loads = np.zeros((desc.n_walls, 7))
    assert harness.jr3_host_wall_loads(C.addressof(desc), U.ctypes.data, loads.ctypes.data) == 0
    got = surface3(loads, plan, case.flow)
    keys = sorted(k[len(f"{name}_surface_"):] for k in z.files if k.startswith(f"{name}_surface_"))
    assert sorted(got) == keys
    for key in keys:
        ref = z[f"{name}_surface_{key}"]
        scale = max(float(np.abs(ref).max()), 1e-300)
        assert np.allclose(got[key], ref, rtol=0.0, atol=1e-11 * scale), key


@pytest.mark.parametrize("name", NAMES)
def test_the_two_phase_residual_is_the_fused_one_bit_for_bit(harness, z, cases, described, name):
    """The device's two phases -- every face's flux once into a buffer (unwritten entries
    NaN here, so a read of one would show), then each cell's sums -- give the fused
    per-cell form's R2, R1 and J.v bit for bit."""
    desc, _ = described[name]
    U, v = np.ascontiguousarray(z[f"{name}_U"]), np.ascontiguousarray(z[f"{name}_v"])
    for dv, fo in ((None, 0), (None, 1), (v, 1)):
        fused, faces = np.zeros_like(U), np.zeros_like(U)
        ptr = None if dv is None else dv.ctypes.data
        assert harness.jr3_host_eval(C.addressof(desc), U.ctypes.data, ptr, fused.ctypes.data, fo) == 0
        assert harness.jr3_host_eval_faces(C.addressof(desc), U.ctypes.data, ptr, faces.ctypes.data, fo) == 0
        assert np.array_equal(fused, faces)


@pytest.mark.parametrize("name", NAMES)
def test_the_in_place_ghost_fill_is_the_double_buffered_one(harness, z, cases, described, name):
    """The device's ghost stages in place (each stage's values first, then its stores)
    give the double-buffered stages' canvas bit for bit: a stage writes each ghost once."""
    desc, _ = described[name]
    U = np.ascontiguousarray(z[f"{name}_U"])
    inplace, copying = np.zeros_like(U), np.zeros_like(U)
    assert harness.jr3_host_fill(C.addressof(desc), U.ctypes.data, inplace.ctypes.data, 0) == 0
    assert harness.jr3_host_fill(C.addressof(desc), U.ctypes.data, copying.ctypes.data, 1) == 0
    assert np.array_equal(inplace, copying)
    _, plan = cases[name]
    from jaxrans_b200.native3d import records_of
    rec = records_of(plan)
    at = 0
    for count in rec.counts:                       # each stage writes a ghost once
        ghosts = rec.ghost[at:at + count]
        assert len(np.unique(ghosts)) == len(ghosts)
        at += count


@pytest.mark.parametrize("name", NAMES)
def test_the_3d_oracle_gives_the_reference_residual_and_jvp(z, cases, name):
    """The NumPy restatement (``oracle.numerics3d``) on the multi-block, pole and variant
    cases -- every interface orientation, Roe and minmod, Sutherland's law, unlimited MUSCL
    with kappa, QCR2000 -- against the reference's own residual and J.v."""
    from oracle import numerics3d as n3
    from jaxrans_b200.solver3d import physics3
    case, plan = cases[name]
    ph = physics3(case)
    model = n3.Model3(plan, ph["q_inf"], ph["gamma"], ph["flux"], ph["limiter"], ph["kappa"], ph["mu_inf"],
                      ph["sutherland"], len(ph["q_inf"]) == 6, plan.distance, ph["c_cr1"])
    inside = plan.interior
    U, v = z[f"{name}_U"], z[f"{name}_v"]
    assert rows_rel(n3.residual(U, model), z[f"{name}_R2"], inside) < 1e-12
    assert rows_rel(n3.residual(U, model, first_order=True), z[f"{name}_R1"], inside) < 1e-12
    Jv, ref = n3.jvp(U, v, model), z[f"{name}_Jv"]
    assert rows_rel(Jv[:5], ref[:5], inside) < 1e-11
    if Jv.shape[0] > 5:
        assert rows_rel(Jv[5:], ref[5:], inside) < 1e-10


@pytest.mark.parametrize("name", WALLED)
def test_the_3d_oracle_gives_the_reference_forces_and_surface(z, cases, name):
    """The oracle's wall loads (``oracle.forces3d``) on the multi-block walls: the force
    coefficients and, face by face, cp and the skin-friction vector of the reference."""
    from oracle import forces3d as f3
    from oracle import numerics3d as n3
    from jaxrans_b200.solver3d import physics3
    case, plan = cases[name]
    ph = physics3(case)
    model = n3.Model3(plan, ph["q_inf"], ph["gamma"], ph["flux"], ph["limiter"], ph["kappa"], ph["mu_inf"],
                      ph["sutherland"], len(ph["q_inf"]) == 6, plan.distance, ph["c_cr1"])
    U = z[f"{name}_U"]
    spec = case.grid_spec
    f = f3.forces(U, model, spec.reference_area, spec.reference_length, tuple(spec.moment_centre))
    assert np.allclose(f, z[f"{name}_forces"], rtol=1e-11, atol=1e-16)
    p, S, shear = f3.wall_loads(U, model)
    q = 0.5 * case.flow.mach ** 2
    ref_cp = z[f"{name}_surface_cp"]
    assert np.allclose(p / q, ref_cp, rtol=0.0, atol=1e-11 * np.abs(ref_cp).max())
    if not case.flow.inviscid:
        area = np.linalg.norm(S, axis=0)
        for c, axis in enumerate("xyz"):
            ref = z[f"{name}_surface_cf_{axis}"]
            assert np.allclose(shear[c] / area / q, ref, rtol=0.0, atol=1e-11 * np.abs(ref).max())


@pytest.mark.parametrize("name", WALLED)
def test_the_3d_oracle_gives_the_reference_line_solve(z, cases, name):
    """The oracle's line_j (cyclic reduction and block Thomas) across block interfaces:
    chains along each block's wall-normal index, against the reference's solve."""
    from oracle import implicit3d as i3
    from oracle import numerics3d as n3
    from jaxrans_b200.solver3d import physics3
    case, plan = cases[name]
    ph = physics3(case)
    model = n3.Model3(plan, ph["q_inf"], ph["gamma"], ph["flux"], ph["limiter"], ph["kappa"], ph["mu_inf"],
                      ph["sutherland"], len(ph["q_inf"]) == 6, plan.distance, ph["c_cr1"])
    U, r = z[f"{name}_U"], z[f"{name}_prec_r"]
    lam = n3.wave_speeds(U, model)
    for solver in ("cr", "thomas"):
        got = i3.precondition(U, lam, 25.0, model, solver=solver)(r)
        assert rows_rel(got, z[f"{name}_prec_z"], plan.interior) < 1e-10, solver


def test_the_wing_workloads_cell_counts():
    """``workloads.wing3d_cells`` (the bench's cell count, no plan built) is the generated
    grid's: config 5's 3.93M cells and the small wing's."""
    from jaxrans_b200.geometry import section_source
    from jaxrans_b200.grid3d import wing_ch_blocks
    from jaxrans_b200.workloads import WING3D, WING3D_PLANFORM, wing3d_cells
    assert wing3d_cells("wing_ch_4blk") == 3932160
    g = wing_ch_blocks(section_source("naca0012"), **WING3D["wing_ch_4blk_small"], **WING3D_PLANFORM)
    assert wing3d_cells("wing_ch_4blk_small") == sum(int(np.prod([n - 1 for n in b.shape[1:]])) for b in g.blocks)
