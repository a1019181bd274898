"""The 3D kernels' per-cell and per-record bodies (csrc/residual3d.cuh) run on the host
by a test-only harness (tests/host3d/harness.cu, built with nvcc for the host by the
``harness`` fixture of conftest.py), in
the order the device runs them: the kernels' indexing and arithmetic checked against the
3D oracle and the reference's outputs on the wing fixture, without a GPU."""

from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from jaxrans_b200.case import flow_conditions
from jaxrans_b200.geometry import section_source
from jaxrans_b200.grid3d import wing_block
from jaxrans_b200.native3d import describe
from jaxrans_b200.plan3d import build_plan3d

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden" / "ch_sa3d.npz"
KINDS = {"wall": "no_slip_wall", "farfield": "far_field", "root": "symmetry", "tip": "symmetry"}


@pytest.fixture(scope="module")
def case3d():
    z = np.load(GOLDEN)
    w = json.loads(str(z["wing_json"]))
    doc = json.loads(str(z["case_json"]))
    plan = build_plan3d([wing_block(section_source(w.pop("section")), **w).with_kinds(KINDS)])
    flow = flow_conditions(doc["case"])
    a = flow.alpha_rad
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma,
                      flow.nu_tilde_ratio])
    cv = doc["numerical"]["convective_fluxes"]
    desc, keep = describe(plan, q_inf, flow.gamma, cv["riemann_solver"], cv["limiter"], 0.0, flow.mu_inf,
                          flow.sutherland_ratio)
    return z, plan, desc, keep


def evaluate(lib, desc, U, v=None, first_order=False):
    U = np.ascontiguousarray(U, dtype=np.float64)
    R = np.zeros_like(U)
    dU = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
    rc = lib.jr3_host_eval(C.addressof(desc), U.ctypes.data, None if dU is None else dU.ctypes.data,
                           R.ctypes.data, int(first_order))
    assert rc == 0
    return R


def rows_rel(a, b):
    return max(float(np.abs(a[k] - b[k]).max() / max(np.abs(b[k]).max(), 1e-300)) for k in range(a.shape[0]))


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_residual(harness, case3d, state):
    z, plan, desc, _ = case3d
    U = z[f"{state}_U"]
    assert rows_rel(evaluate(harness, desc, U), z[f"{state}_R2"]) < 1e-12
    assert rows_rel(evaluate(harness, desc, U, first_order=True), z[f"{state}_R1"]) < 1e-12


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_jvp(harness, case3d, state):
    z, plan, desc, _ = case3d
    Jv, ref = evaluate(harness, desc, z[f"{state}_U"], z[f"{state}_v"]), z[f"{state}_Jv"]
    assert rows_rel(Jv[:5], ref[:5]) < 1e-12
    assert rows_rel(Jv[5:], ref[5:]) < 1e-10


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_wave_speeds(harness, case3d, state):
    z, plan, desc, _ = case3d
    harness.jr3_host_wave_speeds.restype = C.c_int
    harness.jr3_host_wave_speeds.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    U = np.ascontiguousarray(z[f"{state}_U"])
    shapes = [tuple(n + (a == x) for x, n in enumerate(plan.shape)) for a in range(3)]
    lam = np.zeros(sum(int(np.prod(s)) for s in shapes))
    assert harness.jr3_host_wave_speeds(C.addressof(desc), U.ctypes.data, lam.ctypes.data) == 0
    at = 0
    for a, s in enumerate(shapes):
        part = lam[at:at + int(np.prod(s))].reshape(s)
        at += int(np.prod(s))
        assert np.allclose(part, z[f"{state}_lam{a}"], rtol=1e-14, atol=0.0)


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_line_solve(harness, case3d, state):
    """Block Thomas along the chains (the device's order) against the oracle's block Thomas
    (bitwise order) and the reference's cyclic reduction (to round-off)."""
    from oracle import implicit3d as i3
    from oracle import numerics3d as n3
    import json as _json
    z, plan, desc, _ = case3d
    harness.jr3_host_precondition.restype = C.c_int
    harness.jr3_host_precondition.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    U = np.ascontiguousarray(z[f"{state}_U"])
    r = np.ascontiguousarray(z[f"{state}_prec_r"])
    out = np.zeros_like(r)
    assert harness.jr3_host_precondition(C.addressof(desc), U.ctypes.data, 25.0, r.ctypes.data, out.ctypes.data) == 0
    assert rows_rel(out, z[f"{state}_prec_z"]) < 1e-10
    flow = flow_conditions(_json.loads(str(z["case_json"]))["case"])
    a = flow.alpha_rad
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma, flow.nu_tilde_ratio])
    model = n3.Model3(plan, q_inf, flow.gamma, "hllc", "van_albada_smooth", 0.0, flow.mu_inf,
                      flow.sutherland_ratio, True, plan.distance)
    lam = n3.wave_speeds(U, model)
    thomas = i3.precondition(U, lam, 25.0, model, solver="thomas")(r)
    assert rows_rel(out, thomas) < 1e-13


def test_newton_steps_match_the_reference(harness, case3d):
    """Three pseudo-transient Newton steps (GMRES with the line preconditioner, the
    relaxation, acceptance and CFL ramp) driven by csrc/newton3d.cuh over host loops,
    from the 'rand0' state at CFL 25 (src/jaxrans/solvers/implicit.py:84-168)."""
    import json as _json
    from jaxrans_b200.case import implicit_config
    z, plan, desc, _ = case3d
    doc = _json.loads(str(z["case_json"]))
    cfg = implicit_config(doc["numerical"])
    config = np.array([cfg.krylov_tol, cfg.krylov_success,
                       cfg.max_relative_update if cfg.max_relative_update is not None else -1.0,
                       cfg.cfl_min, cfg.cfl_max, cfg.cfl_growth, cfg.cfl_cutback])
    iconfig = np.array([cfg.krylov_subspace, cfg.krylov_restarts, 1], dtype=np.int32)
    harness.jr3_host_newton_steps.restype = C.c_int
    harness.jr3_host_newton_steps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_int, C.c_void_p]
    U = np.ascontiguousarray(z["rand0_U"]).copy()
    cfl, res = C.c_double(25.0), C.c_double(np.inf)
    hist = np.zeros(3)
    assert harness.jr3_host_newton_steps(C.addressof(desc), config.ctypes.data, iconfig.ctypes.data, U.ctypes.data,
                                         C.byref(cfl), C.byref(res), 3, hist.ctypes.data) == 0
    # per-step |R| before the update; the final state and CFL
    for k in range(3):
        assert np.isclose(hist[k], float(z[f"newton{k}_norm"]), rtol=1e-11, atol=0.0)
    assert rows_rel(U, z["newton2_U"]) < 1e-9
    assert np.isclose(cfl.value, float(z["newton2_cfl"]), rtol=1e-12)


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_forces(harness, case3d, state):
    import json as _json
    z, plan, desc, _ = case3d
    f = harness.jr3_host_forces
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    area = _json.loads(str(z["case_json"]))["case"]["domain"]["reference_area"]
    U = np.ascontiguousarray(z[f"{state}_U"])
    centre = np.array([0.25, 0.0, 0.0])
    out = np.zeros(4)
    assert f(C.addressof(desc), U.ctypes.data, area, 0.8, centre.ctypes.data, out.ctypes.data) == 0
    assert np.allclose(out, z[f"{state}_forces"], rtol=1e-11, atol=1e-16)


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_the_mixed_line_solve_stays_within_fp32_of_fp64(harness, case3d, state):
    """The mixed form's line factor and apply in FP32 (``line_precision = 1``) against the
    FP64 solve: FP32 round-off grown through the chain's block eliminations."""
    z, plan, desc, _ = case3d
    U = np.ascontiguousarray(z[f"{state}_U"])
    r = np.ascontiguousarray(z[f"{state}_prec_r"])
    exact, mixed = np.zeros_like(r), np.zeros_like(r)
    assert harness.jr3_host_precondition(C.addressof(desc), U.ctypes.data, 25.0, r.ctypes.data, exact.ctypes.data) == 0
    desc.line_precision = 1
    try:
        assert harness.jr3_host_precondition(C.addressof(desc), U.ctypes.data, 25.0, r.ctypes.data,
                                             mixed.ctypes.data) == 0
    finally:
        desc.line_precision = 0
    err = rows_rel(mixed, exact)
    assert 0.0 < err < 1e-4


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_coupled_line_solve(harness, case3d, state):
    """The coupled (6x6) form of the line solve (descriptor preconditioner 2): the factor's
    SA coupling rows and the apply's forward substitution against the oracle's coupled
    solve (itself checked against dense block solves)."""
    import json as _json
    from oracle import implicit3d as i3
    from oracle import numerics3d as n3
    z, plan, desc, _ = case3d
    U = np.ascontiguousarray(z[f"{state}_U"])
    r = np.ascontiguousarray(z[f"{state}_prec_r"])
    out = np.zeros_like(r)
    desc.preconditioner = 2
    try:
        assert harness.jr3_host_precondition(C.addressof(desc), U.ctypes.data, 25.0, r.ctypes.data,
                                             out.ctypes.data) == 0
    finally:
        desc.preconditioner = 1
    flow = flow_conditions(_json.loads(str(z["case_json"]))["case"])
    a = flow.alpha_rad
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma, flow.nu_tilde_ratio])
    model = n3.Model3(plan, q_inf, flow.gamma, "hllc", "van_albada_smooth", 0.0, flow.mu_inf,
                      flow.sutherland_ratio, True, plan.distance)
    lam = n3.wave_speeds(U, model)
    ref = i3.precondition_coupled(U, lam, 25.0, model, solver="thomas")(r)
    assert rows_rel(out, ref) < 1e-12
    split = i3.precondition(U, lam, 25.0, model, solver="thomas")(r)
    assert rows_rel(out[5:], split[5:]) > 1e-9          # the coupling changes the SA row
    assert rows_rel(out[:5], split[:5]) < 1e-13         # and not the mean flow


def test_newton_steps_with_the_coupled_and_mixed_line_solve(harness, case3d):
    """The Newton driver over the coupled 6x6 line blocks in FP32 (config 5's
    preconditioner): the residual falls as with line_j in FP64, step for step within a
    few per cent."""
    import json as _json
    from jaxrans_b200.case import implicit_config
    z, plan, desc, _ = case3d
    doc = _json.loads(str(z["case_json"]))
    cfg = implicit_config(doc["numerical"])
    config = np.array([cfg.krylov_tol, cfg.krylov_success,
                       cfg.max_relative_update if cfg.max_relative_update is not None else -1.0,
                       cfg.cfl_min, cfg.cfl_max, cfg.cfl_growth, cfg.cfl_cutback])

    def steps(preconditioner, precision):
        iconfig = np.array([cfg.krylov_subspace, cfg.krylov_restarts, preconditioner], dtype=np.int32)
        U = np.ascontiguousarray(z["rand0_U"]).copy()
        cfl, res = C.c_double(25.0), C.c_double(np.inf)
        hist = np.zeros(4)
        desc.preconditioner, desc.line_precision = preconditioner, precision
        try:
            assert harness.jr3_host_newton_steps(C.addressof(desc), config.ctypes.data, iconfig.ctypes.data,
                                                 U.ctypes.data, C.byref(cfl), C.byref(res), 4, hist.ctypes.data) == 0
        finally:
            desc.preconditioner, desc.line_precision = 1, 0
        return hist

    plain, coupled = steps(1, 0), steps(2, 1)
    assert plain[0] == coupled[0]                       # the same state before the first step
    assert np.all(np.isfinite(coupled)) and coupled[-1] < coupled[0]
    assert np.allclose(coupled, plain, rtol=5e-2)
