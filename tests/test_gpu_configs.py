"""Device parity on the benchmark workloads' own grids, through the C ABI, against the
reference's outputs on those grids (tests/golden/make_golden_configs.py):

* ``o_euler_257``: 2D Euler, NACA 0012, O-grid 257 x 65 nodes, far field at 50 chords,
  HLLC with van Albada;
* ``c_sa_385``: SA-noft2, NACA 4412, C-grid 385 x 97 nodes (192-cell wake chains), Roe
  with minmod;
* ``c_sa_513``: the uneven 513 x 129 SA C-grid of the batched polar (256-cell chains,
  many waves of residual tiles).

Tolerances as in test_gpu_parity.py: R 1e-12 relative to each row's largest entry (2e-12
on the 513 x 129 grid, below), J.v 1e-12 on the mean-flow rows and 1e-10 on the SA row,
wave speeds 1e-13, the line solve 1e-10, forces 1e-12.

Measured on a B200: R2 on the 385 x 97 grid within 3.2e-13 of the reference; on the 513 x
129 grid the x-momentum row differs by 1.1e-12 of its largest entry (2.8e-15 absolute,
about ten units in the last place of the O(1) face fluxes whose difference it is), at the
far-field cells, where the characteristic condition's powers round differently in CUDA's
libm and the host's; the other rows within 4.5e-13."""

from __future__ import annotations

import numpy as np
import pytest

from goldens import config_state, config_vector, converged, load, rel

pytestmark = pytest.mark.gpu


def row_rel(a, b):
    return max(float(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300)) for v in range(b.shape[0]))


@pytest.fixture(scope="module")
def configs():
    """One device plan per workload grid, made on first use and kept for the module."""
    from jaxrans_b200.native import DevicePlan
    made = {}

    def get(name):
        if name not in made:
            z, case, plan = load(name)
            made[name] = (z, case, plan, DevicePlan(plan, case.flow, case.numerics, case.implicit))
        return made[name]

    yield get
    for *_, dev in made.values():
        dev.close()


@pytest.mark.parametrize("name,state", [("o_euler_257", "sin"), ("o_euler_257", "rand0"), ("c_sa_385", "sin"),
                                        ("c_sa_385", "rand0"), ("c_sa_513", "sin")])
def test_residual_on_config_grids(cuda, configs, name, state):
    z, case, plan, dev = configs(name)
    U = config_state(z, plan, state)
    assert row_rel(dev.residual(U), z[f"{state}_R2"]) < (2e-12 if name == "c_sa_513" else 1e-12)
    if f"{state}_R1" in z:
        assert row_rel(dev.residual(U, first_order=True), z[f"{state}_R1"]) < 1e-12


@pytest.mark.parametrize("name,state", [("o_euler_257", "sin"), ("o_euler_257", "rand0"), ("c_sa_385", "sin"),
                                        ("c_sa_385", "rand0")])
def test_jvp_on_config_grids(cuda, configs, name, state):
    z, case, plan, dev = configs(name)
    U = config_state(z, plan, state)
    ref = z[f"{state}_Jv"]
    Jv = dev.jvp(U, config_vector(plan, state, "v", ref.shape[0]))
    assert row_rel(Jv[:4], ref[:4]) < 1e-12
    if ref.shape[0] > 4:
        assert row_rel(Jv[4:], ref[4:]) < 1e-10


@pytest.mark.parametrize("name", ["o_euler_257", "c_sa_385"])
def test_wave_speeds_on_config_grids(cuda, configs, name):
    z, case, plan, dev = configs(name)
    li, lj = dev.wave_speeds(config_state(z, plan, "sin"))
    live_i = np.zeros(li.shape, bool)
    live_i[:-1] |= plan.interior
    live_i[1:] |= plan.interior
    live_j = np.zeros(lj.shape, bool)
    live_j[:, :-1] |= plan.interior
    live_j[:, 1:] |= plan.interior
    assert rel(li[live_i], z["sin_lam_i"][live_i]) < 1e-13
    assert rel(lj[live_j], z["sin_lam_j"][live_j]) < 1e-13


@pytest.mark.parametrize("name", ["o_euler_257", "c_sa_385", "c_sa_513"])
def test_line_solve_on_config_grids(cuda, configs, name):
    z, case, plan, dev = configs(name)
    ref = z["sin_prec_z"]
    out = dev.precondition(config_state(z, plan, "sin"), 25.0, config_vector(plan, "sin", "r", ref.shape[0]))
    assert rel(out, ref) < 1e-10


@pytest.mark.parametrize("name,state", [("o_euler_257", "sin"), ("c_sa_385", "sin"), ("c_sa_385", "rand0")])
def test_forces_on_config_grids(cuda, configs, name, state):
    z, case, plan, dev = configs(name)
    f = dev.forces(config_state(z, plan, state))
    assert np.abs(f - z[f"{state}_forces"]).max() < 1e-12


def test_converged_forces_on_config_1_grid(cuda):
    """Config 1 (o_euler_257: Euler, HLLC with van Albada, residual tolerance 1e-10) run
    from the freestream to the reference's own exit test on the device: CL, CD and CM
    against the reference's converged run on the same grid (tests/golden/
    o_euler_257_converged.npz: converged after 3840 Newton steps, the residual 10.06
    orders below its peak; CL 0.3453720421, CD 0.0226314963, CM -0.0375774112), 1e-6."""
    from jaxrans_b200.native import DevicePlan
    from jaxrans_b200.solver import march
    ref = converged("o_euler_257")
    assert ref is not None and str(ref["reason"]) == "converged"
    z, case, plan = load("o_euler_257")
    dev = DevicePlan(plan, case.flow, case.numerics, case.implicit)
    try:
        result = march(case, plan, device=dev)
    finally:
        dev.close()
    assert result.history.reason in ("converged", "settled")
    f = result.forces
    assert abs(f.cl - ref["forces"][0]) < 1e-6
    assert abs(f.cd - ref["forces"][1]) < 1e-6
    assert abs(f.cm - ref["forces"][2]) < 1e-6


@pytest.mark.parametrize("name", ["c_sa_385", "c_sa_513"])
def test_every_line_schedule_on_config_grids(cuda, configs, name):
    """Every line-solve schedule the autotuner may pick -- 64, 128 or 256 threads per chain
    for the factor and for the solve, the solve's factor read from global memory or staged
    from each level -- on the workloads' own chains (192 and 256 cells through the wake
    cut): bitwise the same solve, within 1e-10 of the reference's (FP64); and the FP32
    (mixed) solve bitwise the same under every schedule."""
    from dataclasses import replace
    from jaxrans_b200.native import DevicePlan, NativeError
    z, case, plan, _ = configs(name)
    U = config_state(z, plan, "sin")
    ref = z["sin_prec_z"]
    r = config_vector(plan, "sin", "r", ref.shape[0])
    for precision in ("fp64", "mixed"):
        dev = DevicePlan(plan, case.flow, case.numerics, replace(case.implicit, precision=precision))
        outs = {}
        try:
            for f in (64, 128, 256):
                for a in (64, 128, 256):
                    for stage in range(5):
                        try:
                            dev.line_schedule(f, a, stage)
                        except NativeError:
                            continue   # a form that does not fit this plan's chains
                        outs[(f, a, stage)] = dev.precondition(U, 25.0, r)
        finally:
            dev.close()
        assert len(outs) >= 20
        first = next(iter(outs.values()))
        for key, out in outs.items():
            assert np.array_equal(out, first), (precision, key)
        if precision == "fp64":
            assert rel(first, ref) < 1e-10
        else:
            assert rel(first, ref) < 1e-4
