"""Batches through the C ABI: several cases advanced by the same launches.

The reference batches a polar by ``jax.vmap`` of one Newton step over the freestreams
(src/jaxrans/polar.py:80-121); its cases never interact.  Here a batch is one plan
whose every kernel takes all cases, with each case's reductions split exactly as when
it runs alone, so a case's history and state in a batch are bitwise those of the same
case alone.
"""

from __future__ import annotations

import copy
from dataclasses import replace

import numpy as np
import pytest

from goldens import load
from jaxrans_b200.case import parse_case
from jaxrans_b200.config import freestream_primitive
from jaxrans_b200.solver import freestream_state

pytestmark = pytest.mark.gpu

ALPHAS = (-1.0, 2.5)


def flows_of(case, alphas):
    return [replace(case.flow, alpha_deg=float(a)) for a in alphas]


def alone(case, plan, flow, steps):
    from jaxrans_b200.native import DevicePlan
    dev = DevicePlan(plan, flow, case.numerics, case.implicit)
    dev.set_state(freestream_state(replace(case, flow=flow), plan), case.implicit.cfl)
    hist = dev.newton_steps(steps)
    U, cfl, res, status = dev.get_state()
    return hist, U, cfl, dev.forces()


@pytest.mark.parametrize("name", ["o_euler", "c_sa"])
def test_batch_is_bitwise_the_cases_alone(cuda, name):
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load(name)
    flows = flows_of(case, ALPHAS)
    dev = DevicePlan.batch(plan, flows, case.numerics, case.implicit)
    U0 = np.concatenate([freestream_state(replace(case, flow=f), plan).ravel() for f in flows])
    dev.set_state(U0, case.implicit.cfl)
    steps = 12
    hist = dev.newton_steps(steps)
    assert hist.shape == (steps, len(flows))
    forces = dev.forces()
    for k, flow in enumerate(flows):
        h1, U1, cfl1, f1 = alone(case, plan, flow, steps)
        Uk, cflk, _, _ = dev.case_state(k)
        assert np.array_equal(hist[:, k], h1)
        assert np.array_equal(Uk, U1)
        assert cflk == cfl1
        assert np.array_equal(forces[k], f1)


def test_batch_of_two_grids(cuda):
    """Cases of different canvas sizes in one batch (the launches span the largest)."""
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("o_euler")
    import json
    doc = json.loads(str(z["case_json"]))
    small_doc = copy.deepcopy(doc)
    small_doc["case"]["domain"]["cells_airfoil"] = 40
    small_doc["case"]["domain"]["cells_normal"] = 24
    small = parse_case(small_doc["case"], small_doc["numerical"])
    small_plan = small.grid()
    assert small_plan.NI * small_plan.NJ < plan.NI * plan.NJ
    dev = DevicePlan.batch([plan, small_plan], [case.flow, small.flow], case.numerics, case.implicit)
    U0 = np.concatenate([freestream_state(case, plan).ravel(), freestream_state(small, small_plan).ravel()])
    dev.set_state(U0, case.implicit.cfl)
    hist = dev.newton_steps(8)
    for k, (c, p) in enumerate([(case, plan), (small, small_plan)]):
        h1, U1, _, _ = alone(c, p, c.flow, 8)
        assert np.array_equal(hist[:, k], h1)
        assert np.array_equal(dev.case_state(k)[0], U1)


def test_disabled_case_is_untouched(cuda):
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("o_euler")
    flows = flows_of(case, ALPHAS)
    dev = DevicePlan.batch(plan, flows, case.numerics, case.implicit)
    U0 = np.concatenate([freestream_state(replace(case, flow=f), plan).ravel() for f in flows])
    dev.set_state(U0, case.implicit.cfl)
    dev.enable(1, False)
    dev.newton_steps(5)
    U1, _, _, _ = dev.case_state(1)
    assert np.array_equal(U1, freestream_state(replace(case, flow=flows[1]), plan))
    h0, U0k, _, _ = alone(case, plan, flows[0], 5)
    assert np.array_equal(dev.case_state(0)[0], U0k)
    dev.enable(1, True)
    hist = dev.newton_steps(5)
    h1, U1k, _, _ = alone(case, plan, flows[1], 5)
    assert np.array_equal(hist[:, 1], h1)


def test_new_inflow_equals_a_new_case(cuda):
    """Changing a case's freestream in place gives the case built at that angle."""
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("c_sa")
    flows = flows_of(case, ALPHAS)
    dev = DevicePlan.batch(plan, [flows[0], flows[0]], case.numerics, case.implicit)
    dev.set_inflow(1, freestream_primitive(flows[1]))
    U0 = np.concatenate([freestream_state(replace(case, flow=f), plan).ravel() for f in flows])
    dev.set_state(U0, case.implicit.cfl)
    hist = dev.newton_steps(6)
    h1, U1, _, f1 = alone(case, plan, flows[1], 6)
    assert np.array_equal(hist[:, 1], h1)
    assert np.array_equal(dev.forces()[1], f1)


def test_polar_angles_equal_their_runs_alone(cuda):
    """run_polar (src/jaxrans/polar.py:80-121) on the device batch: each angle's history,
    exit and forces are bitwise those of ``march`` of that angle alone."""
    from jaxrans_b200.polar import at_alpha, run_polar
    from jaxrans_b200.solver import march
    z, case, plan = load("c_sa")
    case = replace(case, numerics=replace(case.numerics, max_iters=80))
    polar = run_polar(case, [-2.0, 3.0, 7.5], grid=plan)
    assert polar.table().shape == (3, 9)
    for a, r in zip(polar.alphas, polar.results):
        alone = march(at_alpha(case, a), plan)
        assert r.history.reason == alone.history.reason
        assert np.array_equal(r.history.residual, alone.history.residual)
        assert np.array_equal(r.U, alone.U)
        assert r.forces == alone.forces


def test_uneven_batch_equals_runs_alone(cuda):
    """Cases on grids of different sizes and different flows in one batch."""
    import json
    from jaxrans_b200.batch import run_batch
    from jaxrans_b200.solver import march
    z, case, plan = load("o_euler")
    doc = json.loads(str(z["case_json"]))
    other_doc = copy.deepcopy(doc)
    other_doc["case"]["domain"]["cells_airfoil"] = 64
    other_doc["case"]["domain"]["cells_normal"] = 24
    other_doc["case"]["freestream"]["mach"] = 0.5
    other = parse_case(other_doc["case"], other_doc["numerical"])
    cases = [replace(c, numerics=replace(c.numerics, max_iters=60)) for c in (case, other)]
    grids = [plan, other.grid()]
    results = run_batch(cases, grids)
    for c, g, r in zip(cases, grids, results):
        alone = march(c, g)
        assert np.array_equal(r.history.residual, alone.history.residual)
        assert np.array_equal(r.U, alone.U)


def test_skipped_krylov_cycles_launch_nothing(cuda):
    """A Krylov cycle no case needs is skipped on the device (a conditional graph node):
    the launch count stays below steps x the kernels of a step with every cycle run."""
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("o_euler")
    dev = DevicePlan(plan, case.flow, case.numerics, replace(case.implicit, krylov_restarts=3))
    dev.set_state(freestream_state(case, plan), case.implicit.cfl)
    full = dev.kernels_per_step()
    before = dev.launch_count()
    dev.newton_steps(10)
    launched = dev.launch_count() - before
    assert 0 < launched < 10 * full


def test_autotuned_schedule_gives_the_same_steps(cuda):
    """The autotuner only changes the line solve's block sizes: the steps are bitwise the
    same whatever it picks."""
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("c_sa")
    runs = []
    for tune in (False, True):
        dev = DevicePlan(plan, case.flow, case.numerics, case.implicit)
        if tune:
            chosen = dev.autotune(3)
            assert chosen["line_factor_threads"] in (64, 128, 256)
            assert chosen["line_apply_threads"] in (64, 128, 256)
        dev.set_state(freestream_state(case, plan), case.implicit.cfl)
        runs.append((dev.newton_steps(8), dev.get_state()[0]))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


@pytest.mark.parametrize("name,precision", [("c_sa", "fp64"), ("c_sa", "mixed"), ("o_euler", "fp64")])
def test_staged_line_solve_gives_the_same_steps(cuda, name, precision):
    """The line solve with its chains' factor staged in shared memory by one bulk
    asynchronous copy (all levels, or from the first, second or third level down) steps
    bitwise as the one reading the factor level by level from global memory."""
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load(name)
    implicit = replace(case.implicit, precision=precision)
    runs = []
    for stage in (0, 1, 2, 3, 4):
        dev = DevicePlan(plan, case.flow, case.numerics, implicit)
        dev.line_schedule(128, 64, stage)
        dev.set_state(freestream_state(case, plan), case.implicit.cfl)
        hist = dev.newton_steps(8)
        U, cfl, res, status = dev.get_state()
        assert status & 8 == 0
        runs.append((hist, U))
        dev.close()
    for hist, U in runs[1:]:
        assert np.array_equal(runs[0][0], hist)
        assert np.array_equal(runs[0][1], U)
