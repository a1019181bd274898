"""The exit test on the device (jr_monitor_*) against the host's (CaseMonitor): the same
case run to its exit both ways stops on the same block for the same reason, with bitwise
the same residual history, force samples, state and forces -- for single runs that
converge, settle or run out of iterations, and for a polar batch whose cases leave the
launches at different blocks (src/jaxrans/solvers/driver.py:161-190,
src/jaxrans/simulation.py:259-272)."""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from goldens import load

pytestmark = pytest.mark.gpu


def with_numerics(case, **kw):
    return replace(case, numerics=replace(case.numerics, **kw))


def same_result(a, b):
    assert a.history.reason == b.history.reason
    assert a.history.n_iters == b.history.n_iters
    assert np.array_equal(a.history.residual, b.history.residual)
    assert np.array_equal(a.cl_history, b.cl_history)
    assert np.array_equal(a.coefficients, b.coefficients)
    assert np.array_equal(a.U, b.U)
    assert (a.forces.cl, a.forces.cd, a.forces.cm) == (b.forces.cl, b.forces.cd, b.forces.cm)


@pytest.mark.parametrize("name,kw,reason", [
    ("o_euler", {}, "converged"),
    ("c_laminar", {}, "converged"),
    ("c_sa", {"forces_tol": 1e-6, "tol": 1e-14}, "settled"),
    ("o_euler", {"max_iters": 60}, "max_iters"),
])
def test_device_monitor_stops_where_the_host_monitor_stops(cuda, name, kw, reason):
    from jaxrans_b200.solver import device_for, march
    z, case, plan = load(name)
    case = with_numerics(case, **kw) if kw else case
    dev = device_for(case, plan, autotune=False)
    try:
        host = march(case, plan, device=dev, monitor="host")
        device = march(case, plan, device=dev, monitor="device")
        again = march(case, plan, device=dev, monitor="device")   # the plan is reusable after a run
    finally:
        dev.close()
    assert host.history.reason == reason
    same_result(host, device)
    same_result(device, again)


def test_device_monitor_in_a_polar_batch(cuda):
    from jaxrans_b200.batch import batch_device, run_batch
    z, case, plan = load("c_sa")
    case = with_numerics(case, forces_tol=1e-6, tol=1e-14, max_iters=1200)
    cases = [replace(case, flow=replace(case.flow, alpha_deg=a)) for a in (-2.0, 4.0, 10.0)]
    cases[0] = with_numerics(cases[0], max_iters=200)   # this one stops early, at max_iters
    dev = batch_device(cases, [plan] * 3, autotune=False)
    try:
        host = run_batch(cases, [plan] * 3, device=dev, monitor="host")
        device = run_batch(cases, [plan] * 3, device=dev, monitor="device")
    finally:
        dev.close()
    for a, b in zip(host, device):
        same_result(a, b)
    assert len({r.history.n_iters for r in device}) > 1   # the cases left at different blocks
