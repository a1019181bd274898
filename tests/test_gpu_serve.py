"""The serving loop on the device: continuous batching with slots reused by new requests
(jr_case_load), every result the same as its case run alone (bitwise: slots never
interact and each keeps the reductions of a single case)."""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from goldens import load

pytestmark = pytest.mark.gpu

# two small C-grid sizes (nodes): cells round the airfoil, along each wake side, normal
SMALL = {(49, 17): (32, 8, 16), (65, 17): (44, 10, 16)}


def test_served_results_equal_runs_alone(cuda):
    from jaxrans_b200.serve import Server, poisson_requests, summary
    from jaxrans_b200.solver import march
    z, template, plan = load("c_sa")
    requests = poisson_requests(6, template, rate=200.0, seed=3, classes=SMALL)
    # short runs: 60 Newton steps at most
    requests = [replace(r, case=replace(r.case, numerics=replace(r.case.numerics, max_iters=60)))
                for r in requests]
    server = Server(max_slots=2, n_classes=len(SMALL))
    served = server.serve(requests, realtime=True)
    assert len(served) == len(requests)
    assert any(p.slots == 2 for p in server.pools)
    s = summary(served, max(x.finished for x in served))
    assert s["requests"] == 6 and s["p99_s"] >= s["p50_s"] > 0.0
    for x in served:
        alone = march(x.request.case, x.request.case.grid())
        assert x.reason == alone.history.reason
        assert np.array_equal(x.history.residual, alone.history.residual, equal_nan=True)
        assert np.array_equal(x.U, alone.U, equal_nan=True)
        f = lambda r: np.array([r.cl, r.cd, r.cm, r.cd_friction, r.fx, r.fy])  # noqa: E731
        assert np.array_equal(f(x.forces), f(alone.forces), equal_nan=True)
    server.close()


def test_a_slot_refuses_a_case_of_another_shape(cuda):
    from jaxrans_b200.native import DevicePlan, NativeError
    from jaxrans_b200.serve import request_case
    z, template, plan = load("c_sa")
    a = request_case(template, "naca2412", (49, 17), 0.3, 2.0, 3e6, "a", SMALL)
    b = request_case(template, "naca2412", (65, 17), 0.3, 2.0, 3e6, "b", SMALL)
    dev = DevicePlan.batch([a.grid()], [a.flow], a.numerics, a.implicit)
    with pytest.raises(NativeError, match="differ"):
        dev.load_case(0, b.grid(), b.flow, b.numerics, b.implicit)


def test_another_pool_of_a_size_when_its_slots_are_taken(cuda):
    """One-slot pools of one grid size: requests arriving together each get a pool of
    their own (free memory allows), and every result is the same as its case run alone."""
    from jaxrans_b200.serve import Server, poisson_requests
    from jaxrans_b200.solver import march
    z, template, plan = load("c_sa")
    one = {(49, 17): (32, 8, 16)}
    requests = poisson_requests(3, template, rate=1000.0, seed=5, classes=one)
    requests = [replace(r, case=replace(r.case, numerics=replace(r.case.numerics, max_iters=40)))
                for r in requests]
    server = Server(max_slots=1, n_classes=1)
    served = server.serve(requests, realtime=True)
    assert len(served) == 3
    assert server.made >= 2 and all(p.slots == 1 for p in server.pools)
    for x in served:
        alone = march(x.request.case, x.request.case.grid())
        assert np.array_equal(x.history.residual, alone.history.residual, equal_nan=True)
        assert np.array_equal(x.U, alone.U, equal_nan=True)
    server.close()
