"""The batch driver's host logic on a fake device (no GPU): each case stops by the exit
test of a single run (``src/jaxrans/solvers/driver.py:161-190``) and leaves the launches
at once; the others keep going."""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from goldens import load
from jaxrans_b200.batch import run_batch_blocks
from jaxrans_b200.solver import CaseMonitor, ExitReason, run_blocks


class FakeBatch:
    """Residual norms per case from a function of (case, step); constant forces."""

    def __init__(self, norms, n_cases, forces=None):
        self.norms, self.n_cases = norms, n_cases
        self.step = np.zeros(n_cases, dtype=int)
        self.enabled = np.ones(n_cases, dtype=bool)
        self.disabled_at = {}
        self.forces_value = forces if forces is not None else np.tile([0.5, 0.01, -0.1, 0.005, 0.0, 0.0],
                                                                      (n_cases, 1))
        self.blocks = 0

    def newton_steps(self, n):
        hist = np.empty((n, self.n_cases))
        for k in range(self.n_cases):
            for s in range(n):
                hist[s, k] = self.norms(k, self.step[k] + s)
            if self.enabled[k]:
                self.step[k] += n
        self.blocks += 1
        return hist

    def forces(self):
        return self.forces_value

    def enable(self, k, on=True):
        self.enabled[k] = on
        if not on:
            self.disabled_at[k] = self.blocks


def small_case(**convergence):
    z, case, plan = load("o_euler")
    return replace(case, numerics=replace(case.numerics, **convergence)) if convergence else case


def test_cases_stop_on_their_own_exit_and_leave_the_launches():
    case = small_case(max_iters=200, tol=1e-6, forces_tol=None)

    def norms(k, s):
        if k == 0:      # falls 1e-7 below its peak by step 60: converged
            return 1.0 * 10.0 ** (-s / 8.0)
        if k == 1:      # frozen from step 40: stalled
            return 0.5 if s >= 40 else 1.0 - 0.01 * s
        return 1.0 + 0.001 * np.sin(s)   # runs to max_iters

    dev = FakeBatch(norms, 3)
    monitors, _, _ = run_batch_blocks([case] * 3, dev, monitor="host")
    assert [m.reason for m in monitors] == [ExitReason.CONVERGED, ExitReason.STALLED, ExitReason.MAX_ITERS]
    block = case.block_iters
    assert monitors[0].iterations == 3 * block           # 10^(-59/8) < 1e-6 in the third block
    assert dev.disabled_at[0] == 3 and dev.disabled_at[1] == 3   # steps 40-59 all equal
    assert monitors[2].iterations == 200
    assert 2 in dev.disabled_at                           # the last one leaves too


def test_a_case_in_a_batch_sees_what_it_sees_alone():
    """The shared monitor: a case's exit and history in a batch equal its single run."""
    case = small_case(max_iters=400, tol=1e-8, forces_tol=None)

    def norms(k, s):
        return (2.0 + k) * 10.0 ** (-s / (20.0 + 7 * k))

    batch = FakeBatch(norms, 2)
    monitors, _, _ = run_batch_blocks([case, case], batch, monitor="host")

    class Single:
        def __init__(self, k):
            self.inner = FakeBatch(lambda _, s: norms(k, s), 1)

        def newton_steps(self, n):
            return self.inner.newton_steps(n)[:, 0]

        def forces(self):
            return self.inner.forces()[0]

    for k in range(2):
        alone = run_blocks(case, Single(k), monitor="host")
        assert alone.reason == monitors[k].reason
        assert np.array_equal(alone.residual, monitors[k].residual())


def test_settling_by_forces_per_case():
    case = small_case(max_iters=2000, tol=1e-14, forces_tol=1e-6)
    forces = np.array([[0.5, 0.01, -0.1, 0.0, 0.0, 0.0], [0.6, 0.02, -0.1, 0.0, 0.0, 0.0]])
    dev = FakeBatch(lambda k, s: 1.0 + 0.1 * np.cos(s), 2, forces)
    monitors, _, _ = run_batch_blocks([case, case], dev, monitor="host")
    # constant forces: settled once four samples lie in the last quarter (13 blocks: 13 - 9)
    assert all(m.reason == ExitReason.SETTLED for m in monitors)
    assert all(len(m.blocks) == 13 for m in monitors)


def test_batch_needs_one_block_length():
    a = small_case()
    b = replace(a, block_iters=a.block_iters + 1)
    with pytest.raises(ValueError, match="block_iters"):
        run_batch_blocks([a, b], FakeBatch(lambda k, s: 1.0, 2), monitor="host")


def test_monitor_counts_max_iters_in_blocks():
    case = small_case(max_iters=45, tol=1e-12, forces_tol=None)
    mon = CaseMonitor(case)
    assert mon.n_blocks == -(-45 // case.block_iters)


class FakeMonitored(FakeBatch):
    """FakeBatch with the device monitor's calls (jr_monitor_*): after every block the
    exit test of k_monitor, restated here in its order -- non-finite, converged, stalled,
    settled, max_iters -- and a stopped case leaves the launches when `release` is set."""

    MONITOR_BLOCKS = 1024

    def __init__(self, norms, n_cases, forces=None):
        super().__init__(norms, n_cases, forces)
        self.mon = [None] * n_cases

    def monitor_set(self, k, tol, forces_tol, max_blocks, release=True):
        self.mon[k] = {"tol": tol, "forces_tol": -1.0 if forces_tol is None else forces_tol, "peak": 0.0,
                       "max": max_blocks, "blocks": 0, "reason": "running", "release": release, "coef": []}
        self.enabled[k] = True

    def monitor_blocks(self, n_blocks, block_iters):
        rows = np.full((n_blocks * block_iters, self.n_cases), np.nan)
        pos = [0] * self.n_cases
        for _ in range(n_blocks):
            hist = self.newton_steps(block_iters)
            for k in range(self.n_cases):
                m = self.mon[k]
                if not self.enabled[k] or m is None or m["reason"] != "running":
                    continue
                h = hist[:, k]
                rows[pos[k]:pos[k] + block_iters, k] = h
                pos[k] += block_iters
                f = self.forces_value[k][:3]
                m["coef"].append(tuple(f))
                finite = h[np.isfinite(h)]
                if finite.size:
                    m["peak"] = max(m["peak"], float(finite.max()))
                m["blocks"] += 1
                n = m["blocks"]
                tail = np.array(m["coef"][3 * n // 4:])
                settled = m["forces_tol"] >= 0 and len(tail) >= 4 and all(
                    tail[:, c].max() - tail[:, c].min() < m["forces_tol"] for c in range(3))
                if not np.all(np.isfinite(h)) or not np.all(np.isfinite(f)):
                    m["reason"] = "non_finite"
                elif m["peak"] > 0 and h[-1] <= m["tol"] * m["peak"]:
                    m["reason"] = "converged"
                elif block_iters > 1 and np.all(h == h[0]):
                    m["reason"] = "stalled"
                elif settled:
                    m["reason"] = "settled"
                elif n >= m["max"]:
                    m["reason"] = "max_iters"
                if m["reason"] != "running" and m["release"]:
                    self.enable(k, False)
        return rows

    def monitor_get(self, k):
        m = self.mon[k]
        return m["reason"], m["blocks"], m["peak"], np.array(m["coef"]).reshape(-1, 3)


@pytest.mark.parametrize("chunk", [1, 3, 4])
def test_the_device_monitor_driver_gives_the_host_monitor_s_results(chunk):
    """device_monitored over a fake device running the device exit test: the same reasons,
    blocks, histories and force samples as the host monitor, whatever the chunk."""
    from jaxrans_b200.solver import device_monitored
    case = small_case(max_iters=400, tol=1e-6, forces_tol=1e-6)

    def norms(k, s):
        if k == 0:
            return 10.0 ** (-s / 8.0)                      # converged
        if k == 1:
            return 0.5 if s >= 40 else 1.0 - 0.01 * s      # stalled
        if k == 2:
            return 1.0 + 0.001 * np.sin(s)                  # settled (constant forces)
        return float("nan") if s >= 70 else 1.0 + s        # non-finite

    host, _, _ = run_batch_blocks([case] * 4, FakeBatch(norms, 4), monitor="host")
    device, _, _ = device_monitored([case] * 4, FakeMonitored(norms, 4), chunk=chunk)
    for h, d in zip(host, device):
        assert h.reason == d.reason
        assert len(h.blocks) == len(d.blocks)
        assert np.array_equal(h.residual(), d.residual(), equal_nan=True)
        assert h.coefficients == d.coefficients
    assert [m.reason for m in device] == [ExitReason.CONVERGED, ExitReason.STALLED, ExitReason.SETTLED,
                                          ExitReason.NON_FINITE]
