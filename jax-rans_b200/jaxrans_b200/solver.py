"""The iteration driver and ``run``: blocks of Newton steps on the device, the host
between blocks for the exit tests and force monitoring.

Exit semantics follow ``src/jaxrans/solvers/driver.py:123-201`` and
``src/jaxrans/simulation.py:40-50, 243-284``: converged when the last residual of a
block is ``tol`` times the running peak; settled when CL, CD and CM each vary by less
than ``forces_tol`` over the last quarter of the blocks (at least four samples there);
stalled when a whole block's residual is bitwise constant; non-finite on any NaN.
One device->host synchronisation per block (the residual history and the forces).
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .case import Case
from .config import freestream_primitive
from .plan import Plan


class ExitReason:
    CONVERGED = "converged"
    SETTLED = "settled"
    MAX_ITERS = "max_iters"
    NON_FINITE = "non_finite"
    STALLED = "stalled"


@dataclass
class ConvergenceHistory:
    residual: np.ndarray
    reason: str
    n_iters: int
    seconds: float = float("nan")
    first_block_seconds: float = float("nan")
    case_reasons: tuple = ()

    @property
    def converged(self) -> bool:
        return self.reason == ExitReason.CONVERGED

    @property
    def peak(self) -> float:
        finite = self.residual[np.isfinite(self.residual)]
        return float(finite.max()) if finite.size else float("nan")

    @property
    def orders_dropped(self) -> float:
        if self.residual.size == 0:
            return 0.0
        peak, last = self.peak, self.residual[-1]
        if not (np.isfinite(peak) and np.isfinite(last)) or peak <= 0 or last <= 0:
            return float("nan")
        return float(np.log10(peak / last))

    def summary(self) -> str:
        return (f"{self.reason} after {self.n_iters} iterations, residual peak {self.peak:.6e} -> "
                f"{self.residual[-1]:.6e} ({self.orders_dropped:.2f} orders from peak)")


@dataclass(frozen=True)
class Forces:
    cl: float
    cd: float
    cm: float
    fx: float
    fy: float
    cd_friction: float = 0.0

    def summary(self) -> str:
        friction = f" (friction {self.cd_friction:+.6f})" if self.cd_friction else ""
        return f"CL = {self.cl:+.6f}   CD = {self.cd:+.6f}{friction}   CM = {self.cm:+.6f}"


def forces_of(values) -> Forces:
    cl, cd, cm, cdf, fx, fy = (float(v) for v in values)
    return Forces(cl, cd, cm, fx, fy, cdf)


@dataclass(frozen=True)
class Timing:
    total: float
    first_block: float
    iterations: int
    block_iters: int
    cells: int
    cases: int = 1

    @property
    def per_iteration(self) -> float:
        later = self.iterations - self.block_iters
        return (self.total - self.first_block) / later if later > 0 else float("nan")

    def record(self) -> dict:
        return {"total_s": self.total, "per_iteration_s": self.per_iteration, "iterations": self.iterations,
                "cells": self.cells, "cases": self.cases}


@dataclass
class Result:
    """A run: ``U`` on the canvas ``(nvar, NI, NJ)``, forces, the residual history,
    the lift at the end of every block (``src/jaxrans/simulation.py:104-169``)."""

    case: Case
    grid: Plan
    U: np.ndarray
    forces: Forces
    history: ConvergenceHistory
    cl_history: np.ndarray
    timing: Timing
    coefficients: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    wall: np.ndarray | None = None   # per wall face: gauge p, area into the fluid (2), viscous force (2)

    @property
    def cells(self) -> int:
        return self.grid.cells

    @property
    def seconds(self) -> float:
        return self.timing.total

    def surface(self) -> dict:
        """Wall distributions per face: ``x``, ``y``, ``body``, ``cp`` and, viscous, ``cf``
        along the downstream-pointing tangent (``src/jaxrans/post/forces.py:203-226``)."""
        if self.wall is None:
            raise ValueError("this result carries no wall loads")
        if getattr(self.grid, "dim", 2) == 3:
            from .solver3d import surface3
            return surface3(np.asarray(self.wall), self.grid, self.case.flow)
        p, sx, sy, fx, fy = (np.asarray(self.wall)[:, k] for k in range(5))
        q = 0.5 * self.case.flow.mach ** 2
        walls = self.grid.walls
        out = {"x": walls.mid[:, 0], "y": walls.mid[:, 1], "body": walls.body.astype(float), "cp": p / q}
        if not self.case.flow.inviscid:
            length = np.hypot(sx, sy)
            tx, ty = sy / length, -sx / length
            sign = np.where(tx >= 0.0, 1.0, -1.0)
            out["cf"] = sign * (fx * tx + fy * ty) / length / q
        return out

    def write(self, directory=None, extra: dict | None = None):
        """The run's files in the reference's layout (``src/jaxrans/simulation.py:135-169``,
        ``src/jaxrans/io/output.py:70-128``): ``<name>_metadata.json``, ``_residual.dat``,
        ``_lift.dat``, ``_surface.dat`` and ``_fields.npz`` (U and nodes per block)."""
        from .output import write_result
        return write_result(self, directory, extra)

    @property
    def cl_spread(self) -> float:
        return cl_spread(self.cl_history)


def cl_spread(history) -> float:
    """The range over the last quarter of the blocks; NaN with fewer than 4 samples there."""
    tail = np.asarray(history)[3 * len(history) // 4:]
    return float(tail.max() - tail.min()) if tail.size >= 4 else float("nan")


def freestream_state(case: Case, plan: Plan) -> np.ndarray:
    """The freestream on every canvas cell, conservative (``src/jaxrans/numerics/residual.py:250-258``)."""
    q = freestream_primitive(case.flow)
    g = case.flow.gamma
    rho, u, v, p = q[:4]
    rows = [rho, rho * u, rho * v, p / (g - 1.0) + 0.5 * rho * (u * u + v * v)]
    if len(q) > 4:
        rows.append(rho * q[4])
    return np.broadcast_to(np.array(rows)[:, None, None], (len(rows),) + plan.shape).copy()


def device_for(case: Case, plan: Plan, autotune: bool = True):
    from .native import DevicePlan
    spec = case.grid_spec
    dev = DevicePlan(plan, case.flow, case.numerics, case.implicit, spec.reference_length,
                     tuple(spec.moment_centre[:2]))
    if autotune:
        dev.autotune()
    return dev


@dataclass
class Blocks:
    """What ``run_blocks`` returns: the history, the exit reason, the force monitor."""

    residual: np.ndarray
    reason: str
    cl_history: np.ndarray
    coefficients: np.ndarray
    last_forces: Forces
    seconds: float
    first_block: float
    blocks: int


class CaseMonitor:
    """The exit test of one case, fed one block of residual norms and the forces after it
    at a time: ``src/jaxrans/solvers/driver.py:161-190`` for one case, with the force
    settling of ``src/jaxrans/simulation.py:243-284``.  A single run and every case of a
    batch go through this same code."""

    def __init__(self, case: Case, max_iters=None):
        num = case.numerics
        self.tol, self.forces_tol = num.tol, num.forces_tol
        self.block_iters = case.block_iters
        max_iters = num.max_iters if max_iters is None else max_iters
        self.n_blocks = max(1, -(-max_iters // self.block_iters))
        self.blocks: list[np.ndarray] = []
        self.cl_history: list[float] = []
        self.coefficients: list[tuple] = []
        self.peak, self.reason, self.forces = 0.0, ExitReason.MAX_ITERS, None
        self.seconds = float("nan")   # set by a batch driver when the case stops

    @property
    def done(self) -> bool:
        return self.reason != ExitReason.MAX_ITERS or len(self.blocks) >= self.n_blocks

    @property
    def iterations(self) -> int:
        return len(self.blocks) * self.block_iters

    def orders(self) -> float:
        last = float(self.blocks[-1][-1])
        return float(np.log10(self.peak / last)) if self.peak > 0 and last > 0 else 0.0

    def feed(self, hist: np.ndarray, forces) -> bool:
        """One block; true once the case has stopped."""
        hist = np.asarray(hist, dtype=np.float64)
        f = forces if isinstance(forces, Forces) else forces_of(forces)
        self.forces = f
        self.blocks.append(hist)
        self.cl_history.append(f.cl)
        self.coefficients.append((f.cl, f.cd, f.cm))
        finite = hist[np.isfinite(hist)]
        if finite.size:
            self.peak = max(self.peak, float(finite.max()))
        stop = self.forces_tol is not None and all(cl_spread(h) < self.forces_tol
                                                   for h in np.transpose(self.coefficients))
        last = hist[-1]
        failed = not np.all(np.isfinite(hist)) or not np.all(np.isfinite([f.cl, f.cd, f.cm]))
        if failed:
            self.reason = ExitReason.NON_FINITE
        elif self.peak > 0 and last <= self.tol * self.peak:
            self.reason = ExitReason.CONVERGED
        elif len(hist) > 1 and np.all(hist == hist[0]):
            self.reason = ExitReason.STALLED
        elif stop:
            self.reason = ExitReason.SETTLED
        return self.done

    def residual(self) -> np.ndarray:
        return np.concatenate(self.blocks) if self.blocks else np.zeros(0)


_DEVICE_REASONS = {"converged": ExitReason.CONVERGED, "settled": ExitReason.SETTLED,
                   "max_iters": ExitReason.MAX_ITERS, "non_finite": ExitReason.NON_FINITE,
                   "stalled": ExitReason.STALLED, "running": ExitReason.MAX_ITERS}


def device_monitored(cases, dev, max_iters=None, chunk: int = 4, release: bool = True, on_block=None):
    """Blocks of Newton steps of every case of ``dev`` with each case's exit test run on
    the device after every block (``jr_monitor_blocks``): the host synchronises once per
    ``chunk`` blocks instead of once per block, and a case that stops mid-chunk leaves the
    launches already queued.  The decisions are the host monitor's (``CaseMonitor``), made
    on the device with the same arithmetic; the returned monitors hold what the host
    monitor would -- each case's blocks of |R|, its force samples (CL, CD, CM), its peak
    and reason -- with ``forces`` left for the caller to read at the end (a stopped case's
    state, and so its forces, stay as they were at its exit).  ``on_block(k, monitor)``
    runs for every new block of case k, after its chunk."""
    block_iters = {c.block_iters for c in cases}
    if len(block_iters) != 1:
        raise ValueError("the cases of a batch must share convergence.block_iters")
    block_iters = block_iters.pop()
    monitors = [CaseMonitor(c, max_iters) for c in cases]
    if any(m.n_blocks > dev.MONITOR_BLOCKS for m in monitors):
        raise ValueError(f"the device monitor holds at most {dev.MONITOR_BLOCKS} blocks")
    for k, (c, m) in enumerate(zip(cases, monitors)):
        dev.monitor_set(k, c.numerics.tol, c.numerics.forces_tol, m.n_blocks, release)
    started = time.perf_counter()
    first_block = float("nan")
    while not all(m.done for m in monitors):
        left = max(m.n_blocks - len(m.blocks) for m in monitors if not m.done)
        n = max(1, min(chunk, left, 4096 // block_iters))
        hist = dev.monitor_blocks(n, block_iters)
        if np.isnan(first_block):
            first_block = time.perf_counter() - started
        for k, m in enumerate(monitors):
            if m.done:
                continue
            reason, blocks, peak, coef = dev.monitor_get(k)
            for b in range(blocks - len(m.blocks)):
                m.blocks.append(hist[b * block_iters:(b + 1) * block_iters, k].copy())
                cl, cd, cm = (float(x) for x in coef[len(m.blocks) - 1])
                m.cl_history.append(cl)
                m.coefficients.append((cl, cd, cm))
                if on_block is not None:
                    on_block(k, m)
            m.peak = peak
            if reason != "running":
                m.reason = _DEVICE_REASONS[reason]
                m.seconds = time.perf_counter() - started
                if reason == "max_iters":
                    m.blocks = m.blocks[:m.n_blocks]
    return monitors, time.perf_counter() - started, first_block


def run_blocks(case: Case, dev, max_iters=None, progress=None, monitor: str = "device") -> Blocks:
    """Blocks of ``block_iters`` Newton steps from the device's current state until the
    exit test of ``src/jaxrans/solvers/driver.py:123-201`` stops the case: run on the
    device (``monitor="device"``, a host synchronisation every few blocks), or on the host
    after every block (``"host"``, the reference's own rhythm).  Both stop on the same
    block with the same history."""
    started = time.perf_counter()
    if monitor == "device":
        def report(_, m):
            if progress is not None:
                progress(m.iterations, float(m.blocks[-1][-1]), m.orders(),
                         Forces(*m.coefficients[-1], float("nan"), float("nan")))
        (mon,), seconds, first_block = device_monitored([case], dev, max_iters, on_block=report)
        mon.forces = forces_of(dev.forces())
        return Blocks(mon.residual(), mon.reason, np.asarray(mon.cl_history), np.asarray(mon.coefficients),
                      mon.forces, seconds, first_block, len(mon.blocks))
    mon = CaseMonitor(case, max_iters)
    first_block = float("nan")
    while not mon.done:
        hist = dev.newton_steps(mon.block_iters)
        if not mon.blocks:
            first_block = time.perf_counter() - started
        mon.feed(hist, dev.forces())
        if progress is not None:
            progress(mon.iterations, float(hist[-1]), mon.orders(), mon.forces)
    return Blocks(mon.residual(), mon.reason, np.asarray(mon.cl_history), np.asarray(mon.coefficients),
                  mon.forces, time.perf_counter() - started, first_block, len(mon.blocks))


def march(case: Case, plan: Plan, progress=None, initial=None, device=None, max_iters=None,
          monitor: str = "device") -> Result:
    """One grid to steady state from the freestream, or from ``initial`` on the block cells."""
    dev = device if device is not None else device_for(case, plan)
    U0 = freestream_state(case, plan)
    if initial is not None:
        U0 = np.where(plan.interior, np.asarray(initial), U0)
    dev.set_state(U0, case.implicit.cfl, float("inf"))
    blk = run_blocks(case, dev, max_iters, progress, monitor)
    U, _, _, _ = dev.get_state()
    history = ConvergenceHistory(blk.residual, blk.reason, int(blk.residual.size), blk.seconds, blk.first_block)
    return Result(case=case, grid=plan, U=U, forces=forces_of(dev.forces()), history=history,
                  cl_history=blk.cl_history,
                  timing=Timing(blk.seconds, blk.first_block, int(blk.residual.size), case.block_iters, plan.cells),
                  coefficients=blk.coefficients, wall=dev.wall_loads())


def run(case: Case, grid: Plan | None = None, progress=None, on_level=None, devices=None, *, initial=None) -> Result:
    """March ``case`` to steady state on ``grid`` (default ``case.grid()``; a 3D grid
    file gives a 3D plan, marched by ``solver3d.march3d``) on one GPU
    (``src/jaxrans/simulation.py:213-240``).  ``devices`` (slabs over several GPUs) is
    not part of jaxrans_b200."""
    if devices is not None and len(devices) > 1:
        raise ValueError("splitting one case over several devices is not implemented in jaxrans_b200")
    plan = case.grid() if grid is None else grid
    if on_level is not None:
        on_level(0, plan)
    if getattr(plan, "dim", 2) == 3:
        from .solver3d import march3d
        return march3d(case, plan, progress=progress, initial=initial)
    return march(case, plan, progress=progress, initial=initial)
