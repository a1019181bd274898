"""Many cases advanced by the same launches: a polar, grids of uneven sizes, a batch of
requests.

The reference batches a polar by ``jax.vmap`` of one Newton step over the freestream
vectors (``src/jaxrans/polar.py:80-121``) and marches the batch with its driver
(``src/jaxrans/solvers/driver.py:123-201``), each case with its own CFL ramp and exit.
Here the batch is one device plan (``jr_batch_create``): every kernel of a Newton step
takes all cases, so one captured graph steps the whole batch, and cases on grids of
different sizes share it.  Each case's reductions are split exactly as when it runs
alone, so a case's history and state in a batch are bitwise those of the case alone.

A case leaves the launches at its own exit (``release``, the default): its slot is
disabled and its state stays the one its exit test stopped on -- the result of running
that case alone.  With ``release=False`` every case keeps stepping until the last one
stops, as the reference's vmapped batch does.
"""

from __future__ import annotations

import time

import numpy as np

from .case import Case
from .plan import Plan
from .solver import (CaseMonitor, ConvergenceHistory, Result, Timing, device_monitored, forces_of,
                     freestream_state)


def batch_device(cases: list[Case], grids: list[Plan], autotune: bool = True):
    """One device plan for ``cases`` on ``grids`` (each case's own numerics, CFL settings
    and force reference; the model, precision and Krylov settings must agree)."""
    from .native import DevicePlan
    specs = [c.grid_spec for c in cases]
    dev = DevicePlan.batch(list(grids), [c.flow for c in cases], [c.numerics for c in cases],
                           [c.implicit for c in cases], [s.reference_length for s in specs],
                           [tuple(s.moment_centre[:2]) for s in specs])
    if autotune:
        dev.autotune()
    return dev


def start_batch(dev, cases: list[Case], grids: list[Plan], initial=None) -> None:
    """Every case from its freestream (or from ``initial[k]`` on the block cells), at its
    own starting CFL."""
    for k, (case, grid) in enumerate(zip(cases, grids)):
        U0 = freestream_state(case, grid)
        if initial is not None and initial[k] is not None:
            U0 = np.where(grid.interior, np.asarray(initial[k]), U0)
        dev.set_case_state(k, U0, case.implicit.cfl, float("inf"))
        dev.enable(k, True)


def run_batch_blocks(cases: list[Case], dev, max_iters=None, progress=None, release: bool = True,
                     monitor: str = "device"):
    """Blocks of Newton steps of every case of the device batch until each has stopped by
    the exit test of a single run, run on the device (``monitor="device"``: one host
    synchronisation every few blocks, each case leaving the launches at its own exit) or
    on the host after every block (``"host"``).  Returns the monitors (with each case's
    exit time in ``seconds`` and its forces at the end), the seconds and the first block's
    seconds."""
    if monitor == "device":
        monitors, seconds, first_block = device_monitored(cases, dev, max_iters, release=release)
        forces = np.atleast_2d(dev.forces())
        for k, m in enumerate(monitors):
            m.forces = forces_of(forces[k])
        if progress is not None:
            progress(max(m.iterations for m in monitors), np.array([m.cl_history[-1] for m in monitors]))
        return monitors, seconds, first_block
    block_iters = {c.block_iters for c in cases}
    if len(block_iters) != 1:
        raise ValueError("the cases of a batch must share convergence.block_iters")
    block_iters = block_iters.pop()
    monitors = [CaseMonitor(c, max_iters) for c in cases]
    started = time.perf_counter()
    first_block = float("nan")
    while not all(m.done for m in monitors):
        hist = dev.newton_steps(block_iters)
        if np.ndim(hist) == 1:
            hist = hist[:, None]
        forces = np.atleast_2d(dev.forces())
        if np.isnan(first_block):
            first_block = time.perf_counter() - started
        for k, mon in enumerate(monitors):
            if mon.done:
                continue
            if mon.feed(hist[:, k], forces[k]):
                mon.seconds = time.perf_counter() - started   # the case's latency in the batch
                if release and dev.n_cases > 1:
                    dev.enable(k, False)
        if progress is not None:
            progress(max(m.iterations for m in monitors), np.array([m.cl_history[-1] for m in monitors]))
    return monitors, time.perf_counter() - started, first_block


def run_batch(cases: list[Case], grids: list[Plan] | None = None, progress=None, release: bool = True,
              initial=None, device=None, monitor: str = "device") -> list[Result]:
    """Each case of ``cases`` to steady state, all advanced together on one GPU; one
    ``Result`` per case, as ``run`` gives it alone (``monitor``: where the exit tests run,
    as in ``run_batch_blocks``)."""
    if not cases:
        return []
    if grids is None:
        made: dict = {}
        grids = []
        for c in cases:
            key = repr(c.grid_spec)
            if key not in made:
                made[key] = c.grid()
            grids.append(made[key])
    dev = device if device is not None else batch_device(cases, grids)
    start_batch(dev, cases, grids, initial)
    monitors, seconds, first_block = run_batch_blocks(cases, dev, progress=progress, release=release,
                                                      monitor=monitor)
    iterations = max(m.iterations for m in monitors)
    cells = sum(g.cells for g in grids)
    timing = Timing(seconds, first_block, iterations, cases[0].block_iters, cells, cases=len(cases))
    results = []
    walls = dev.wall_loads()
    if dev.n_cases == 1:
        walls = [walls]
    for k, (case, grid, mon) in enumerate(zip(cases, grids, monitors)):
        U = dev.case_state(k)[0]
        residual = mon.residual()
        history = ConvergenceHistory(residual, mon.reason, int(residual.size), seconds, first_block)
        forces = mon.forces if release else forces_of(np.atleast_2d(dev.forces())[k])
        results.append(Result(case=case, grid=grid, U=U, forces=forces, history=history,
                              cl_history=np.asarray(mon.cl_history), timing=timing,
                              coefficients=np.asarray(mon.coefficients), wall=walls[k]))
    return results
