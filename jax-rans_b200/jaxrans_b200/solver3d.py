"""The 3D march: a case on a 3D grid file to steady state on the device.

The same driver as the 2D path (``src/jaxrans/simulation.py:243-284``,
``src/jaxrans/solvers/driver.py:123-201``): blocks of ``block_iters`` pseudo-transient
Newton steps (``jr_newton_steps3d``), after each block the force coefficients
(``jr_forces3d``, lift and drag in the x-z plane) and the one exit test every case goes
through (``solver.CaseMonitor``: converged, settled, stalled, non-finite, out of
iterations).  The state stays on the device; each block returns its residual history and
the four coefficients.
"""

from __future__ import annotations

import math
import time

import numpy as np

from .config import freestream_primitive3
from .plan3d import Plan3
from .solver import CaseMonitor, ConvergenceHistory, Forces, Result, Timing


def physics3(case) -> dict:
    """The 3D device plan's physics arguments of ``case``."""
    flow, num = case.flow, case.numerics
    return {"q_inf": np.array(freestream_primitive3(flow)), "gamma": flow.gamma, "flux": num.flux,
            "limiter": num.limiter, "kappa": num.kappa, "mu_inf": None if flow.inviscid else flow.mu_inf,
            "sutherland": flow.sutherland_ratio, "c_cr1": 0.3 if flow.turbulence == "sa_noft2_qcr" else 0.0}


def describe_case(case, plan: Plan3):
    """``(jr_plan3d_desc, arrays it points into)`` of ``case`` on ``plan``."""
    from .native3d import describe
    return describe(plan, **physics3(case), implicit=case.implicit)


def device3_for(case, plan: Plan3):
    from .native3d import DevicePlan3
    return DevicePlan3(plan, **physics3(case), implicit=case.implicit)


def freestream_state3(case, plan: Plan3) -> np.ndarray:
    """The freestream on every canvas cell, conservative (``src/jaxrans/numerics/residual.py:250-258``)."""
    q = freestream_primitive3(case.flow)
    g = case.flow.gamma
    rho, u, v, w, p = q[:5]
    rows = [rho, rho * u, rho * v, rho * w, p / (g - 1.0) + 0.5 * rho * (u * u + v * v + w * w)]
    if len(q) > 5:
        rows.append(rho * q[5])
    return np.broadcast_to(np.array(rows)[:, None, None, None], (len(rows),) + plan.shape).copy()


def forces3_of(values) -> Forces:
    """``(cl, cd, cm, cd_friction)`` of ``jr_forces3d`` as ``Forces`` (no 2D force
    components)."""
    cl, cd, cm, cdf = (float(v) for v in values)
    return Forces(cl, cd, cm, math.nan, math.nan, cdf)


def surface3(loads: np.ndarray, plan: Plan3, flow) -> dict:
    """Per wall face (``src/jaxrans/post/forces.py:229-246``): its ``block`` and running
    position ``i``, ``k`` on its side, the centre ``x``, ``y``, ``z``, ``cp`` and, viscous,
    the skin-friction vector ``cf_x``, ``cf_y``, ``cf_z`` (wall shear over ``q_inf``);
    ``loads`` as ``jr_wall_loads3d`` gives them."""
    q = 0.5 * flow.mach ** 2
    quads = plan.walls.quads
    mid = quads.corners.mean(axis=1)
    out = {"block": quads.block.astype(float), "i": quads.cell[:, 0].astype(float),
           "k": quads.cell[:, 1].astype(float), "x": mid[:, 0], "y": mid[:, 1], "z": mid[:, 2],
           "cp": loads[:, 0] / q}
    if not flow.inviscid:
        area = np.linalg.norm(loads[:, 1:4], axis=1)
        for c, name in enumerate("xyz"):
            out[f"cf_{name}"] = loads[:, 4 + c] / area / q
    return out


def march3d(case, plan: Plan3, progress=None, initial=None, device=None, max_iters=None) -> Result:
    """``plan`` to steady state from the freestream, or from ``initial`` on the block
    cells.  ``device`` is anything with the ``native3d.DevicePlan3`` state methods
    ``set_state``, ``newton_block``, ``state_forces`` and ``get_state`` (default: a new
    device plan of ``case``); the state stays on it between blocks."""
    dev = device if device is not None else device3_for(case, plan)
    U = freestream_state3(case, plan)
    if initial is not None:
        U = np.where(plan.interior, np.asarray(initial), U)
    spec = case.grid_spec
    area, length, centre = spec.reference_area, spec.reference_length, tuple(spec.moment_centre)
    mon = CaseMonitor(case, max_iters)
    dev.set_state(U, case.implicit.cfl, math.inf)
    started = time.perf_counter()
    first_block = math.nan
    while not mon.done:
        hist = dev.newton_block(mon.block_iters)
        if not mon.blocks:
            first_block = time.perf_counter() - started
        mon.feed(hist, forces3_of(dev.state_forces(area, length, centre)))
        if progress is not None:
            progress(mon.iterations, float(hist[-1]), mon.orders(), mon.forces)
    seconds = time.perf_counter() - started
    U = dev.get_state()[0]
    wall = dev.state_wall_loads() if len(plan.walls.cell) else None
    residual = mon.residual()
    history = ConvergenceHistory(residual, mon.reason, int(residual.size), seconds, first_block)
    return Result(case=case, grid=plan, U=U, forces=mon.forces, history=history,
                  cl_history=np.asarray(mon.cl_history),
                  timing=Timing(seconds, first_block, int(residual.size), case.block_iters, plan.cells),
                  coefficients=np.asarray(mon.coefficients), wall=wall)
