"""Wall loads and force coefficients, restated in NumPy (oracle).

Follows ``src/jaxrans/post/forces.py:48-161`` in 2D: gauge pressure from the
cell on each wall face, the laminar viscous shear of the same viscous flux the
residual uses (ghosts filled against the uniform far field), lift normal and
drag along the freestream, the pitching moment of the pressure part about the
moment centre, per ``q_inf`` times the reference length.
"""

from __future__ import annotations

import numpy as np

from . import numerics as nm


def wall_loads(U, model):
    """Per wall face: gauge pressure ``(n,)``, the area vector into the fluid ``(2, n)``
    and the viscous force on the body ``(2, n)`` (``src/jaxrans/post/forces.py:48-68``)."""
    plan, g = model.plan, model.gamma
    q = nm.prim(U[:4], g)
    p = q[3].reshape(-1)[plan.walls.cell] - 1.0 / g
    S = nm.wall_vectors(plan)
    shear = np.zeros_like(S)
    if model.viscous:
        flow_model = nm.Model(plan, model.q_inf[:4], g, model.flux, model.limiter, model.kappa, model.mu_inf,
                              model.sutherland, False, 0.0, "characteristic", None)
        filled = np.pad(nm.fill_ghosts(q, flow_model, "characteristic"), ((0, 0), (1, 1), (1, 1)), mode="edge")
        visc = nm.viscous_fluxes(filled, plan.centres, [plan.faces_i, plan.faces_j], flow_model)
        shear = plan.walls.into_fluid * nm.wall_values(plan, tuple(v[1:3] for v in visc))
    return p, S, shear


def forces(U, model, length: float = 1.0, centre=(0.25, 0.0)):
    """``(cl, cd, cm, cd_friction, fx, fy)``."""
    plan = model.plan
    p, S, shear = wall_loads(U, model)
    rho, u, v = model.q_inf[0], model.q_inf[1], model.q_inf[2]
    speed = np.hypot(u, v)
    pressure = -p * S
    load = pressure + shear
    drag = np.array([u, v]) / speed
    lift = np.array([-drag[1], drag[0]])
    q_area = 0.5 * rho * speed ** 2 * length
    r = plan.walls.mid - np.asarray(centre[:2])
    moment = r[:, -1] * pressure[0] - r[:, 0] * pressure[-1]
    per_face = np.stack([lift @ load, drag @ load, moment / length]) / q_area
    totals = per_face.sum(axis=1)
    force = load.sum(axis=1)
    return np.array([totals[0], totals[1], totals[2], drag @ shear.sum(axis=1) / q_area, force[0], force[1]])
