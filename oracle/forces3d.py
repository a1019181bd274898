"""Force coefficients of a 3D case, restated in NumPy (oracle; TEST INFRASTRUCTURE).

Follows ``src/jaxrans/post/forces.py:48-161`` on a 3D plan: per wall face the gauge
pressure, the area vector into the fluid and the viscous force on the body (the face's
viscous momentum flux), then lift and drag in the plane of incidence (x-z), per
``q_inf * area``, and the pitching moment of pressure and friction about the reference
centre, per ``q_inf * area * length``.
"""

from __future__ import annotations

import numpy as np

from . import numerics3d as n3


def wall_values(plan, fields):
    """A per-family canvas face field at every wall face."""
    W = plan.walls
    out = None
    for a, f in enumerate(fields):
        flat = f.reshape(f.shape[:-3] + (-1,))
        picked = flat[..., np.where(W.family == a, W.face, 0)]
        out = picked if out is None else np.where(W.family == a, picked, out)
    return out


def wall_loads(U, model):
    """``(p - p_inf (n,), S into the fluid (3, n), shear on the body (3, n))``."""
    plan, g = model.plan, model.gamma
    q = n3.prim(U[:5], g)
    p = q[4].ravel()[plan.walls.cell] - 1.0 / g
    S = plan.walls.into_fluid * wall_values(plan, plan.faces)
    shear = np.zeros((3,) + p.shape)
    if model.viscous:
        filled = np.pad(n3.fill_ghosts(q, model), ((0, 0),) + ((1, 1),) * 3, mode="edge")
        visc = n3.viscous_fluxes(filled, plan.centres, plan.faces, model)
        shear = plan.walls.into_fluid * wall_values(plan, [v[1:4] for v in visc])
    return p, S, shear


def forces(U, model, area: float, length: float, centre=(0.25, 0.0, 0.0)):
    """``(cl, cd, cm, cd_friction)``."""
    p, S, shear = wall_loads(U, model)
    q = np.asarray(model.q_inf, dtype=np.float64)
    rho, vel = q[0], q[1:4]
    speed = np.sqrt(n3.dot(vel, vel))
    pressure = -p * S
    load = pressure + shear
    drag = vel / speed
    lift = np.array([-drag[2], 0.0, drag[0]])
    q_area = 0.5 * rho * speed ** 2 * area
    r = model.plan.walls.quads.corners.mean(axis=1) - np.asarray(centre)
    moment = r[:, -1] * load[0] - r[:, 0] * load[-1]
    cl = float(np.sum(lift @ load) / q_area)
    cd = float(np.sum(drag @ load) / q_area)
    cm = float(np.sum(moment / length) / q_area)
    return cl, cd, cm, float(drag @ shear.sum(axis=1) / q_area)
