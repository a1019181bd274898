"""``make_residual``: the reference's residual operator over the device kernels.

Mirrors ``make_residual(grid, flow, numerics, first_order=False, freestream=None,
distance=None, mu_inf=None) -> ResidualOperator`` (``src/jaxrans/numerics/residual.py:
207-334``): ``.residual(U)``, ``.wave_speeds(U)``, ``.norm(R)`` and ``.initial_state()``
on canvas fields ``(nvar, NI, NJ)``.  Fields may be NumPy arrays (copied to the device
and back) or float64 CUDA tensors (used in place).  On a 3D plan (``plan3d.Plan3``) the
same operator runs the 3D kernels on fields ``(nvar, NI, NJ, NK)`` (NumPy arrays).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .config import FlowConditions, ImplicitConfig, NumericsConfig, freestream_primitive
from .plan import Plan


@dataclass
class ResidualOperator:
    plan: Plan
    flow: FlowConditions
    numerics: NumericsConfig
    first_order: bool
    device: object

    @property
    def grid(self) -> Plan:
        return self.plan

    @property
    def gamma(self) -> float:
        return self.flow.gamma

    def residual(self, U):
        return self.device.residual(U, first_order=self.first_order)

    def jvp(self, U, v):
        """The exact tangent of the first-order residual at ``U`` along ``v``."""
        return self.device.jvp(U, v)

    def wave_speeds(self, U):
        return self.device.wave_speeds(U)

    def norm(self, R, variable: int = 0) -> float:
        """The volume-weighted L2 norm of one row over the block cells
        (``src/jaxrans/numerics/residual.py:237-240``), on the device for a 2D plan."""
        if getattr(self.plan, "dim", 2) == 2:
            return self.device.norm(R, variable)
        R = np.asarray(R if isinstance(R, np.ndarray) else R.cpu().numpy())
        w = np.where(self.plan.interior, self.plan.volume, 0.0)
        return float(np.sqrt(np.sum(w * R[variable] ** 2) / np.sum(w)))

    def initial_state(self) -> np.ndarray:
        if getattr(self.plan, "dim", 2) == 3:
            from .solver3d import freestream_state3
            return freestream_state3(self, self.plan)
        q = freestream_primitive(self.flow)
        g = self.flow.gamma
        rho, u, v, p = q[:4]
        rows = [rho, rho * u, rho * v, p / (g - 1.0) + 0.5 * rho * (u * u + v * v)]
        if len(q) > 4:
            rows.append(rho * q[4])
        return np.broadcast_to(np.array(rows)[:, None, None], (len(rows),) + self.plan.shape).copy()


def make_residual(grid: Plan, flow: FlowConditions, numerics: NumericsConfig, first_order: bool = False,
                  freestream=None, distance=None, mu_inf=None) -> ResidualOperator:
    """The residual of one case on its plan.  ``freestream`` and ``mu_inf`` (traced
    parameters of a sensitivity in the reference) are not supported: the flow's own
    are used, and a value passed is refused."""
    if freestream is not None or mu_inf is not None:
        raise ValueError("freestream / mu_inf overrides are not implemented in jaxrans_b200; set them in flow")
    if distance is not None:
        grid.distance = np.asarray(distance, dtype=np.float64)
    if getattr(grid, "dim", 2) == 3:
        from .config import freestream_primitive3
        from .native3d import DevicePlan3
        if flow.turbulence is not None and grid.distance is None:
            raise ValueError("a 3D plan for the SA model needs its wall distance (build_plan3d with_distance)")
        device = DevicePlan3(grid, np.array(freestream_primitive3(flow)), flow.gamma, numerics.flux, numerics.limiter,
                             numerics.kappa, None if flow.inviscid else flow.mu_inf, flow.sutherland_ratio,
                             ImplicitConfig(), c_cr1=0.3 if flow.turbulence == "sa_noft2_qcr" else 0.0)
        return ResidualOperator(grid, flow, numerics, first_order, device)
    if flow.turbulence is not None and grid.distance is None:
        from .plan import wall_distance
        grid.distance = grid.pack(wall_distance(grid.mesh, grid.walls), 1.0)
    from .native import DevicePlan
    return ResidualOperator(grid, flow, numerics, first_order, DevicePlan(grid, flow, numerics, ImplicitConfig()))
