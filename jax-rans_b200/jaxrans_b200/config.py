"""Frozen run configurations: the flow, the discretization and the implicit solver.

The fields, defaults and checks are those of the reference's configs
(``src/jaxrans/core/config.py:21-212``), so a case parsed here means the same
thing as there.  Everything is FP64 on the device unless the mixed form is asked
for (``precision``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

GAMMA_AIR = 1.4
PRANDTL_LAMINAR = 0.72
PRANDTL_TURBULENT = 0.9
MIN_DENSITY = 1.0e-10
MIN_PRESSURE = 1.0e-10

TURBULENCE_MODELS = ("sa_noft2", "sa_noft2_qcr")
SOLVERS = ("explicit", "implicit")
FLUXES = ("hllc", "roe")
LIMITERS = ("minmod", "none", "van_albada", "van_albada_smooth")
PRECONDITIONERS = ("line_j", "line_j_coupled", "none")
FAR_FIELDS = ("characteristic", "characteristic_point_vortex")
PRECISIONS = ("fp64", "mixed")


@dataclass(frozen=True)
class FlowConditions:
    """Freestream and gas (``core/config.py:21-105``): ``reynolds=None`` is
    inviscid, ``sutherland_ratio`` is ``S / T_inf``, ``nu_tilde_ratio`` the far-field
    ``nu~ / nu``."""

    mach: float
    alpha_deg: float = 0.0
    reynolds: float | None = None
    gamma: float = GAMMA_AIR
    sutherland_ratio: float | None = None
    turbulence: str | None = None
    nu_tilde_ratio: float = 3.0
    sweep_deg: float | None = None

    def __post_init__(self) -> None:
        if not self.mach > 0.0:
            raise ValueError(f"mach must be positive, got {self.mach}")
        if self.sweep_deg is not None:
            raise ValueError("sweep_deg (an infinite swept wing, 2.5D) is not implemented in jaxrans_b200")
        if self.mach >= 1.0:
            raise ValueError(f"freestream mach must be subsonic for the characteristic far-field BC, "
                             f"got {self.mach}")
        if not self.gamma > 1.0:
            raise ValueError(f"gamma must exceed 1, got {self.gamma}")
        if self.reynolds is not None and not self.reynolds > 0.0:
            raise ValueError(f"reynolds must be positive or None, got {self.reynolds}")
        if self.sutherland_ratio is not None:
            if self.reynolds is None:
                raise ValueError("sutherland_ratio given for an inviscid case")
            if not self.sutherland_ratio > 0.0:
                raise ValueError(f"sutherland_ratio must be positive, got {self.sutherland_ratio}")
        if self.turbulence is not None:
            if self.turbulence not in TURBULENCE_MODELS:
                raise ValueError(f"turbulence must be one of {TURBULENCE_MODELS}, got {self.turbulence!r}")
            if self.reynolds is None:
                raise ValueError("a turbulence model needs a Reynolds number")
        if not self.nu_tilde_ratio > 0.0:
            raise ValueError(f"nu_tilde_ratio must be positive, got {self.nu_tilde_ratio}")
        if abs(self.alpha_deg) > 90.0:
            raise ValueError(f"alpha_deg out of range, got {self.alpha_deg}")

    @property
    def inviscid(self) -> bool:
        return self.reynolds is None

    @property
    def alpha_rad(self) -> float:
        return float(np.deg2rad(self.alpha_deg))

    @property
    def mu_inf(self) -> float:
        if self.reynolds is None:
            raise ValueError("mu_inf is undefined for an inviscid case")
        return self.mach / self.reynolds

    @property
    def nvar(self) -> int:
        """Conserved variables on a 2D grid: 4, or 5 with the SA row."""
        return 4 if self.turbulence is None else 5


@dataclass(frozen=True)
class NumericsConfig:
    """Discretization and stepping (``core/config.py:113-154``)."""

    flux: str = "hllc"
    limiter: str = "minmod"
    cfl: float = 1.5
    max_iters: int = 40_000
    tol: float = 1.0e-12
    forces_tol: float | None = 1.0e-4
    n_ghost: int = 2
    solver: str = "explicit"
    far_field: str = "characteristic"
    kappa: float = 0.0

    def __post_init__(self) -> None:
        if self.flux not in FLUXES:
            raise KeyError(f"unknown flux '{self.flux}'. Available: {sorted(FLUXES)}")
        if self.limiter not in LIMITERS:
            raise KeyError(f"unknown limiter '{self.limiter}'. Available: {sorted(LIMITERS)}")
        if not self.cfl > 0.0:
            raise ValueError(f"cfl must be positive, got {self.cfl}")
        if self.max_iters < 1:
            raise ValueError(f"max_iters must be >= 1, got {self.max_iters}")
        if not 0.0 < self.tol < 1.0:
            raise ValueError(f"tol must lie in (0, 1), got {self.tol}")
        if self.forces_tol is not None and not self.forces_tol > 0.0:
            raise ValueError(f"forces_tol must be positive or null, got {self.forces_tol}")
        if self.n_ghost != 2:
            raise ValueError(f"n_ghost must be 2 in jaxrans_b200 (the MUSCL stencil), got {self.n_ghost}")
        if not -1.0 <= self.kappa <= 1.0:
            raise ValueError(f"muscl_kappa must lie in [-1, 1], got {self.kappa}")
        if self.kappa != 0.0 and self.limiter != "none":
            raise ValueError("muscl_kappa other than 0 is implemented without a limiter only "
                             f"(limiter 'none'), got limiter {self.limiter!r}")
        if self.solver not in SOLVERS:
            raise ValueError(f"solver must be one of {SOLVERS}, got {self.solver!r}")
        if self.far_field not in FAR_FIELDS:
            raise ValueError(f"far field model {self.far_field!r} is not available; available: {FAR_FIELDS}")


@dataclass(frozen=True)
class ImplicitConfig:
    """Pseudo-transient Newton-Krylov settings (``core/config.py:158-212``), plus
    ``precision``: ``fp64`` (the plain path) or ``mixed`` (FP32 line
    preconditioner and Krylov basis, FP64 residual, update, least squares and forces)."""

    cfl: float = 10.0
    cfl_max: float = 1.0e3
    cfl_growth: float = 1.3
    cfl_cutback: float = 4.0
    cfl_min: float = 0.5
    preconditioner: str = "line_j"
    jacobian: str = "first_order"
    krylov_tol: float = 1.0e-2
    krylov_subspace: int = 10
    krylov_restarts: int = 2
    krylov_success: float = 0.5
    max_relative_update: float | None = None
    precision: str = "fp64"

    def __post_init__(self) -> None:
        if not self.cfl > 0.0:
            raise ValueError(f"cfl must be positive, got {self.cfl}")
        if self.cfl_max < self.cfl:
            raise ValueError(f"cfl_max must be at least the starting cfl {self.cfl}, got {self.cfl_max}")
        if not 0.0 < self.cfl_min <= self.cfl:
            raise ValueError(f"cfl_min must lie in (0, cfl], got {self.cfl_min}")
        if self.cfl_growth < 1.0:
            raise ValueError(f"cfl_growth must be >= 1, got {self.cfl_growth}")
        if self.cfl_cutback <= 1.0:
            raise ValueError(f"cfl_cutback must exceed 1, got {self.cfl_cutback}")
        if self.jacobian not in ("exact", "first_order"):
            raise ValueError(f"jacobian must be 'exact' or 'first_order', got {self.jacobian!r}")
        if self.preconditioner not in PRECONDITIONERS:
            raise KeyError(f"unknown preconditioner '{self.preconditioner}'. Available: {sorted(PRECONDITIONERS)}")
        if not 0.0 < self.krylov_tol < 1.0:
            raise ValueError(f"krylov_tol must lie in (0, 1), got {self.krylov_tol}")
        if self.krylov_subspace < 1:
            raise ValueError(f"krylov_subspace must be >= 1, got {self.krylov_subspace}")
        if self.krylov_subspace > 64:
            raise ValueError(f"krylov_subspace above 64 is not supported, got {self.krylov_subspace}")
        if self.krylov_restarts < 1:
            raise ValueError(f"krylov_restarts must be >= 1, got {self.krylov_restarts}")
        if self.max_relative_update is not None and not self.max_relative_update > 0.0:
            raise ValueError(f"max_relative_update must be positive or None, got {self.max_relative_update}")
        if not 0.0 < self.krylov_success < 1.0:
            raise ValueError(f"krylov_success must lie in (0, 1), got {self.krylov_success}")
        if self.precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}, got {self.precision!r}")


def freestream_primitive(flow: FlowConditions) -> tuple[float, ...]:
    """``(rho, u, v, p[, nu_hat])`` of the freestream, nondimensional
    (``core/state.py:96-139``): ``rho = 1``, ``V = M (cos a, sin a)``,
    ``p = 1/gamma``; with SA the stored ``nu~ / nu_inf`` ratio."""
    a = flow.alpha_rad
    q = (1.0, float(flow.mach * np.cos(a)), float(flow.mach * np.sin(a)), 1.0 / flow.gamma)
    return q + ((flow.nu_tilde_ratio,) if flow.turbulence is not None else ())


def freestream_primitive3(flow: FlowConditions) -> tuple[float, ...]:
    """``(rho, u, v, w, p[, nu_hat])`` of the 3D freestream: the incidence in the x-z
    plane (x chordwise, y along the span, z up), ``V = M (cos a, 0, sin a)``
    (``src/jaxrans/core/state.py:96-139``)."""
    a = flow.alpha_rad
    q = (1.0, float(flow.mach * np.cos(a)), 0.0, float(flow.mach * np.sin(a)), 1.0 / flow.gamma)
    return q + ((flow.nu_tilde_ratio,) if flow.turbulence is not None else ())
