"""The benchmark workloads as two-JSON case documents.

Seeded synthetic inputs stand in for nothing external: every case is a generated NACA
4-digit section on a generated grid, so the same documents give the same grids here,
on a GPU box and in the oracle.

* ``o_euler_257`` -- 2D Euler, NACA 0012, single-block O-grid 257 x 65 nodes (256 x 64
  cells), far field at 50 chords, M 0.8, alpha 1.25 deg, HLLC with MUSCL van Albada,
  4 variables, freestream start, converged when the density residual has dropped 1e-10
  below its running peak.
* ``c_sa_385`` -- 2D SA-noft2 RANS, NACA 4412, single-block C-grid 385 x 97 nodes (256
  cells round the airfoil, 64 along each wake side, 96 normal), first cell 1e-6 chord with
  a normal growth starting at 1.1 and rising linearly to reach the far field at 50
  chords, Re 6e6, M 0.2, alpha 8 deg, Roe with MUSCL minmod, 5 variables, GMRES restart
  30, steps bounded to 20 % relative change, the CFL ramp allowed up to 1e5.  Minmod's
  kink keeps Newton from converging the residual on this grid: with the reference's
  default CFL ceiling of 1e3 the solution wanders on a limiter limit cycle (CL within
  +-5e-5 over 8000 steps, never settling); with the ramp allowed to 1e5 the limiter's
  switches freeze and the forces settle to 1e-8 within about 700 steps while the residual
  stalls 3.5 orders below its peak.  A solve therefore ends by the reference's own exit
  test: converged at 1e-12 of the peak, or settled once CL, CD and CM each vary by less
  than 1e-6 over the last quarter of the run (a hundredth of a drag count).
"""

from __future__ import annotations

import copy

from .case import Case, parse_case

WORKLOADS = {
    "o_euler_257": (
        {"general": {"case_name": "o_euler_257"},
         "domain": {"grid": "o_grid", "airfoil": "naca0012", "cells_airfoil": 256, "cells_normal": 64,
                    "wall_spacing": 1e-3, "far_field": 50.0},
         "boundary_conditions": {"wall": {"type": "slip_wall"}, "farfield": {"type": "far_field"}},
         "freestream": {"mach": 0.8, "alpha_deg": 1.25}},
        {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "van_albada"},
         "time_integration": {"solver": "implicit"},
         "convergence": {"max_iters": 6000, "tol": 1e-10, "forces_tol": None, "block_iters": 20}},
    ),
    "c_sa_385": (
        {"general": {"case_name": "c_sa_385"},
         "domain": {"grid": "c_grid", "airfoil": "naca4412", "cells_airfoil": 256, "cells_wake": 64,
                    "cells_normal": 96, "wall_spacing": 1e-6, "far_field": 50.0, "normal_stretching": 1.1},
         "boundary_conditions": {"wall": {"type": "no_slip_wall"}, "farfield": {"type": "far_field"}},
         "freestream": {"mach": 0.2, "alpha_deg": 8.0, "reynolds": 6e6},
         "turbulence": {"model": "sa_noft2"}},
        {"convective_fluxes": {"riemann_solver": "roe", "limiter": "minmod"},
         "time_integration": {"solver": "implicit"},
         "implicit": {"krylov_subspace": 30, "max_relative_update": 0.2, "cfl_max": 1e5},
         "convergence": {"max_iters": 4000, "tol": 1e-12, "forces_tol": 1e-6, "block_iters": 20}},
    ),
}


def workload(name: str, **numerical) -> Case:
    """The case of a named workload; ``numerical`` entries ``section.key=value`` override."""
    case_doc, num_doc = copy.deepcopy(WORKLOADS[name])
    for path, value in numerical.items():
        section, key = path.split(".")
        num_doc.setdefault(section, {})[key] = value
    return parse_case(case_doc, num_doc)
