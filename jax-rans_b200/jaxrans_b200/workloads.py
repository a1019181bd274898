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
* ``c_sa_257`` / ``c_sa_513`` / ``c_sa_769`` -- the uneven grids of the batched polar:
  SA-noft2 on C-grids of 257 x 65 (NACA 0012, M 0.15, Re 3e6), 513 x 129 (NACA 2412,
  M 0.2, Re 6e6) and 769 x 193 nodes (NACA 4415, M 0.3, Re 9e6), two thirds of the
  cells round the airfoil and a sixth along each wake side, the numerics of
  ``c_sa_385``.
* batch ``polar64_uneven`` -- 64 angles uniform on [-4, 16] deg on the ``c_sa_385``
  grid together with the three uneven cases, all in one device batch; ``polar16_uneven``,
  16 angles with the same three uneven cases, is the bounded form the benchmark times;
  ``polar8_769``,
  8 angles with the 769 x 193 case, is the same mix small enough to profile.
* ``wing_ch_4blk`` -- 3D SA-noft2 RANS round a swept, tapered wing: NACA 0012 sections,
  aspect ratio 4 (semispan 1.6 root chords), taper 0.6, leading-edge sweep 25 deg, on a
  four-block point-matched C-H grid of 193 x 65 x 81 nodes per block (3.93M cells; the
  wing and the region past its tip, each in lower and upper halves), first cell 2e-6 root
  chord, far field at 50 root chords, M 0.8, alpha 2.5 deg, Re 1e7, HLLC with MUSCL and
  the smooth van Albada limiter, 6 variables; FP64 residual, J.v and Krylov vectors, the
  coupled 6x6 line preconditioner in FP32.  ``wing_ch_4blk_small`` is the same wing on
  a grid of 49 x 17 x 17 nodes per block, for profiling and tests.  A 3D case is a grid
  file plus its documents: ``wing3d_case`` writes them into a directory and loads them.
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


def _c_sa(name: str, airfoil: str, around: int, wake: int, normal: int, mach: float, reynolds: float):
    case_doc, num_doc = copy.deepcopy(WORKLOADS["c_sa_385"])
    case_doc["general"]["case_name"] = name
    case_doc["domain"].update({"airfoil": airfoil, "cells_airfoil": around, "cells_wake": wake,
                               "cells_normal": normal})
    case_doc["freestream"].update({"mach": mach, "reynolds": reynolds})
    return case_doc, num_doc


WORKLOADS["c_sa_257"] = _c_sa("c_sa_257", "naca0012", 172, 42, 64, 0.15, 3e6)
WORKLOADS["c_sa_513"] = _c_sa("c_sa_513", "naca2412", 344, 84, 128, 0.2, 6e6)
WORKLOADS["c_sa_769"] = _c_sa("c_sa_769", "naca4415", 512, 128, 192, 0.3, 9e6)

# batches: (workload, alpha or None for the workload's own) per case
BATCHES = {
    "polar64_uneven": [("c_sa_385", float(a)) for a in
                       [-4.0 + 20.0 * k / 63 for k in range(64)]] + [("c_sa_257", None), ("c_sa_513", None),
                                                                      ("c_sa_769", None)],
    # a quarter of it, timed beside the plain FP64 line: 16 angles and the three uneven grids
    "polar16_uneven": [("c_sa_385", float(a)) for a in
                       [-4.0 + 20.0 * k / 15 for k in range(16)]] + [("c_sa_257", None), ("c_sa_513", None),
                                                                      ("c_sa_769", None)],
    # a small batch of the same kinds, for profiling captures (about 1.5 GB on the device)
    "polar8_769": [("c_sa_385", float(a)) for a in [-4.0 + 20.0 * k / 7 for k in range(8)]] + [("c_sa_769", None)],
}


def batch_workload(name: str, **numerical) -> list[Case]:
    """The cases of a named batch; ``numerical`` overrides apply to every case."""
    import dataclasses
    cases = []
    for work, alpha in BATCHES[name]:
        case = workload(work, **numerical)
        if alpha is not None:
            flow = dataclasses.replace(case.flow, alpha_deg=alpha)
            case = dataclasses.replace(case, flow=flow, name=f"{case.name}_a{alpha:+.2f}")
        cases.append(case)
    return cases



WING3D = {
    "wing_ch_4blk": {"cells_airfoil": 256, "cells_wake": 64, "cells_normal": 64, "cells_span": 80,
                     "cells_tip": 80, "wall_spacing": 2e-6, "far_field": 50.0, "cap_cells": 4},
    "wing_ch_4blk_small": {"cells_airfoil": 64, "cells_wake": 16, "cells_normal": 16, "cells_span": 16,
                           "cells_tip": 16, "wall_spacing": 1e-4, "far_field": 20.0, "cap_cells": 3},
}
WING3D_PLANFORM = {"semispan": 1.6, "taper": 0.6, "sweep_deg": 25.0}
WING3D_FLOW = {"freestream": {"mach": 0.8, "alpha_deg": 2.5, "reynolds": 1e7}, "turbulence": {"model": "sa_noft2"}}
WING3D_NUMERICS = {"convective_fluxes": {"riemann_solver": "hllc", "limiter": "van_albada_smooth"},
                   "time_integration": {"solver": "implicit"},
                   "implicit": {"krylov_subspace": 30, "max_relative_update": 0.2,
                                "preconditioner": "line_j_coupled", "precision": "mixed"},
                   "convergence": {"max_iters": 6000, "tol": 1e-10, "block_iters": 20}}


def wing3d_cells(name: str) -> int:
    """Cells of the 3D workload's grid: four blocks, each half the C round the section by
    the normal layers by the wing's or the tip region's stations."""
    w = WING3D[name]
    return 2 * (w["cells_airfoil"] // 2 + w["cells_wake"]) * w["cells_normal"] * (w["cells_span"] + w["cells_tip"])


def wing3d_case(name: str, directory, **numerical) -> Case:
    """Write the 3D workload ``name`` (its Plot3D grid ``grid.x``, ``case.json`` and
    ``numerical.json``) into ``directory`` and load it as a case."""
    import json
    from pathlib import Path
    from .case import load_case
    from .geometry import section_source
    from .grid3d import wing_ch_blocks, write_plot3d
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    grid = wing_ch_blocks(section_source("naca0012"), **WING3D[name], **WING3D_PLANFORM)
    write_plot3d(directory / "grid.x", grid.blocks)
    case_doc = {"general": {"case_name": name},
                "domain": {"grid": "file", "file": "grid.x", "patches": grid.patches,
                           "reference_area": grid.reference_area, "reference_length": grid.reference_length,
                           "moment_centre": list(grid.moment_centre)},
                "boundary_conditions": {"wall": {"type": "no_slip_wall"}, "farfield": {"type": "far_field"},
                                        "symmetry": {"type": "symmetry"}},
                **copy.deepcopy(WING3D_FLOW)}
    num_doc = copy.deepcopy(WING3D_NUMERICS)
    for path, value in numerical.items():
        section, key = path.split(".")
        num_doc.setdefault(section, {})[key] = value
    (directory / "case.json").write_text(json.dumps(case_doc, indent=1))
    (directory / "numerical.json").write_text(json.dumps(num_doc, indent=1))
    return load_case(directory)


def workload(name: str, **numerical) -> Case:
    """The case of a named workload; ``numerical`` entries ``section.key=value`` override."""
    case_doc, num_doc = copy.deepcopy(WORKLOADS[name])
    for path, value in numerical.items():
        section, key = path.split(".")
        num_doc.setdefault(section, {})[key] = value
    return parse_case(case_doc, num_doc)
