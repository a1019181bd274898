#!/usr/bin/env python3
"""Record the reference loader's error messages on malformed case documents.

Each entry mutates a valid pair of documents (a C-grid SA case) in one way -- an unknown
section or key, a wrong type, an option not in the schema, a cross-key rule broken, a bad
boundary condition, a malformed override -- and records the ``CaseError`` message the
reference's own ``parse_case`` / ``apply_override`` raise (under the NumPy stand-in for
JAX in ``tests/golden/jaxshim``).  ``tests/test_case_errors.py`` checks that jaxrans_b200's
loader raises the same messages.

    JAXRANS_REFERENCE=<reference checkout> python tests/golden/make_golden_case_errors.py

writes ``tests/golden/case_errors.json``.
"""

from __future__ import annotations

import copy
import json
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
if "JAXRANS_REFERENCE" not in os.environ:
    raise SystemExit("set JAXRANS_REFERENCE to the reference source checkout (the directory holding src/jaxrans)")
sys.path.insert(0, str(HERE / "jaxshim"))
sys.path.insert(1, str(Path(os.environ["JAXRANS_REFERENCE"]) / "src"))

from jaxrans.case.loader import CaseError, apply_override, parse_case  # noqa: E402

BASE_CASE = {"general": {"case_name": "base"},
             "domain": {"grid": "c_grid", "airfoil": "naca0012", "cells_airfoil": 32, "cells_wake": 8,
                        "cells_normal": 16, "wall_spacing": 1e-4, "far_field": 20.0},
             "freestream": {"mach": 0.2, "alpha_deg": 2.0, "reynolds": 1e6},
             "turbulence": {"model": "sa_noft2"}}
BASE_NUMERICAL = {"convective_fluxes": {"riemann_solver": "roe", "limiter": "minmod"},
                  "time_integration": {"solver": "implicit"}}

# (name, file, dotted path, value); the value "<delete>" removes the key
MUTATIONS = [
    ("unknown_section", "case", "extra", {"a": 1}),
    ("unknown_numerical_section", "numerical", "solver_extras", {}),
    ("unknown_key", "case", "domain.cells_around", 3),
    ("missing_case_name", "case", "general.case_name", "<delete>"),
    ("missing_freestream", "case", "freestream", "<delete>"),
    ("missing_mach", "case", "freestream.mach", "<delete>"),
    ("section_not_object", "case", "turbulence", "sa"),
    ("wrong_type_number", "case", "freestream.mach", "0.2"),
    ("wrong_type_integer", "case", "domain.cells_airfoil", 32.5),
    ("bool_not_number", "case", "freestream.alpha_deg", True),
    ("not_nullable", "case", "freestream.alpha_deg", None),
    ("unknown_limiter", "numerical", "convective_fluxes.limiter", "superbee"),
    ("unknown_flux", "numerical", "convective_fluxes.riemann_solver", "ausm"),
    ("unknown_preconditioner", "numerical", "implicit.preconditioner", "ilu"),
    ("missing_grid", "case", "domain.grid", "<delete>"),
    ("unknown_grid", "case", "domain.grid", "h_grid"),
    ("foreign_domain_key", "case", "domain.file", "grid.x"),
    ("missing_cells_wake", "case", "domain.cells_wake", "<delete>"),
    ("inviscid_viscosity", "case", "material_properties", {"dynamic_viscosity": "sutherland"}),
    ("sutherland_no_temperature", "case", "material_properties",
     {"dynamic_viscosity": "sutherland", "sutherland_temperature": 110.4}),
    ("sutherland_temperature_constant", "case", "material_properties", {"sutherland_temperature": 110.4}),
    ("prandtl", "case", "material_properties", {"prandtl_number": 0.7}),
    ("nu_tilde_without_model", "case", "turbulence", {"model": "none", "freestream_nu_tilde_ratio": 5.0}),
    ("bc_not_object", "case", "boundary_conditions", ["wall"]),
    ("bc_entry_not_object", "case", "boundary_conditions", {"wall": "no_slip_wall"}),
    ("bc_unknown_key", "case", "boundary_conditions", {"wall": {"type": "no_slip_wall", "roughness": 1}}),
    ("bc_missing_type", "case", "boundary_conditions", {"wall": {"model": "freestream"}}),
    ("bc_unknown_type", "case", "boundary_conditions", {"wall": {"type": "porous_wall"}}),
    ("bc_model_not_far_field", "case", "boundary_conditions", {"wall": {"type": "no_slip_wall",
                                                                         "model": "point_vortex"}}),
    ("bc_two_models", "case", "boundary_conditions", {"farfield": {"type": "far_field", "model": "point_vortex"},
                                                      "outer": {"type": "far_field"}}),
    ("block_iters", "numerical", "convergence", {"block_iters": -2}),
]
# inviscid variants: the base case without a Reynolds number or turbulence model
INVISCID = [
    ("inviscid_dynamic_viscosity", "case", "material_properties", {"dynamic_viscosity": "constant"}),
    ("inviscid_turbulence", "case", "turbulence", {"model": "sa_noft2"}),
    ("inviscid_no_slip", "case", "boundary_conditions", {"wall": {"type": "no_slip_wall"}}),
]
OVERRIDES = ["numerical.convective_fluxes.limiter", "limiter=none", "solver.limiter=none",
             "mesh.domain.grid=o_grid"]


def mutated(docs, file, path, value):
    docs = copy.deepcopy(docs)
    node = docs[file]
    *head, last = path.split(".")
    for part in head:
        node = node.setdefault(part, {})
    if value == "<delete>":
        node.pop(last, None)
    else:
        node[last] = value
    return docs


def message(docs) -> str | None:
    try:
        parse_case(docs["case"], docs["numerical"])
    except CaseError as error:
        return str(error)
    return None


def main() -> int:
    base = {"case": BASE_CASE, "numerical": BASE_NUMERICAL}
    inviscid = mutated(mutated(base, "case", "freestream.reynolds", "<delete>"), "case", "turbulence", "<delete>")
    out = {"base_case": BASE_CASE, "base_numerical": BASE_NUMERICAL, "parse": [], "override": []}
    for label, start, mutations in (("viscous", base, MUTATIONS), ("inviscid", inviscid, INVISCID)):
        for name, file, path, value in mutations:
            text = message(mutated(start, file, path, value))
            assert text is not None, name
            out["parse"].append({"name": name, "base": label, "file": file, "path": path, "value": value,
                                 "message": text})
    for assignment in OVERRIDES:
        try:
            apply_override(copy.deepcopy(base), assignment)
            text = None
        except CaseError as error:
            text = str(error)
        assert text is not None, assignment
        out["override"].append({"assignment": assignment, "message": text})
    (HERE / "case_errors.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"{len(out['parse'])} parse errors, {len(out['override'])} override errors -> case_errors.json")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
