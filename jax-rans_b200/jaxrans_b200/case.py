"""The two-JSON case format: ``case.json`` (what is solved) and ``numerical.json`` (how).

The keys, types, defaults and cross-key rules are those of the reference's schema and
loader (``src/jaxrans/case/schema.py:67-216``, ``src/jaxrans/case/loader.py:79-373``),
so a case directory written for the reference loads here unchanged.  Unknown keys are
errors naming the key; options this build does not implement (CGNS and multi-element
grids, blunt trailing edges, swept wings, the explicit solver) are refused by name.
"""

from __future__ import annotations

import copy
import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

import numpy as np

from .config import (FLUXES, LIMITERS, PRECONDITIONERS, TURBULENCE_MODELS, FlowConditions, ImplicitConfig,
                     NumericsConfig, PRANDTL_LAMINAR, GAMMA_AIR)
from .geometry import section_source
from .grid3d import KINDS_3D, Block3
from .grids import CONDITION_KINDS, WALL_KINDS, Block, c_grid, o_grid, patch_names
from .plan import Plan, build_plan

CASE_FILE, NUMERICAL_FILE = "case.json", "numerical.json"
REQUIRED = "required"


class CaseError(ValueError):
    """A case that cannot be run as written."""


@dataclass(frozen=True)
class Key:
    name: str
    type: str
    default: Any
    choices: tuple | None = None
    grids: tuple | None = None
    required_for: tuple = ()

    def check(self, path: str, value: Any) -> None:
        if value is None:
            if not self.type.endswith("|null"):
                raise TypeError(f"'{path}' may not be null")
            return
        base = self.type.split("|")[0]
        ok = {"number": lambda v: isinstance(v, (int, float)) and not isinstance(v, bool),
              "integer": lambda v: isinstance(v, int) and not isinstance(v, bool),
              "string": lambda v: isinstance(v, str),
              "boolean": lambda v: isinstance(v, bool),
              "list": lambda v: isinstance(v, list)}[base](value)
        if not ok:
            raise TypeError(f"'{path}' must be {'an' if base[0] in 'aeiou' else 'a'} {base}, got {value!r}")
        if self.choices is not None and value not in self.choices:
            raise ValueError(f"'{path}' = {value!r} is not implemented; choose from {sorted(self.choices)}")


GENERATED = ("o_grid", "c_grid")
SECTION = ("multi_element",)
MADE = GENERATED + SECTION
GRIDS = ("c_grid", "file", "multi_element", "o_grid")
BUILT_GRIDS = ("c_grid", "file", "o_grid")

CASE = {
    "general": (Key("case_name", "string", REQUIRED), Key("description", "string", None),
                Key("save_path", "string", "results")),
    "domain": (
        Key("grid", "string", REQUIRED, choices=GRIDS),
        Key("airfoil", "string", None, grids=GENERATED, required_for=GENERATED),
        Key("cells_airfoil", "integer", None, grids=GENERATED, required_for=GENERATED),
        Key("cells_wake", "integer", None, grids=("c_grid",), required_for=("c_grid",)),
        Key("cells_normal", "integer", None, grids=GENERATED, required_for=GENERATED),
        Key("wall_spacing", "number", None, grids=MADE, required_for=MADE),
        Key("trailing_edge", "string", "as_given", choices=("as_given", "close"), grids=GENERATED),
        Key("far_field", "number", 100.0, grids=MADE),
        Key("leading_edge_spacing", "number", 2e-3, grids=MADE),
        Key("trailing_edge_spacing", "number", 2e-3, grids=MADE),
        Key("elements", "list", [], grids=SECTION, required_for=SECTION),
        Key("cells_per_chord", "integer", None, grids=SECTION, required_for=SECTION),
        Key("layer_cells", "integer", 32, grids=SECTION),
        Key("layer_thickness", "number", 0.02, grids=SECTION),
        Key("gap_cells", "integer", 16, grids=SECTION),
        Key("base_blocks", "boolean", False, grids=("multi_element",)),
        Key("even_cells", "integer", 4, grids=SECTION),
        Key("file", "string", None, grids=("file", "multi_element"), required_for=("file",)),
        Key("format", "string", "auto", choices=("auto", "cgns", "plot3d"), grids=("file",)),
        Key("coordinate_scale", "number", 1.0, grids=("file", "multi_element")),
        Key("patches", "list", [], grids=("file",)),
        Key("reference_length", "number", 1.0),
        Key("reference_area", "number|null", None),
        Key("moment_centre", "list", [0.25, 0.0, 0.0]),
        Key("section", "string", "streamwise", choices=("normal", "streamwise")),
        # this build's own key: the normal-step growth (null: solved to reach the far field)
        Key("normal_stretching", "number|null", None, grids=GENERATED),
    ),
    "freestream": (Key("mach", "number", REQUIRED), Key("alpha_deg", "number", 0.0),
                   Key("sweep_deg", "number|null", None), Key("reynolds", "number|null", None),
                   Key("temperature", "number", None)),
    "material_properties": (Key("specific_heat_ratio", "number", GAMMA_AIR),
                            Key("dynamic_viscosity", "string", "constant", choices=("constant", "sutherland")),
                            Key("sutherland_temperature", "number", None),
                            Key("prandtl_number", "number", PRANDTL_LAMINAR)),
    "turbulence": (Key("model", "string", "none", choices=("none", *TURBULENCE_MODELS)),
                   Key("freestream_nu_tilde_ratio", "number", 3.0)),
}

_N, _I = NumericsConfig, ImplicitConfig
NUMERICAL = {
    "convective_fluxes": (Key("riemann_solver", "string", _N.flux, choices=tuple(sorted(FLUXES))),
                          Key("limiter", "string", _N.limiter, choices=tuple(sorted(LIMITERS))),
                          Key("muscl_kappa", "number", _N.kappa)),
    "time_integration": (Key("solver", "string", _N.solver, choices=("explicit", "implicit")),
                         Key("rk_scheme", "string", "rk5_jameson", choices=("euler", "rk4_jameson", "rk5_jameson")),
                         Key("cfl", "number", _N.cfl)),
    "implicit": (Key("cfl", "number", _I.cfl), Key("cfl_max", "number", _I.cfl_max),
                 Key("cfl_growth", "number", _I.cfl_growth), Key("cfl_cutback", "number", _I.cfl_cutback),
                 Key("cfl_min", "number", _I.cfl_min),
                 Key("preconditioner", "string", _I.preconditioner, choices=tuple(sorted(PRECONDITIONERS))),
                 Key("jacobian", "string", _I.jacobian, choices=("exact", "first_order")),
                 Key("krylov_tol", "number", _I.krylov_tol), Key("krylov_subspace", "integer", _I.krylov_subspace),
                 Key("krylov_restarts", "integer", _I.krylov_restarts),
                 Key("krylov_success", "number", _I.krylov_success),
                 Key("max_relative_update", "number|null", _I.max_relative_update),
                 # this build's own key: the plain FP64 path or the mixed form
                 Key("precision", "string", _I.precision, choices=("fp64", "mixed"))),
    "convergence": (Key("max_iters", "integer", _N.max_iters), Key("tol", "number", _N.tol),
                    Key("forces_tol", "number|null", _N.forces_tol), Key("grid_sequencing", "integer", 0),
                    Key("block_iters", "integer", None)),
}
FILES = {CASE_FILE: CASE, NUMERICAL_FILE: NUMERICAL}
BOUNDARY_KEYS = (Key("type", "string", REQUIRED, choices=CONDITION_KINDS),
                 Key("model", "string", "freestream", choices=("freestream", "point_vortex")))
FAR_FIELD_MODELS = {"freestream": "characteristic", "point_vortex": "characteristic_point_vortex"}
PATCH_RULE_KEYS = {"name", "x_min", "x_max", "y_min", "y_max", "z_min", "z_max"}


def keys(file: str, section: str) -> dict[str, Key]:
    return {k.name: k for k in FILES[file][section]}


@dataclass(frozen=True)
class GridSpec:
    grid: str = "c_grid"
    airfoil: str | None = None
    cells_airfoil: int | None = None
    cells_wake: int | None = None
    cells_normal: int | None = None
    wall_spacing: float | None = None
    far_field: float = 100.0
    trailing_edge: str = "as_given"
    normal_stretching: float | None = None
    reference_length: float = 1.0
    reference_area: float | None = None
    moment_centre: tuple = (0.25, 0.0, 0.0)
    file: str | None = None
    format: str = "auto"
    coordinate_scale: float = 1.0
    patches: tuple = ()

    def resolve(self, base: Path) -> Path:
        """The grid file, relative to the case directory or the working directory
        (``src/jaxrans/case/domain.py:122-129``)."""
        for root in (Path(base), Path.cwd()):
            path = Path(self.file) if Path(self.file).is_absolute() else root / self.file
            if path.is_file():
                return path
        raise CaseError(f"'domain.file' {self.file!r} not found in {base} or {Path.cwd()}")

    def build(self, base: Path) -> list[Block]:
        if self.grid not in BUILT_GRIDS:
            raise CaseError(f"'domain.grid' = {self.grid!r} is not implemented in this build; "
                            f"choose from {sorted(BUILT_GRIDS)}")
        if self.grid == "file":
            from .gridfile import PatchRule, load_grid, read_plot3d_2d
            from .gridfile3d import is_3d, load_grid3d
            path = self.resolve(base)
            if self.format == "cgns" or path.suffix.lower() == ".cgns":
                raise CaseError("a CGNS grid file is not implemented in this build; use Plot3D")
            try:
                rules = tuple(PatchRule(**rule) for rule in self.patches)
            except TypeError as error:
                raise CaseError(f"'domain.patches': {error}") from None
            try:
                if is_3d(path):
                    if self.reference_area is None:
                        raise CaseError("a 3D case needs 'domain.reference_area'")
                    return load_grid3d(path, self.coordinate_scale, rules)
                read_plot3d_2d(path)
                return load_grid(path, self.coordinate_scale, rules)
            except ValueError as error:
                if isinstance(error, CaseError):
                    raise
                raise CaseError(str(error)) from None
        section = section_source(self.airfoil, base).normalised()
        if self.trailing_edge == "close" and not section.sharp:
            raise CaseError("'domain.trailing_edge' = 'close' on a blunt section is not implemented in this build")
        if self.grid == "o_grid":
            return [o_grid(section, self.cells_airfoil, self.cells_normal, self.wall_spacing, self.far_field,
                           self.normal_stretching)]
        return [c_grid(section, self.cells_airfoil, self.cells_wake, self.cells_normal, self.wall_spacing,
                       self.far_field, self.normal_stretching)]


@dataclass(frozen=True)
class Case:
    """One case, resolved (``src/jaxrans/case/loader.py:35-73``)."""

    name: str
    description: str
    output: Path
    grid_spec: GridSpec
    conditions: dict
    flow: FlowConditions
    numerics: NumericsConfig
    implicit: ImplicitConfig
    block_iters: int
    directory: Path
    raw: dict = field(compare=False, repr=False)
    sequencing: int = 0

    def grid(self):
        """The grid, every patch given its condition, packed into a plan: a ``Plan``, or
        for a 3D grid file a ``plan3d.Plan3``."""
        mesh = self.grid_spec.build(self.directory)
        kinds = resolve_conditions(self.conditions, patch_names(mesh), self.flow)
        mesh = [b.with_kinds(kinds) for b in mesh]
        turbulent = self.flow.turbulence is not None
        if mesh and isinstance(mesh[0], Block3):
            from .plan3d import build_plan3d
            unsupported = sorted({k for k in kinds.values() if k not in KINDS_3D})
            if unsupported:
                raise CaseError(f"boundary condition(s) {unsupported} are not implemented on the 3D path; "
                                f"it has {sorted(KINDS_3D)}")
            if self.numerics.far_field != "characteristic":
                raise CaseError("the far-field 'model' point_vortex is a 2D model (a vortex in the plane); "
                                "a 3D case takes the freestream far field")
            return build_plan3d(mesh, with_distance=turbulent)
        return build_plan(mesh, self.numerics.n_ghost, with_distance=turbulent)


def _section(doc: dict, file: str, name: str, required: bool = False) -> dict:
    if name not in doc:
        if required:
            raise CaseError(f"missing section '{name}'")
        return {}
    section = doc[name]
    if not isinstance(section, dict):
        raise CaseError(f"'{name}' must be an object, got {type(section).__name__}")
    allowed = keys(file, name)
    unknown = set(section) - set(allowed) - {"notes"}
    if unknown:
        raise CaseError(f"unknown key(s) {sorted(f'{name}.{k}' for k in unknown)}; allowed: {sorted(allowed)}")
    return {k: v for k, v in section.items() if k != "notes"}


def _values(section: dict, file: str, name: str) -> dict:
    out = {}
    for key in FILES[file][name]:
        path = f"{name}.{key.name}"
        if key.name in section:
            try:
                key.check(path, section[key.name])
            except (TypeError, ValueError) as error:
                raise CaseError(str(error)) from None
            out[key.name] = section[key.name]
        elif key.default is REQUIRED:
            raise CaseError(f"missing '{path}'")
        else:
            out[key.name] = key.default
    return out


def _top_level(doc: dict, file: str) -> None:
    unknown = set(doc) - set(FILES[file]) - ({"boundary_conditions"} if file == CASE_FILE else set())
    if unknown:
        raise CaseError(f"{file}: unknown section(s) {sorted(unknown)}; allowed: {sorted(FILES[file])}")


def _grid_spec(case_doc: dict) -> GridSpec:
    raw = _section(case_doc, CASE_FILE, "domain", required=True)
    if "grid" not in raw:
        raise CaseError(f"missing 'domain.grid'; choose from {sorted(GRIDS)}")
    domain = _values(raw, CASE_FILE, "domain")
    kind = domain["grid"]
    ks = keys(CASE_FILE, "domain")
    foreign = sorted(k for k in raw if ks[k].grids is not None and kind not in ks[k].grids)
    if foreign:
        takes = sorted(k for k, key in ks.items() if key.grids and kind in key.grids)
        raise CaseError(f"'domain.{foreign[0]}' does not apply to grid {kind!r}; it takes {takes}")
    for name, key in ks.items():
        if kind in key.required_for and domain[name] is None:
            raise CaseError(f"'domain.{name}' is required for grid {kind!r}")
    if kind not in BUILT_GRIDS:
        raise CaseError(f"'domain.grid' = {kind!r} is not implemented in this build; choose from "
                        f"{sorted(BUILT_GRIDS)}")
    return GridSpec(grid=kind, airfoil=domain["airfoil"], cells_airfoil=domain["cells_airfoil"],
                    cells_wake=domain["cells_wake"], cells_normal=domain["cells_normal"],
                    wall_spacing=domain["wall_spacing"], far_field=domain["far_field"],
                    trailing_edge=domain["trailing_edge"], normal_stretching=domain["normal_stretching"],
                    reference_length=domain["reference_length"], reference_area=domain["reference_area"],
                    moment_centre=tuple(domain["moment_centre"]), file=domain["file"], format=domain["format"],
                    coordinate_scale=domain["coordinate_scale"], patches=tuple(domain["patches"] or ()))


def _flow(case_doc: dict) -> FlowConditions:
    given = {name: _section(case_doc, CASE_FILE, name, required=name == "freestream")
             for name in ("freestream", "material_properties", "turbulence")}
    freestream, material, turbulence = (_values(given[n], CASE_FILE, n) for n in given)
    inviscid = freestream["reynolds"] is None
    sutherland = None
    if inviscid:
        for key in ("dynamic_viscosity", "prandtl_number", "sutherland_temperature"):
            if key in given["material_properties"]:
                raise CaseError(f"'material_properties.{key}' given for an inviscid case "
                                f"(freestream.reynolds is null)")
    else:
        if material["dynamic_viscosity"] == "sutherland":
            if freestream["temperature"] is None or material["sutherland_temperature"] is None:
                raise CaseError("Sutherland's law needs 'freestream.temperature' and "
                                "'material_properties.sutherland_temperature', in one absolute unit")
            sutherland = material["sutherland_temperature"] / freestream["temperature"]
        elif material["sutherland_temperature"] is not None:
            raise CaseError("'material_properties.sutherland_temperature' given with a constant viscosity")
        if material["prandtl_number"] != PRANDTL_LAMINAR:
            raise CaseError(f"'material_properties.prandtl_number' = {material['prandtl_number']} is not "
                            f"implemented; only {PRANDTL_LAMINAR}")
    model = turbulence["model"]
    if model != "none" and inviscid:
        raise CaseError("'turbulence.model' needs a viscous case (freestream.reynolds)")
    if model == "none" and "freestream_nu_tilde_ratio" in given["turbulence"]:
        raise CaseError("'turbulence.freestream_nu_tilde_ratio' given without a model")
    if freestream["sweep_deg"] is not None:
        raise CaseError("'freestream.sweep_deg' (an infinite swept wing) is not implemented in this build")
    try:
        return FlowConditions(mach=freestream["mach"], alpha_deg=freestream["alpha_deg"],
                              reynolds=freestream["reynolds"], gamma=material["specific_heat_ratio"],
                              sutherland_ratio=sutherland, turbulence=None if model == "none" else model,
                              nu_tilde_ratio=turbulence["freestream_nu_tilde_ratio"])
    except ValueError as error:
        raise CaseError(str(error)) from None


def default_conditions(flow: FlowConditions) -> dict[str, str]:
    return {"wall": "slip_wall" if flow.inviscid else "no_slip_wall", "farfield": "far_field",
            "symmetry": "symmetry", "inflow": "inflow_total", "outflow": "outflow_static"}


def _boundaries(case_doc: dict, flow: FlowConditions) -> tuple[dict, str]:
    section = case_doc.get("boundary_conditions", {})
    if not isinstance(section, dict):
        raise CaseError("'boundary_conditions' must be an object")
    kinds, models = {}, set()
    allowed = {k.name: k for k in BOUNDARY_KEYS}
    for patch, entry in section.items():
        if patch == "notes":
            continue
        where = f"boundary_conditions.{patch}"
        if not isinstance(entry, dict):
            raise CaseError(f"'{where}' must be an object with a 'type', got {entry!r}")
        unknown = set(entry) - set(allowed) - {"notes"}
        if unknown:
            raise CaseError(f"unknown key(s) {sorted(f'{where}.{k}' for k in unknown)}; allowed: {sorted(allowed)}")
        if "type" not in entry:
            raise CaseError(f"missing '{where}.type'")
        for name in set(entry) - {"notes"}:
            try:
                allowed[name].check(f"{where}.{name}", entry[name])
            except (TypeError, ValueError) as error:
                raise CaseError(str(error)) from None
        if "model" in entry and entry["type"] != "far_field":
            raise CaseError(f"'{where}.model' applies to a far_field patch only")
        if entry["type"] == "far_field":
            models.add(entry.get("model", "freestream"))
        if entry["type"] == "no_slip_wall" and flow.inviscid:
            raise CaseError(f"'{where}.type' = 'no_slip_wall' in an inviscid case (freestream.reynolds is null)")
        kinds[patch] = entry["type"]
    if len(models) > 1:
        raise CaseError(f"far-field patches name different models {sorted(models)}; one model per case")
    return kinds, FAR_FIELD_MODELS[models.pop() if models else "freestream"]


def resolve_conditions(named: dict, grid_patches: list, flow: FlowConditions) -> dict:
    unknown = [p for p in named if p not in grid_patches]
    if unknown:
        raise CaseError(f"'boundary_conditions' names patch(es) {unknown} the grid does not have; "
                        f"its patches are {grid_patches}")
    defaults = default_conditions(flow)
    missing = [p for p in grid_patches if p not in named and p not in defaults]
    if missing:
        raise CaseError(f"no boundary condition for patch(es) {missing}")
    return {p: named.get(p, defaults.get(p)) for p in grid_patches}


def parse_case(case_doc: dict, numerical_doc: dict, directory: Path = Path(".")) -> Case:
    _top_level(case_doc, CASE_FILE)
    _top_level(numerical_doc, NUMERICAL_FILE)
    general = _values(_section(case_doc, CASE_FILE, "general", required=True), CASE_FILE, "general")
    spec = _grid_spec(case_doc)
    flow = _flow(case_doc)
    if "section" in case_doc["domain"]:
        raise CaseError("'domain.section' applies to a swept case only ('freestream.sweep_deg')")
    conditions, far_field = _boundaries(case_doc, flow)
    fluxes, stepping, implicit, convergence = (
        _values(_section(numerical_doc, NUMERICAL_FILE, n), NUMERICAL_FILE, n)
        for n in ("convective_fluxes", "time_integration", "implicit", "convergence"))
    if stepping["solver"] != "implicit":
        raise CaseError("'time_integration.solver' = 'explicit' (multistage Runge-Kutta) is not implemented in "
                        "this build; set it to 'implicit'")
    if implicit["jacobian"] != "first_order":
        raise CaseError("'implicit.jacobian' = 'exact' is not implemented in this build; use 'first_order'")
    try:
        imp = ImplicitConfig(**implicit)
        numerics = NumericsConfig(flux=fluxes["riemann_solver"], limiter=fluxes["limiter"],
                                  kappa=fluxes["muscl_kappa"], cfl=stepping["cfl"],
                                  max_iters=convergence["max_iters"], tol=convergence["tol"],
                                  forces_tol=convergence["forces_tol"], solver=stepping["solver"],
                                  far_field=far_field)
    except (ValueError, KeyError) as error:
        raise CaseError(str(error)) from None
    block_iters = convergence["block_iters"] or 20
    if block_iters < 1:
        raise CaseError(f"'convergence.block_iters' must be >= 1, got {block_iters}")
    if convergence["grid_sequencing"] != 0:
        raise CaseError("'convergence.grid_sequencing' other than 0 is not implemented in this build")
    directory = Path(directory)
    output = Path(general["save_path"])
    return Case(name=general["case_name"], description=general["description"] or general["case_name"],
                output=output if output.is_absolute() else directory / output, grid_spec=spec,
                conditions=conditions, flow=flow, numerics=numerics, implicit=imp, block_iters=block_iters,
                directory=directory, raw={"case": case_doc, "numerical": numerical_doc})


def apply_override(docs: dict, assignment: str) -> None:
    """``file.section.key=value`` (``src/jaxrans/case/loader.py:329-346``)."""
    if "=" not in assignment:
        raise CaseError(f"override {assignment!r} is not of the form file.section.key=value")
    path, text = assignment.split("=", 1)
    parts = path.strip().split(".")
    if len(parts) != 3 or parts[0] not in docs:
        raise CaseError(f"override path {path!r} must be case|numerical.section.key")
    try:
        value = json.loads(text)
    except json.JSONDecodeError:
        value = text
    docs[parts[0]].setdefault(parts[1], {})[parts[2]] = value


def load_case(directory: str | Path, overrides: tuple[str, ...] = ()) -> Case:
    """Read a case directory, apply overrides, parse (``src/jaxrans/case/loader.py:349-373``)."""
    directory = Path(directory)
    if not (directory / CASE_FILE).is_file():
        raise FileNotFoundError(f"{directory} holds no {CASE_FILE}")
    docs = {}
    for label, filename in (("case", CASE_FILE), ("numerical", NUMERICAL_FILE)):
        path = directory / filename
        try:
            docs[label] = json.loads(path.read_text()) if path.is_file() else {}
        except json.JSONDecodeError as error:
            raise CaseError(f"{path}: {error}") from None
    docs = copy.deepcopy(docs)
    for assignment in overrides:
        apply_override(docs, assignment)
    try:
        return parse_case(docs["case"], docs["numerical"], directory)
    except CaseError as error:
        raise CaseError(f"{directory}: {error}") from None
