"""The two-JSON case format: ``case.json`` (what is solved) and ``numerical.json`` (how).

The keys, types, defaults and cross-key rules are those of the reference's schema and
loader (``src/jaxrans/case/schema.py:67-216``, ``src/jaxrans/case/loader.py:79-373``),
so a case directory written for the reference loads here unchanged.  Unknown keys are
errors naming the key; options jaxrans_b200 does not implement (CGNS and multi-element
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


# what each schema type accepts (a bool is neither a number nor an integer)
_ACCEPTS = {
    "number": lambda v: isinstance(v, (int, float)) and not isinstance(v, bool),
    "integer": lambda v: isinstance(v, int) and not isinstance(v, bool),
    "string": lambda v: isinstance(v, str),
    "boolean": lambda v: isinstance(v, bool),
    "list": lambda v: isinstance(v, list),
}


@dataclass(frozen=True)
class Key:
    """One key of a section: its type (``"|null"`` when null is allowed), its default
    (``REQUIRED`` when it has none), the values implemented, and for domain keys the grid
    sources that take it and those that require it."""

    name: str
    type: str
    default: Any
    choices: tuple | None = None
    grids: tuple | None = None
    required_for: tuple = ()

    def problem(self, path: str, value: Any) -> str | None:
        """What is wrong with ``value`` at ``path``, worded for the user; None if nothing."""
        kind, _, null = self.type.partition("|")
        if value is None:
            return None if null == "null" else f"'{path}' may not be null"
        if not _ACCEPTS[kind](value):
            article = "an" if kind[0] in "aeiou" else "a"
            return f"'{path}' must be {article} {kind}, got {value!r}"
        if self.choices is not None and value not in self.choices:
            return f"'{path}' = {value!r} is not implemented; choose from {sorted(self.choices)}"
        return None


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
        # a key of jaxrans_b200's own: the normal-step growth (null: solved to reach the far field)
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
                 # a key of jaxrans_b200's own: the plain FP64 path or the mixed form
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
            raise CaseError(f"'domain.grid' = {self.grid!r} is not implemented in jaxrans_b200; "
                            f"choose from {sorted(BUILT_GRIDS)}")
        if self.grid == "file":
            from .gridfile import PatchRule, load_grid, read_plot3d_2d
            from .gridfile3d import is_3d, load_grid3d
            path = self.resolve(base)
            if self.format == "cgns" or path.suffix.lower() == ".cgns":
                raise CaseError("a CGNS grid file is not implemented in jaxrans_b200; use Plot3D")
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
            raise CaseError("'domain.trailing_edge' = 'close' on a blunt section is not implemented in jaxrans_b200")
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


# --- reading a document against its schema ------------------------------------------------


def _fields(container: dict, name: str, allowed, where: str, required: bool = False) -> dict:
    """The object ``container[name]`` without its ``notes``: it must be a JSON object
    whose keys are all in ``allowed``.  Absent: {} (or ``CaseError`` when required)."""
    if name not in container:
        if required:
            raise CaseError(f"missing section '{name}'")
        return {}
    obj = container[name]
    if not isinstance(obj, dict):
        raise CaseError(f"'{where}' must be an object, got {type(obj).__name__}")
    stray = sorted(f"{where}.{k}" for k in obj if k not in allowed and k != "notes")
    if stray:
        raise CaseError(f"unknown key(s) {stray}; allowed: {sorted(allowed)}")
    return {k: v for k, v in obj.items() if k != "notes"}


def _complete(given: dict, schema: tuple, where: str) -> dict:
    """Every key of ``schema``: the given value once checked, else the key's default."""
    values = {}
    for key in schema:
        path = f"{where}.{key.name}"
        if key.name in given:
            message = key.problem(path, given[key.name])
            if message:
                raise CaseError(message)
            values[key.name] = given[key.name]
        elif key.default is REQUIRED:
            raise CaseError(f"missing '{path}'")
        else:
            values[key.name] = key.default
    return values


class Document:
    """One of the two JSON documents read against its schema (``FILES[file]``): an unknown
    section or key, a value of the wrong type, or an option not implemented is a
    ``CaseError`` naming it; ``given(name)`` is what the document wrote in a section,
    ``values(name)`` every key of it with the defaults filled in."""

    def __init__(self, doc: dict, file: str):
        self.doc, self.file, self.schema = doc, file, FILES[file]
        extra = {"boundary_conditions"} if file == CASE_FILE else set()
        stray = sorted(set(doc) - set(self.schema) - extra)
        if stray:
            raise CaseError(f"{file}: unknown section(s) {stray}; allowed: {sorted(self.schema)}")

    def given(self, name: str, required: bool = False) -> dict:
        return _fields(self.doc, name, {k.name for k in self.schema[name]}, name, required)

    def values(self, name: str, required: bool = False) -> dict:
        return _complete(self.given(name, required), self.schema[name], name)


def _raise_first(problems) -> None:
    """Raise the first message a rule generator yields, if any."""
    for message in problems:
        raise CaseError(message)


# --- cross-key rules, each a generator of messages in the order they are checked -----------


def _domain_problems(written: dict, domain: dict):
    kind = domain["grid"]
    table = keys(CASE_FILE, "domain")
    foreign = sorted(k for k in written if table[k].grids is not None and kind not in table[k].grids)
    if foreign:
        takes = sorted(k for k, key in table.items() if key.grids and kind in key.grids)
        yield f"'domain.{foreign[0]}' does not apply to grid {kind!r}; it takes {takes}"
    for name, key in table.items():
        if kind in key.required_for and domain[name] is None:
            yield f"'domain.{name}' is required for grid {kind!r}"
    if kind not in BUILT_GRIDS:
        yield f"'domain.grid' = {kind!r} is not implemented in jaxrans_b200; choose from {sorted(BUILT_GRIDS)}"


def _flow_problems(written_material: dict, written_turbulence: dict, freestream: dict, material: dict,
                   turbulence: dict):
    if freestream["reynolds"] is None:
        for key in ("dynamic_viscosity", "prandtl_number", "sutherland_temperature"):
            if key in written_material:
                yield f"'material_properties.{key}' given for an inviscid case (freestream.reynolds is null)"
    else:
        if material["dynamic_viscosity"] == "sutherland":
            if freestream["temperature"] is None or material["sutherland_temperature"] is None:
                yield ("Sutherland's law needs 'freestream.temperature' and "
                       "'material_properties.sutherland_temperature', in one absolute unit")
        elif material["sutherland_temperature"] is not None:
            yield "'material_properties.sutherland_temperature' given with a constant viscosity"
        if material["prandtl_number"] != PRANDTL_LAMINAR:
            yield (f"'material_properties.prandtl_number' = {material['prandtl_number']} is not implemented; "
                   f"only {PRANDTL_LAMINAR}")
    if turbulence["model"] != "none" and freestream["reynolds"] is None:
        yield "'turbulence.model' needs a viscous case (freestream.reynolds)"
    if turbulence["model"] == "none" and "freestream_nu_tilde_ratio" in written_turbulence:
        yield "'turbulence.freestream_nu_tilde_ratio' given without a model"
    if freestream["sweep_deg"] is not None:
        yield "'freestream.sweep_deg' (an infinite swept wing) is not implemented in jaxrans_b200"


def _patch_problems(where: str, entry, inviscid: bool):
    if not isinstance(entry, dict):
        yield f"'{where}' must be an object with a 'type', got {entry!r}"
        return
    table = {k.name: k for k in BOUNDARY_KEYS}
    stray = sorted(f"{where}.{k}" for k in entry if k not in table and k != "notes")
    if stray:
        yield f"unknown key(s) {stray}; allowed: {sorted(table)}"
    if "type" not in entry:
        yield f"missing '{where}.type'"
    for name in entry:
        if name != "notes":
            message = table[name].problem(f"{where}.{name}", entry[name])
            if message:
                yield message
    if "model" in entry and entry["type"] != "far_field":
        yield f"'{where}.model' applies to a far_field patch only"
    if entry["type"] == "no_slip_wall" and inviscid:
        yield f"'{where}.type' = 'no_slip_wall' in an inviscid case (freestream.reynolds is null)"


# --- the parts of a case --------------------------------------------------------------------


def _grid_spec(case: Document) -> GridSpec:
    written = case.given("domain", required=True)
    if "grid" not in written:
        raise CaseError(f"missing 'domain.grid'; choose from {sorted(GRIDS)}")
    d = case.values("domain")
    _raise_first(_domain_problems(written, d))
    return GridSpec(grid=d["grid"], airfoil=d["airfoil"], cells_airfoil=d["cells_airfoil"],
                    cells_wake=d["cells_wake"], cells_normal=d["cells_normal"], wall_spacing=d["wall_spacing"],
                    far_field=d["far_field"], trailing_edge=d["trailing_edge"],
                    normal_stretching=d["normal_stretching"], reference_length=d["reference_length"],
                    reference_area=d["reference_area"], moment_centre=tuple(d["moment_centre"]), file=d["file"],
                    format=d["format"], coordinate_scale=d["coordinate_scale"], patches=tuple(d["patches"] or ()))


def _flow_of(case: Document) -> FlowConditions:
    written = {n: case.given(n, required=n == "freestream") for n in ("freestream", "material_properties",
                                                                       "turbulence")}
    fs, mat, turb = (_complete(written[n], case.schema[n], n) for n in written)
    _raise_first(_flow_problems(written["material_properties"], written["turbulence"], fs, mat, turb))
    sutherland = None
    if fs["reynolds"] is not None and mat["dynamic_viscosity"] == "sutherland":
        sutherland = mat["sutherland_temperature"] / fs["temperature"]
    try:
        return FlowConditions(mach=fs["mach"], alpha_deg=fs["alpha_deg"], reynolds=fs["reynolds"],
                              gamma=mat["specific_heat_ratio"], sutherland_ratio=sutherland,
                              turbulence=None if turb["model"] == "none" else turb["model"],
                              nu_tilde_ratio=turb["freestream_nu_tilde_ratio"])
    except ValueError as error:
        raise CaseError(str(error)) from None


def flow_conditions(case_doc: dict) -> FlowConditions:
    """The flow a ``case.json`` document describes (its freestream, material and
    turbulence sections)."""
    return _flow_of(Document(case_doc, CASE_FILE))


def implicit_config(numerical_doc: dict) -> ImplicitConfig:
    """The implicit solver's settings a ``numerical.json`` document gives."""
    try:
        return ImplicitConfig(**Document(numerical_doc, NUMERICAL_FILE).values("implicit"))
    except ValueError as error:
        raise CaseError(str(error)) from None


def default_conditions(flow: FlowConditions) -> dict[str, str]:
    """The condition of a patch the case does not name, by the patch's name."""
    return {"wall": "slip_wall" if flow.inviscid else "no_slip_wall", "farfield": "far_field",
            "symmetry": "symmetry", "inflow": "inflow_total", "outflow": "outflow_static"}


def _boundaries(case_doc: dict, flow: FlowConditions) -> tuple[dict, str]:
    """The conditions the case names (patch -> kind) and the one far-field model."""
    section = case_doc.get("boundary_conditions", {})
    if not isinstance(section, dict):
        raise CaseError("'boundary_conditions' must be an object")
    entries = {patch: entry for patch, entry in section.items() if patch != "notes"}
    for patch, entry in entries.items():
        _raise_first(_patch_problems(f"boundary_conditions.{patch}", entry, flow.inviscid))
    models = sorted({e.get("model", "freestream") for e in entries.values() if e["type"] == "far_field"})
    if len(models) > 1:
        raise CaseError(f"far-field patches name different models {models}; one model per case")
    return {p: e["type"] for p, e in entries.items()}, FAR_FIELD_MODELS[models[0] if models else "freestream"]


def resolve_conditions(named: dict, grid_patches: list, flow: FlowConditions) -> dict:
    """Every grid patch's condition: the one the case names, else its name's default."""
    unknown = [p for p in named if p not in grid_patches]
    if unknown:
        raise CaseError(f"'boundary_conditions' names patch(es) {unknown} the grid does not have; "
                        f"its patches are {grid_patches}")
    defaults = default_conditions(flow)
    missing = [p for p in grid_patches if p not in named and p not in defaults]
    if missing:
        raise CaseError(f"no boundary condition for patch(es) {missing}: give each a 'type' in "
                        f"'boundary_conditions' (the grid's patches are {grid_patches})")
    return {p: named.get(p, defaults.get(p)) for p in grid_patches}


# what jaxrans_b200 refuses among the options the schema accepts: (file section, key, accepted
# value, message)
_NOT_BUILT = (
    ("time_integration", "solver", "implicit",
     "'time_integration.solver' = 'explicit' (multistage Runge-Kutta) is not implemented in jaxrans_b200; set it "
     "to 'implicit'"),
    ("implicit", "jacobian", "first_order",
     "'implicit.jacobian' = 'exact' is not implemented in jaxrans_b200; use 'first_order'"),
    ("convergence", "grid_sequencing", 0,
     "'convergence.grid_sequencing' other than 0 is not implemented in jaxrans_b200"),
)


def parse_case(case_doc: dict, numerical_doc: dict, directory: Path = Path(".")) -> Case:
    """A ``Case`` from the two documents (``src/jaxrans/case/loader.py:273-323``);
    ``CaseError`` names the offending key."""
    case, numerical = Document(case_doc, CASE_FILE), Document(numerical_doc, NUMERICAL_FILE)
    general = case.values("general", required=True)
    spec = _grid_spec(case)
    flow = _flow_of(case)
    if "section" in case_doc["domain"]:
        raise CaseError("'domain.section' applies to a swept case only ('freestream.sweep_deg')")
    conditions, far_field = _boundaries(case_doc, flow)
    sections = {n: numerical.values(n) for n in ("convective_fluxes", "time_integration", "implicit", "convergence")}
    for section, key, built, message in _NOT_BUILT[:2]:
        if sections[section][key] != built:
            raise CaseError(message)
    fluxes, stepping, conv = sections["convective_fluxes"], sections["time_integration"], sections["convergence"]
    try:
        imp = ImplicitConfig(**sections["implicit"])
        numerics = NumericsConfig(flux=fluxes["riemann_solver"], limiter=fluxes["limiter"],
                                  kappa=fluxes["muscl_kappa"], cfl=stepping["cfl"], max_iters=conv["max_iters"],
                                  tol=conv["tol"], forces_tol=conv["forces_tol"], solver=stepping["solver"],
                                  far_field=far_field)
    except (ValueError, KeyError) as error:
        raise CaseError(str(error)) from None
    block_iters = conv["block_iters"] or 20
    if block_iters < 1:
        raise CaseError(f"'convergence.block_iters' must be >= 1, got {block_iters}")
    section, key, built, message = _NOT_BUILT[2]
    if sections[section][key] != built:
        raise CaseError(message)
    out = Path(general["save_path"])
    directory = Path(directory)
    return Case(name=general["case_name"], description=general["description"] or general["case_name"],
                output=out if out.is_absolute() else directory / out, grid_spec=spec, conditions=conditions,
                flow=flow, numerics=numerics, implicit=imp, block_iters=block_iters, directory=directory,
                raw={"case": case_doc, "numerical": numerical_doc})


# --- case directories and overrides ----------------------------------------------------------

_OVERRIDE_FILES = ("case", "numerical")


def apply_override(docs: dict, assignment: str) -> None:
    """Set one ``file.section.key=value`` in the raw documents (``file`` is case or
    numerical; the value is read as JSON, else taken as a bare string), as the
    reference's ``--set`` does (``src/jaxrans/case/loader.py:329-346``)."""
    path, eq, text = assignment.partition("=")
    if not eq:
        raise CaseError(f"override {assignment!r} is not of the form file.section.key=value")
    where = path.strip().split(".")
    if len(where) != 3 or where[0] not in docs:
        raise CaseError(f"override path {path!r} must be {'|'.join(_OVERRIDE_FILES)}.section.key, "
                        f"e.g. numerical.convective_fluxes.limiter")
    file, section, key = where
    try:
        value = json.loads(text)
    except json.JSONDecodeError:
        value = text
    docs[file].setdefault(section, {})[key] = value


def _read_json(path: Path) -> dict:
    if not path.is_file():
        return {}
    try:
        return json.loads(path.read_text())
    except json.JSONDecodeError as error:
        raise CaseError(f"{path}: {error}") from None


def load_case(directory: str | Path, overrides: tuple[str, ...] = ()) -> Case:
    """A case directory (``case.json`` and, optional, ``numerical.json``) with overrides
    applied, parsed (``src/jaxrans/case/loader.py:349-373``): ``FileNotFoundError`` when
    there is no ``case.json``, ``CaseError`` prefixed with the directory otherwise."""
    directory = Path(directory)
    if not (directory / CASE_FILE).is_file():
        raise FileNotFoundError(f"{directory} holds no {CASE_FILE}")
    docs = copy.deepcopy({"case": _read_json(directory / CASE_FILE),
                          "numerical": _read_json(directory / NUMERICAL_FILE)})
    for assignment in overrides:
        apply_override(docs, assignment)
    try:
        return parse_case(docs["case"], docs["numerical"], directory)
    except CaseError as error:
        raise CaseError(f"{directory}: {error}") from None
