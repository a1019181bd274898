"""Result files in the reference's layout (``src/jaxrans/io/output.py:70-128``,
``src/jaxrans/simulation.py:135-169``): the resolved case and run record as JSON, the
residual and lift histories and the wall distributions as text columns, the fields and
nodes per block as ``.npz``."""

from __future__ import annotations

import dataclasses
import json
import platform
from pathlib import Path

import numpy as np


def _jsonable(obj):
    if isinstance(obj, dict):
        return {str(k): _jsonable(v) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_jsonable(v) for v in obj]
    if isinstance(obj, np.ndarray):
        return obj.tolist()
    if isinstance(obj, (np.floating, np.integer)):
        return obj.item()
    if isinstance(obj, Path):
        return str(obj)
    return obj


def environment_record() -> dict:
    """Where the run ran: host, Python, NumPy, the CUDA device."""
    record = {"python": platform.python_version(), "numpy": np.__version__, "machine": platform.machine()}
    try:
        import torch
        if torch.cuda.is_available():
            record["device"] = torch.cuda.get_device_name(0)
            record["cuda"] = torch.version.cuda
    except Exception:  # provenance never breaks a run
        record["device"] = "unavailable"
    return record


def write_result(result, directory=None, extra: dict | None = None) -> Path:
    case = result.case
    directory = Path(directory) if directory is not None else Path(case.output) / case.name
    directory.mkdir(parents=True, exist_ok=True)
    name = case.name
    configs = {"flow": case.flow, "numerics": case.numerics, "implicit": case.implicit}
    payload = {
        "config": {k: _jsonable(dataclasses.asdict(v)) for k, v in configs.items()},
        "environment": environment_record(),
        "extra": _jsonable({
            "case_setup": case.raw, "cells": result.cells,
            "cl": result.forces.cl, "cd": result.forces.cd, "cd_friction": result.forces.cd_friction,
            "cm": result.forces.cm, "exit_reason": result.history.reason,
            "orders_dropped": result.history.orders_dropped, "iterations": result.history.n_iters,
            "seconds": result.seconds, "cl_spread": result.cl_spread, "timing": result.timing.record(),
            **(extra or {}),
        }),
    }
    (directory / f"{name}_metadata.json").write_text(json.dumps(payload, indent=2, sort_keys=True, default=str))
    residual = np.asarray(result.history.residual)
    np.savetxt(directory / f"{name}_residual.dat", np.column_stack([np.arange(1, residual.size + 1), residual]),
               header="iteration residual_l2", fmt=["%d", "%.12e"])
    cl = np.asarray(result.cl_history)
    np.savetxt(directory / f"{name}_lift.dat", np.column_stack([case.block_iters * np.arange(1, cl.size + 1), cl]),
               header="iteration cl", fmt=["%d", "%.12e"])
    if result.wall is not None:
        surface = result.surface()
        names = {"x": "x_over_c", "y": "y_over_c", "z": "z_over_c", "x_streamwise": "x_streamwise_over_c"}
        np.savetxt(directory / f"{name}_surface.dat", np.column_stack([np.asarray(v) for v in surface.values()]),
                   header=" ".join(names.get(k, k) for k in surface), fmt="%.12e")
    blocks = result.grid.unpack(np.asarray(result.U))
    arrays = {"n_blocks": np.asarray(len(blocks))}
    for k, (U, b) in enumerate(zip(blocks, result.grid.mesh)):
        arrays[f"U_{k}"] = U
        for axis, c in zip("xyz", _nodes(b)):
            arrays[f"{axis}_node_{k}"] = c
    np.savez_compressed(directory / f"{name}_fields.npz", **arrays)
    if getattr(result.grid, "dim", 2) == 3:
        for k, (U, b) in enumerate(zip(blocks, result.grid.mesh)):
            write_vts(directory / f"{name}_block{k}.vts", b.nodes, cell_fields3(U, case.flow.gamma))
    return directory


def _nodes(block):
    return block.nodes if hasattr(block, "nodes") else (block.x, block.y)


def cell_fields3(U: np.ndarray, gamma: float) -> dict:
    """Density, velocity, pressure and Mach number of a 3D block's cells
    (``src/jaxrans/simulation.py:172-177``)."""
    rho = U[0]
    velocity = U[1:4] / rho
    p = (gamma - 1.0) * (U[4] - 0.5 * rho * np.sum(velocity * velocity, axis=0))
    mach = np.sqrt(np.sum(velocity * velocity, axis=0)) / np.sqrt(gamma * p / rho)
    return {"density": rho, "velocity": velocity, "pressure": p, "mach": mach}


def write_vts(path: Path, nodes: np.ndarray, cells: dict) -> Path:
    """One 3D block for ParaView (``src/jaxrans/io/output.py:136-185``): a VTK XML
    structured grid, little-endian raw appended data with 64-bit length headers; the
    nodes ``(3, ni+1, nj+1, nk+1)`` as points, every array of ``cells`` (scalars of the
    cell shape, or 3-vectors ``(3, ...)``) as cell data; VTK's order runs ``i`` fastest."""
    ni, nj, nk = (n - 1 for n in nodes.shape[1:])
    extent = f"0 {ni} 0 {nj} 0 {nk}"
    blobs, tags, offset = [], [], 0

    def add(label: str, values: np.ndarray, components: int, group: list):
        nonlocal offset
        if components == 1:
            data = np.asarray(values, dtype="<f8").ravel(order="F")
        else:
            data = np.stack([np.asarray(c, dtype="<f8").ravel(order="F") for c in values], axis=1).ravel()
        raw = data.tobytes()
        blobs.append(np.array([len(raw)], dtype="<u8").tobytes() + raw)
        group.append(f'<DataArray type="Float64" Name="{label}" NumberOfComponents="{components}" '
                     f'format="appended" offset="{offset}"/>')
        offset += 8 + len(raw)

    points: list = []
    cell_tags: list = []
    add("Points", nodes, 3, points)
    for label, values in cells.items():
        values = np.asarray(values)
        add(label, values, 3 if values.ndim == 4 else 1, cell_tags)
    head = (f'<?xml version="1.0"?>\n<VTKFile type="StructuredGrid" version="1.0" byte_order="LittleEndian" '
            f'header_type="UInt64"><StructuredGrid WholeExtent="{extent}"><Piece Extent="{extent}">'
            f'<Points>{"".join(points)}</Points><CellData>{"".join(cell_tags)}</CellData>'
            f'</Piece></StructuredGrid><AppendedData encoding="raw">_')
    path = Path(path)
    with open(path, "wb") as out:
        out.write(head.encode())
        for blob in blobs:
            out.write(blob)
        out.write(b"</AppendedData></VTKFile>\n")
    return path
