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
        names = {"x": "x_over_c", "y": "y_over_c"}
        np.savetxt(directory / f"{name}_surface.dat", np.column_stack([np.asarray(v) for v in surface.values()]),
                   header=" ".join(names.get(k, k) for k in surface), fmt="%.12e")
    blocks = result.grid.unpack(np.asarray(result.U))
    arrays = {"n_blocks": np.asarray(len(blocks))}
    for k, (U, b) in enumerate(zip(blocks, result.grid.mesh)):
        arrays[f"U_{k}"] = U
        arrays[f"x_node_{k}"] = b.x
        arrays[f"y_node_{k}"] = b.y
    np.savez_compressed(directory / f"{name}_fields.npz", **arrays)
    return directory
