"""Result files in the reference's layout, written from a result held in memory (no GPU)."""

from __future__ import annotations

import json

import numpy as np

from goldens import load
from jaxrans_b200.solver import ConvergenceHistory, Forces, Result, Timing, freestream_state


def test_result_files(tmp_path):
    z, case, plan = load("c_laminar")
    n = len(plan.walls.cell)
    wall = np.zeros((n, 5))
    wall[:, 0] = np.linspace(-0.1, 0.1, n)
    S = np.array([[0.0, 1.0]] * n)
    wall[:, 1:3] = S * 0.01
    wall[:, 3] = 1e-6
    result = Result(case=case, grid=plan, U=freestream_state(case, plan), forces=Forces(0.5, 0.02, -0.1, 0, 0, 0.01),
                    history=ConvergenceHistory(np.array([1.0, 0.1, 0.01]), "converged", 3),
                    cl_history=np.array([0.4, 0.5]), timing=Timing(1.0, 0.5, 40, 20, plan.cells), wall=wall)
    out = result.write(tmp_path / "run")
    names = sorted(p.name for p in out.iterdir())
    assert names == sorted(f"{case.name}_{s}" for s in ("metadata.json", "residual.dat", "lift.dat",
                                                         "surface.dat", "fields.npz"))
    meta = json.loads((out / f"{case.name}_metadata.json").read_text())
    assert meta["extra"]["exit_reason"] == "converged" and meta["extra"]["cl"] == 0.5
    res = np.loadtxt(out / f"{case.name}_residual.dat")
    assert res.shape == (3, 2) and res[-1, 1] == 0.01
    lift = np.loadtxt(out / f"{case.name}_lift.dat")
    assert np.array_equal(lift[:, 0], [20, 40])
    surf = np.loadtxt(out / f"{case.name}_surface.dat")
    q = 0.5 * case.flow.mach ** 2
    assert surf.shape == (n, 5)                      # x, y, body, cp, cf (viscous)
    assert np.allclose(surf[:, 3], wall[:, 0] / q)
    fields = np.load(out / f"{case.name}_fields.npz")
    assert int(fields["n_blocks"]) == len(plan.mesh)
    assert fields["U_0"].shape[0] == case.flow.nvar
