"""Loading the golden fixtures (made by ``tests/golden/make_golden.py`` from the
reference itself) into this build's plan and configs, and the oracle's model."""

from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

from jaxrans_b200 import plan as P
from jaxrans_b200.case import parse_case
from jaxrans_b200.config import freestream_primitive
from oracle import numerics as nm

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("o_euler", "c_sa", "c_laminar", "o_sa_qcr")


@lru_cache(maxsize=None)
def load(name: str):
    z = dict(np.load(GOLDEN / f"{name}.npz"))
    doc = json.loads(str(z["case_json"]))
    case = parse_case(doc["case"], doc["numerical"])
    blocks = [P.block_from_record(z[f"block{b}_x"], z[f"block{b}_y"], json.loads(str(z[f"block{b}_sides"])))
              for b in range(int(z["n_blocks"]))]
    plan = P.build_plan(blocks, with_distance=case.flow.turbulence is not None)
    return z, case, plan


def oracle_model(case, plan) -> nm.Model:
    flow, num = case.flow, case.numerics
    return nm.Model(plan, np.array(freestream_primitive(flow)), flow.gamma, num.flux, num.limiter, num.kappa,
                    None if flow.inviscid else flow.mu_inf, flow.sutherland_ratio, flow.turbulence is not None,
                    0.3 if flow.turbulence == "sa_noft2_qcr" else 0.0, num.far_field, plan.distance)


def converged(name: str):
    path = GOLDEN / f"{name}_converged.npz"
    return dict(np.load(path)) if path.is_file() else None


def rel(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
