"""Loading the golden fixtures (made by ``tests/golden/make_golden.py`` from the
reference itself) into jaxrans_b200's plan and configs, and the oracle's model."""

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


# The benchmark workloads' own grids (tests/golden/make_golden_configs.py): the 2D Euler
# O-grid of 257 x 65 nodes, the SA C-grid of 385 x 97 and the uneven SA C-grid of 513 x 129
CONFIGS = ("o_euler_257", "c_sa_385", "c_sa_513")
CONFIG_SEEDS = {("sin", "v"): 11, ("sin", "r"): 12, ("rand0", "v"): 13, ("rand0", "r"): 14}


def config_state(z, plan, state: str) -> np.ndarray:
    """The state a config golden was made on, drawn again: U0 (1 + 1e-3 sin(k)), or
    U0 (1 + 1e-2 u) with u uniform from np.random.default_rng(0)."""
    U0 = np.broadcast_to(z["U_inf"].reshape((-1,) + (1,) * len(plan.shape)), (z["U_inf"].size,) + plan.shape)
    U0 = np.array(U0)
    if state == "sin":
        return U0 * (1.0 + 1e-3 * np.sin(np.arange(U0.size).reshape(U0.shape)))
    return U0 * (1.0 + 1e-2 * np.random.default_rng(0).uniform(-1.0, 1.0, U0.shape))


def config_vector(plan, state: str, what: str, nvar: int) -> np.ndarray:
    """The J.v direction ("v") or the preconditioner's right-hand side ("r") of a config
    golden: standard normals from a fixed seed, zero off the interior."""
    shape = (nvar,) + plan.shape
    return np.where(plan.interior, np.random.default_rng(CONFIG_SEEDS[(state, what)]).standard_normal(shape), 0.0)
