"""The 3D kernels' per-cell and per-record bodies (csrc/residual3d.cuh) run on the host
by a test-only harness (tests/host3d/harness.cu, built here with nvcc for the host), in
the order the device runs them: the kernels' indexing and arithmetic checked against the
3D oracle and the reference's outputs on the wing fixture, without a GPU."""

from __future__ import annotations

import ctypes as C
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from jaxrans_b200.case import _flow
from jaxrans_b200.geometry import section_source
from jaxrans_b200.grid3d import wing_block
from jaxrans_b200.native3d import describe
from jaxrans_b200.plan3d import build_plan3d

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden" / "ch_sa3d.npz"
KINDS = {"wall": "no_slip_wall", "farfield": "far_field", "root": "symmetry", "tip": "symmetry"}


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc is not available")
    out = tmp_path_factory.mktemp("host3d") / "libjr3host.so"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Xcompiler", "-fPIC", "-shared",
                    "-gencode", "arch=compute_100a,code=compute_100a", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests" / "host3d" / "harness.cu"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    lib.jr3_host_eval.restype = C.c_int
    lib.jr3_host_eval.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    return lib


@pytest.fixture(scope="module")
def case3d():
    z = np.load(GOLDEN)
    w = json.loads(str(z["wing_json"]))
    doc = json.loads(str(z["case_json"]))
    plan = build_plan3d([wing_block(section_source(w.pop("section")), **w).with_kinds(KINDS)])
    flow = _flow(doc["case"])
    a = flow.alpha_rad
    q_inf = np.array([1.0, flow.mach * np.cos(a), 0.0, flow.mach * np.sin(a), 1.0 / flow.gamma,
                      flow.nu_tilde_ratio])
    cv = doc["numerical"]["convective_fluxes"]
    desc, keep = describe(plan, q_inf, flow.gamma, cv["riemann_solver"], cv["limiter"], 0.0, flow.mu_inf,
                          flow.sutherland_ratio)
    return z, plan, desc, keep


def evaluate(lib, desc, U, v=None, first_order=False):
    U = np.ascontiguousarray(U, dtype=np.float64)
    R = np.zeros_like(U)
    dU = None if v is None else np.ascontiguousarray(v, dtype=np.float64)
    rc = lib.jr3_host_eval(C.addressof(desc), U.ctypes.data, None if dU is None else dU.ctypes.data,
                           R.ctypes.data, int(first_order))
    assert rc == 0
    return R


def rows_rel(a, b):
    return max(float(np.abs(a[k] - b[k]).max() / max(np.abs(b[k]).max(), 1e-300)) for k in range(a.shape[0]))


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_residual(harness, case3d, state):
    z, plan, desc, _ = case3d
    U = z[f"{state}_U"]
    assert rows_rel(evaluate(harness, desc, U), z[f"{state}_R2"]) < 1e-12
    assert rows_rel(evaluate(harness, desc, U, first_order=True), z[f"{state}_R1"]) < 1e-12


@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_kernel_bodies_give_the_reference_jvp(harness, case3d, state):
    z, plan, desc, _ = case3d
    Jv, ref = evaluate(harness, desc, z[f"{state}_U"], z[f"{state}_v"]), z[f"{state}_Jv"]
    assert rows_rel(Jv[:5], ref[:5]) < 1e-12
    assert rows_rel(Jv[5:], ref[5:]) < 1e-10
