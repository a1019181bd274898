"""The oracle pinned against the reference's own outputs (the golden fixtures)."""

from __future__ import annotations

import numpy as np
import pytest

from goldens import CASES, load, oracle_model, rel
from jaxrans_b200 import plan as P
from oracle import implicit as im
from oracle import numerics as nm
import oracle


@pytest.mark.parametrize("name", CASES)
def test_plan_matches_reference_atlas(name):
    z, case, plan = load(name)
    assert np.array_equal(plan.interior, z["interior"])
    for mine, key in ((plan.volume, "volume"), (plan.faces_i, "faces_i"), (plan.faces_j, "faces_j"),
                      (plan.centres, "centres")):
        assert np.array_equal(mine, z[key]), key
    assert np.array_equal(plan.neighbours, z["neighbours"])
    for s, st in enumerate(plan.stages):
        index = np.arange(plan.n_canvas)
        copy = st.kind == 0
        index[st.ghost[copy]] = st.source[copy]
        off = plan.n_canvas
        for kind in st.order:
            m = st.kind == P.KIND_CODES[kind]
            index[st.ghost[m]] = off + np.arange(m.sum())
            off += m.sum()
        assert np.array_equal(index, z[f"stage{s}_index"])
    for key in ("cells", "up_face", "up_sign", "down_face", "down_sign"):
        assert np.array_equal(getattr(plan.chains, key), z[f"lines_{key}"]), key
    W = plan.walls
    for key in ("cell", "family", "face", "into_fluid", "body", "a", "b"):
        assert np.array_equal(getattr(W, key), z[f"walls_{key}"]), key
    assert tuple(plan.quarter_chord) == tuple(z["quarter_chord"])
    if "distance" in z:
        assert np.array_equal(plan.distance, z["distance"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("state", ["sin", "rand0"])
def test_oracle_matches_reference(name, state):
    z, case, plan = load(name)
    m = oracle_model(case, plan)
    U = z[f"{state}_U"]
    assert rel(nm.residual(U, m), z[f"{state}_R2"]) < 1e-14
    assert rel(nm.residual(U, m, True), z[f"{state}_R1"]) < 1e-14
    assert rel(nm.jvp(U, z[f"{state}_v"], m), z[f"{state}_Jv"]) < 1e-14
    lam = nm.wave_speeds(U, m)
    assert rel(lam[0], z[f"{state}_lam_i"]) < 1e-15 and rel(lam[1], z[f"{state}_lam_j"]) < 1e-15
    lo, di, up = im.chain_blocks_flow(U, lam, 25.0, m)
    for mine, key in ((lo, "lower"), (di, "diag"), (up, "upper")):
        assert rel(mine, z[f"{state}_flow_{key}"]) < 1e-15
    if m.sa:
        lo, di, up = im.chain_blocks_sa(U, lam, 25.0, m)
        for mine, key in ((lo, "lower"), (di, "diag"), (up, "upper")):
            assert rel(mine, z[f"{state}_sa_{key}"]) < 1e-15
    assert rel(im.precondition(U, lam, 25.0, m)(z[f"{state}_prec_r"]), z[f"{state}_prec_z"]) < 1e-14
    assert rel(im.precondition(U, lam, 25.0, m, "thomas")(z[f"{state}_prec_r"]), z[f"{state}_prec_z"]) < 1e-12
    assert np.abs(oracle.forces(U, m) - z[f"{state}_forces"]).max() < 1e-15


@pytest.mark.parametrize("name", CASES)
def test_oracle_gmres_and_newton_match_reference(name):
    z, case, plan = load(name)
    m = oracle_model(case, plan)
    cfg = case.implicit
    U = z["rand0_U"]
    R = nm.residual(U, m)
    lam = nm.wave_speeds(U, m)
    vdt = nm.cell_sum(lam) / 25.0
    dU, act = im.gmres_right(lambda d: vdt[None] * d + nm.jvp(U, d, m), -R, im.precondition(U, lam, 25.0, m),
                             cfg.krylov_subspace, cfg.krylov_restarts, cfg.krylov_tol)
    assert rel(dU, z["gmres_dU"]) < 1e-12
    st = im.NewtonState(U, 25.0, np.inf)
    for k in range(3):
        st, n = im.newton_step(st, m, cfg)
        assert abs(n - float(z[f"newton{k}_norm"])) <= 1e-12 * float(z[f"newton{k}_norm"])
        assert st.cfl == pytest.approx(float(z[f"newton{k}_cfl"]), rel=1e-14)
    assert rel(st.U, z["newton2_U"]) < 1e-11
