"""The coupled (5x5) line preconditioner of the oracle against a dense solve of the same
block-tridiagonal chains (CPU).  The coupled form is the 5x5 variant of line_j:
the SA row gains its coupling to the mean flow; the reference has only the split form."""

from __future__ import annotations

import numpy as np

from goldens import load, oracle_model
from oracle import implicit as im
from oracle import numerics as nm


def test_coupled_preconditioner_is_the_dense_block_solve():
    z, case, plan = load("c_sa")
    model = oracle_model(case, plan)
    U = z["rand0_U"]
    lam = nm.wave_speeds(U, model)
    cfl = 25.0
    r = z["rand0_prec_r"]
    out = im.precondition_coupled(U, lam, cfl, model)(r)
    lf, df, uf = im.chain_blocks_flow(U, lam, cfl, model)
    ls, ds, us = im.chain_blocks_sa(U, lam, cfl, model)
    lc, uc = im.chain_coupling_sa(U, model)
    ch = plan.chains
    L = ch.cells.shape[1]
    checked = 0
    for c in range(ch.cells.shape[0]):
        n = int(ch.lengths[c])
        A = np.zeros((5 * n, 5 * n))
        for k in range(n):
            blk = lambda f, s, cpl: np.block([[f, np.zeros((4, 1))], [cpl[None, :], s]])  # noqa: E731
            A[5 * k:5 * k + 5, 5 * k:5 * k + 5] = blk(df[k, c], ds[k, c], np.zeros(4))
            if k > 0:
                A[5 * k:5 * k + 5, 5 * (k - 1):5 * k] = blk(lf[k, c], ls[k, c], lc[k, c])
            if k < n - 1:
                A[5 * k:5 * k + 5, 5 * (k + 1):5 * k + 10] = blk(uf[k, c], us[k, c], uc[k, c])
        cells = ch.cells[c, :n]
        rhs = np.concatenate([r.reshape(5, -1)[:, cell] for cell in cells])
        x = np.linalg.solve(A, rhs)
        got = np.concatenate([out.reshape(5, -1)[:, cell] for cell in cells])
        assert np.abs(got - x).max() <= 1e-10 * max(np.abs(x).max(), 1e-300)
        checked += 1
    assert checked == ch.cells.shape[0] and L >= 1


def test_coupling_changes_only_the_sa_row():
    z, case, plan = load("c_sa")
    model = oracle_model(case, plan)
    U = z["rand0_U"]
    lam = nm.wave_speeds(U, model)
    r = z["rand0_prec_r"]
    split = im.precondition(U, lam, 25.0, model)(r)
    coupled = im.precondition_coupled(U, lam, 25.0, model)(r)
    assert np.array_equal(split[:4], coupled[:4])
    assert np.abs(split[4] - coupled[4]).max() > 0.0
