"""The oracle against the reference's own outputs on the benchmark workloads' grids
(tests/golden/make_golden_configs.py): the O-grid of 257 x 65 nodes (2D Euler, HLLC, van
Albada) and the C-grid of 385 x 97 nodes (SA, Roe, minmod).  The plans built from the
reference's blocks and sides are the reference's (volume, faces, interior); R2, R1, J.v,
the wave speeds and the line_j solve agree to round-off."""

from __future__ import annotations

import numpy as np
import pytest

from goldens import config_state, config_vector, load, oracle_model, rel
from oracle import implicit as im
from oracle import numerics as nm


@pytest.mark.parametrize("name", ["o_euler_257", "c_sa_385"])
def test_oracle_matches_reference_on_config_grids(name):
    z, case, plan = load(name)
    m = oracle_model(case, plan)
    nvar = z["U_inf"].size
    U = config_state(z, plan, "sin")
    assert np.array_equal(nm.initial_state(m), np.broadcast_to(z["U_inf"].reshape(-1, 1, 1), U.shape))
    assert rel(nm.residual(U, m), z["sin_R2"]) < 1e-13
    assert rel(nm.residual(U, m, True), z["sin_R1"]) < 1e-13
    assert rel(nm.jvp(U, config_vector(plan, "sin", "v", nvar), m), z["sin_Jv"]) < 1e-13
    lam = nm.wave_speeds(U, m)
    assert rel(lam[0], z["sin_lam_i"]) < 1e-14 and rel(lam[1], z["sin_lam_j"]) < 1e-14
    z_ref = z["sin_prec_z"]
    assert rel(im.precondition(U, lam, 25.0, m)(config_vector(plan, "sin", "r", nvar)), z_ref) < 1e-12
    U = config_state(z, plan, "rand0")
    assert rel(nm.residual(U, m), z["rand0_R2"]) < 1e-13
