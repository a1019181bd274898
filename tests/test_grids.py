"""The grid generator against the reference's own generated grids (the golden blocks):
node coordinates within 1e-12 chord (the marching solves each layer with a sparse
direct solver, whose round-off differs from the reference's solver)."""

from __future__ import annotations

import numpy as np
import pytest

from goldens import CASES, load


@pytest.mark.parametrize("name", CASES)
def test_generated_grid_matches_reference(name):
    z, case, plan = load(name)
    block = case.grid_spec.build(case.directory)[0]
    assert block.x.shape == z["block0_x"].shape
    assert np.abs(block.x - z["block0_x"]).max() < 1e-12
    assert np.abs(block.y - z["block0_y"]).max() < 1e-12
