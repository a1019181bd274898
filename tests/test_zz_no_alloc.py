"""jr_residual_noalloc against jr_residual, through the C ABI.

jr_residual_noalloc is the residual for callers that cannot allocate device memory at
call time (a handler inside another framework's step, whose allocator owns the device):
its scratch is a static device array in the library, shared by every call and keeping
the last call's contents.  So each check makes calls in a row -- two states, both orders
-- and compares every one with jr_residual at the residual tolerance of the parity tests
(1e-12 relative to each row's largest entry).  The file is collected last, so it also
runs after every other test has used the library.
"""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from goldens import load

pytestmark = pytest.mark.gpu


def row_rel(a, b):
    return max(float(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300)) for v in range(b.shape[0]))


def residual_pair(dev, U, first):
    import torch
    lib = dev.lib
    ref = torch.empty_like(U)
    out = torch.full_like(U, float("nan"))
    torch.cuda.synchronize()
    assert lib.jr_residual(dev.handle, U.data_ptr(), ref.data_ptr(), int(first)) == 0, lib.jr_last_error()
    assert lib.jr_residual_noalloc(dev.handle, U.data_ptr(), out.data_ptr(), int(first)) == 0, lib.jr_last_error()
    assert lib.jr_synchronize(dev.handle) == 0
    return out.cpu().numpy(), ref.cpu().numpy()


@pytest.mark.parametrize("name", ["c_sa", "o_euler"])
def test_noalloc_residual_equals_jr_residual(cuda, name):
    import torch
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load(name)
    dev = DevicePlan(plan, case.flow, case.numerics, case.implicit)
    for state in ("sin", "rand0"):
        U = torch.as_tensor(z[f"{state}_U"], device="cuda").contiguous()
        for first in (False, True):
            out, ref = residual_pair(dev, U, first)
            assert row_rel(out, ref) < 1e-12
            assert row_rel(out, z[f"{state}_R1" if first else f"{state}_R2"]) < 1e-12


def test_noalloc_residual_of_a_batch(cuda):
    import torch
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("c_sa")
    flows = [replace(case.flow, alpha_deg=a) for a in (-1.0, 2.5)]
    dev = DevicePlan.batch(plan, flows, case.numerics, case.implicit)
    U = torch.as_tensor(np.concatenate([z["rand0_U"].ravel(), z["sin_U"].ravel()]), device="cuda")
    for first in (False, True):
        out, ref = residual_pair(dev, U, first)
        assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()


def test_noalloc_refuses_a_plan_beyond_its_scratch(cuda):
    """Six cases of the 385 x 97 C-grid need about 9.3 MB of canvas: more than 8 MiB."""
    import torch
    from jaxrans_b200.native import DevicePlan
    from jaxrans_b200.workloads import workload
    case = workload("c_sa_385")
    plan = case.grid()
    dev = DevicePlan.batch(plan, [case.flow] * 6, case.numerics, case.implicit)
    U = torch.zeros(dev.n_vec, dtype=torch.float64, device="cuda")
    R = torch.full_like(U, 7.0)
    torch.cuda.synchronize()
    assert dev.lib.jr_residual_noalloc(dev.handle, U.data_ptr(), R.data_ptr(), 0) == 1
    assert b"8 MiB" in dev.lib.jr_last_error()
    assert bool((R == 7.0).all())


def test_noalloc_residual_after_newton_steps(cuda):
    """After Newton steps the plan's own ghost canvas holds that march's values, not zeros;
    the two entry points still agree on the plan's current state."""
    import torch
    from jaxrans_b200.native import DevicePlan
    z, case, plan = load("c_sa")
    dev = DevicePlan(plan, case.flow, case.numerics, case.implicit)
    dev.set_state(z["rand0_U"], 25.0, float("inf"))
    dev.newton_steps(3)
    U_host = dev.get_state()[0]
    U = torch.as_tensor(U_host, device="cuda").contiguous()
    for first in (False, True, False):
        out, ref = residual_pair(dev, U, first)
        assert row_rel(out, ref) < 1e-12
