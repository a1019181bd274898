"""The hot path as jax.ffi custom calls, for JAX programs (the reference's own driver).

``register()`` builds the handlers (``csrc/ffi/jr_ffi.cc``, against JAX's FFI headers)
and registers three CUDA targets:

* ``jaxrans_b200_residual`` -- ``make_residual(...).residual`` (src/jaxrans/numerics/
  residual.py:273-334): R(U) on the plan's canvas(es);
* ``jaxrans_b200_jvp`` -- the jvp of ``jax.linearize(jacobian_source.residual, U)``
  (src/jaxrans/solvers/implicit.py:104-116): the exact J.v of the first-order residual;
* ``jaxrans_b200_newton_block`` -- the driver's block of Newton steps
  (src/jaxrans/solvers/driver.py:87-105) on the plan's solver state.

The plan is a ``native.DevicePlan`` made by the caller and kept alive while the calls
may run; its handle travels as an int64 attribute.  XLA owns the buffers and the stream.
JAX is not installed where this package is built and tested, so these functions are
untested; without JAX ``register()`` raises ``ImportError``.
"""

from __future__ import annotations

import ctypes

_TARGETS = {"jaxrans_b200_residual": "JrResidual", "jaxrans_b200_jvp": "JrJvp",
            "jaxrans_b200_newton_block": "JrNewtonBlock"}
_registered = False


def register() -> None:
    """Build (if needed) and register the three targets with jax.ffi, once."""
    global _registered
    if _registered:
        return
    from .build import build_ffi
    path = build_ffi()
    if path is None:
        raise ImportError("jax.ffi is not available: install JAX to use the custom calls")
    import jax
    lib = ctypes.CDLL(str(path))
    for target, symbol in _TARGETS.items():
        jax.ffi.register_ffi_target(target, jax.ffi.pycapsule(getattr(lib, symbol)), platform="CUDA")
    _registered = True


def _handle(plan) -> "numpy.int64":
    import numpy as np
    return np.int64(plan.handle.value if hasattr(plan.handle, "value") else plan.handle)


def residual(U, plan, first_order: bool = False):
    """R(U) as a custom call: U holds nvar x every case's canvas (float64, on the GPU)."""
    import jax
    import numpy as np
    register()
    return jax.ffi.ffi_call("jaxrans_b200_residual", jax.ShapeDtypeStruct(U.shape, U.dtype))(
        U, plan=_handle(plan), first_order=np.int32(first_order))


def jvp(U, v, plan):
    """dR1/dU . v at U as a custom call."""
    import jax
    register()
    return jax.ffi.ffi_call("jaxrans_b200_jvp", jax.ShapeDtypeStruct(U.shape, U.dtype))(U, v, plan=_handle(plan))


def newton_block(U, plan, n_steps: int, cfl: float, restart: bool = False):
    """n_steps Newton steps from U on the plan's solver state: (U after, |R| history of
    shape (n_steps, cases)).  ``restart`` starts every case at CFL ``cfl``; otherwise the
    plan's CFL ramp carries on from its last block."""
    import jax
    import numpy as np
    register()
    out = (jax.ShapeDtypeStruct(U.shape, U.dtype), jax.ShapeDtypeStruct((n_steps, plan.n_cases), U.dtype))
    return jax.ffi.ffi_call("jaxrans_b200_newton_block", out)(
        U, plan=_handle(plan), n_steps=np.int32(n_steps), restart=np.int32(restart), cfl=np.float64(cfl))
