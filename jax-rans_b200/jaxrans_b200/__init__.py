"""jaxrans_b200: the pseudo-transient Newton-Krylov hot path of JAX-RANS on one B200.

The reference's call surface (``src/jaxrans/__init__.py:22-26``) over hand-written
sm_100a kernels reached through a C ABI (``include/jaxrans_b200.h``):

    from jaxrans_b200 import load_case, run
    result = run(load_case("my_case"))     # case.json + numerical.json
    print(result.forces.summary())

``make_residual(...).residual(U)`` gives the residual of one state on the device.
There is no CPU fallback: without the built library and a CUDA device the calls raise.
"""

from .case import Case, CaseError, load_case, parse_case  # noqa: F401
from .config import FlowConditions, ImplicitConfig, NumericsConfig  # noqa: F401
from .residual import ResidualOperator, make_residual  # noqa: F401
from .solver import ConvergenceHistory, ExitReason, Forces, Result, run  # noqa: F401

__all__ = ["Case", "CaseError", "ConvergenceHistory", "ExitReason", "FlowConditions", "Forces", "ImplicitConfig",
           "NumericsConfig", "ResidualOperator", "Result", "load_case", "make_residual", "parse_case", "run"]
__version__ = "0.1.0"
