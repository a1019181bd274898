"""CPU oracle for the JAX-RANS Newton-Krylov hot path (TEST INFRASTRUCTURE).

A NumPy FP64 restatement of the reference's algorithm
(giovannicatalani/jax-rans, ``src/jaxrans``), function by function, each citing
the file:line it follows.  It is the checker the device path is compared with:
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import it.  The library never calls it and has no CPU fallback.

Parity of the oracle itself is pinned against golden vectors made by running the
reference's own sources (``tests/golden/make_golden.py``): residuals, exact
first-order JVPs, wave speeds, chain blocks, preconditioner solves, GMRES,
Newton steps, forces and converged runs.

Derivatives use the complex-step method (``jvp``): every function here accepts
complex input, compares real parts, and gives ``abs``, ``min`` and ``max`` the
JVP rules of JAX (``abs'(0) = +1``; the mean of both tangents at a tie).
"""

from .numerics import (  # noqa: F401
    Model, prim, fill_ghosts, residual, jvp, wave_speeds, cell_sum, norm, initial_state,
)
from .implicit import (  # noqa: F401
    chain_blocks_flow, chain_blocks_sa, cr_factor, cr_solve, thomas_factor, thomas_solve,
    precondition, gmres_right, hessenberg_lstsq, newton_step, NewtonState, relax,
)
from .forces import forces, wall_loads  # noqa: F401
