"""``jax.scipy`` placeholder (test infrastructure)."""
from . import sparse  # noqa: F401
