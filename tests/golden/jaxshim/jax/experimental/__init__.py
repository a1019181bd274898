"""``jax.experimental`` placeholder (test infrastructure)."""
