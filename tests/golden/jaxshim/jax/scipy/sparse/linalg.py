def gmres(*args, **kwargs):
    raise NotImplementedError("jax.scipy.sparse.linalg.gmres is outside the numpy stand-in")
