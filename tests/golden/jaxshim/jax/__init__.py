"""A NumPy-backed stand-in for the parts of ``jax`` the reference solver uses.

Test infrastructure only: JAX is not installed in the build container, and this
module lets the reference's own Python sources run unmodified (FP64, eagerly)
so that golden vectors can be produced from them.  It is put on ``sys.path``
ahead of everything else by ``tests/golden/make_golden.py`` and by nothing else.

Derivatives (``jvp``/``linearize``) use the complex-step method: the function is
evaluated at ``x + i h t`` with ``h = 1e-100`` and the tangent is the imaginary
part over ``h``.  Every non-analytic primitive the reference differentiates
through is given JAX's own JVP rule on complex input:

* ``abs``: ``select(x >= 0, +t, -t)`` (so the slope at 0 is +1);
* ``maximum`` / ``minimum``: the selected operand's tangent, and the mean of
  both tangents at an exact tie (JAX's "balanced" rule);
* comparisons compare real parts, so ``where`` selects as JAX does;
* ``sign``: zero tangent.

``jit`` is the identity, loops are Python loops, ``vmap`` is a loop.
"""

from __future__ import annotations

import numpy as _np

from . import numpy  # noqa: F401  (jax.numpy)
from . import lax, tree_util, ops, config as _config_module  # noqa: F401
from .numpy import ShimArray as Array, asarray as _asarray
from . import scipy  # noqa: F401

config = _config_module.config
__version__ = "0.0-numpy-shim"

STEP = 1e-100


def jit(fun=None, **_kwargs):
    if fun is None:
        return lambda f: f
    return fun


def block_until_ready(x):
    return x


def device_get(x):
    return x


def device_put(x, *_args, **_kwargs):
    return x


class _Device:
    device_kind = "cpu (numpy shim)"
    platform = "cpu"


def devices(*_args):
    return [_Device()]


def default_backend():
    return "cpu"


def _complex_step(fun, primals, tangents):
    args = [(_asarray(p).astype(_np.complex128) + 1j * STEP * _asarray(t)).view(Array)
            for p, t in zip(primals, tangents)]
    out = fun(*args)
    return tree_util.tree_map(lambda y: _np.real(y).view(Array) if isinstance(y, _np.ndarray) else _np.real(y),
                              out), \
        tree_util.tree_map(lambda y: (_np.imag(y) / STEP).view(Array) if isinstance(y, _np.ndarray)
                           else _np.imag(y) / STEP, out)


def jvp(fun, primals, tangents):
    value, tangent = _complex_step(fun, primals, tangents)
    return value, tangent


def linearize(fun, *primals):
    value = fun(*primals)

    def linear(*tangents):
        return _complex_step(fun, primals, tangents)[1]

    return value, linear


def vmap(fun, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = next(_np.shape(a)[ax] for a, ax in zip(args, axes) if ax is not None)
        outs = []
        for k in range(n):
            picked = [a if ax is None else _np.take(a, k, axis=ax).view(Array) for a, ax in zip(args, axes)]
            outs.append(fun(*picked))
        return tree_util.tree_map(lambda *xs: _np.stack(xs, axis=out_axes).view(Array), *outs)

    return mapped
