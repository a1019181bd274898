"""``jax.lax`` loops as Python loops (test infrastructure, see ``jax/__init__.py``)."""

from __future__ import annotations

import numpy as np

from . import tree_util
from .numpy import ShimArray, _wrap


def scan(f, init, xs=None, length=None, reverse=False, unroll=1):
    if xs is None:
        n = length
        items = [None] * n
    else:
        leaves = tree_util.tree_leaves(xs)
        n = np.shape(leaves[0])[0]
        items = [tree_util.tree_map(lambda a: _wrap(a[k]), xs) for k in range(n)]
    order = range(n - 1, -1, -1) if reverse else range(n)
    carry, ys = init, [None] * n
    for k in order:
        carry, y = f(carry, items[k])
        ys[k] = y
    if n == 0 or ys[0] is None:
        return carry, None
    return carry, tree_util.tree_map(lambda *v: np.stack([np.asarray(a) for a in v]).view(ShimArray), *ys)


def fori_loop(lower, upper, body, init):
    carry = init
    for k in range(int(lower), int(upper)):
        carry = body(k, carry)
    return carry


def while_loop(cond, body, init):
    carry = init
    while bool(cond(carry)):
        carry = body(carry)
    return carry


def cond(pred, true_fun, false_fun, *operands):
    return true_fun(*operands) if bool(pred) else false_fun(*operands)


def select(pred, a, b):
    return _wrap(np.where(pred, a, b))


def stop_gradient(x):
    return _wrap(np.real(x)) if np.iscomplexobj(x) else x


def map(f, xs):  # noqa: A001
    return tree_util.tree_map(lambda *v: np.stack(v).view(ShimArray), *[f(x) for x in xs])


def top_k(x, k):
    x = np.asarray(x)
    idx = np.argsort(-x, axis=-1)[..., :k]
    return _wrap(np.take_along_axis(x, idx, -1)), _wrap(idx)


def ppermute(x, *args, **kwargs):
    raise NotImplementedError("ppermute: slabs are outside the numpy stand-in")


def axis_index(*args, **kwargs):
    return 0
