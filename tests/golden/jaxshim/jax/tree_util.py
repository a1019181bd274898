"""``jax.tree_util`` over tuples, lists, dicts, NamedTuples and registered dataclasses."""

from __future__ import annotations

import dataclasses

_DATACLASSES: dict[type, tuple[list[str], list[str]]] = {}


def register_dataclass(cls, data_fields=None, meta_fields=None):
    _DATACLASSES[cls] = (list(data_fields or []), list(meta_fields or []))
    return cls


def register_pytree_node(*_args, **_kwargs):
    return None


def _is_leaf(x):
    return not (isinstance(x, (tuple, list, dict)) or type(x) in _DATACLASSES or x is None)


def tree_leaves(tree):
    if tree is None:
        return []
    if type(tree) in _DATACLASSES:
        return [leaf for f in _DATACLASSES[type(tree)][0] for leaf in tree_leaves(getattr(tree, f))]
    if isinstance(tree, dict):
        return [leaf for k in sorted(tree) for leaf in tree_leaves(tree[k])]
    if isinstance(tree, (tuple, list)):
        return [leaf for x in tree for leaf in tree_leaves(x)]
    return [tree]


def tree_map(f, tree, *rest):
    if tree is None:
        return None
    if type(tree) in _DATACLASSES:
        data, _ = _DATACLASSES[type(tree)]
        return dataclasses.replace(tree, **{k: tree_map(f, getattr(tree, k), *(getattr(r, k) for r in rest))
                                            for k in data})
    if isinstance(tree, dict):
        return {k: tree_map(f, tree[k], *(r[k] for r in rest)) for k in tree}
    if isinstance(tree, tuple) and hasattr(tree, "_fields"):
        return type(tree)(*(tree_map(f, x, *(r[i] for r in rest)) for i, x in enumerate(tree)))
    if isinstance(tree, (tuple, list)):
        return type(tree)(tree_map(f, x, *(r[i] for r in rest)) for i, x in enumerate(tree))
    return f(tree, *rest)
