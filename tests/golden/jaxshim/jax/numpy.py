"""``jax.numpy`` on NumPy, complex-step aware (see the package docstring)."""

from __future__ import annotations

import types

import numpy as np

float64 = np.float64
float32 = np.float32
int64 = np.int64
int32 = np.int32
bool_ = np.bool_
complex128 = np.complex128
pi = np.pi
inf = np.inf
nan = np.nan
ndarray = np.ndarray
newaxis = None
finfo = np.finfo
dtype = np.dtype


class _At:
    def __init__(self, array):
        self.array = array

    def __getitem__(self, index):
        return _Updater(self.array, index)


class _Updater:
    def __init__(self, array, index):
        self.array, self.index = array, index

    def _copy(self, value):
        value = np.asarray(value)
        out = np.array(self.array, dtype=np.result_type(self.array, value)).view(ShimArray)
        return out, value

    def set(self, value, **_kw):
        out, value = self._copy(value)
        out[self.index] = value
        return out

    def add(self, value, **_kw):
        out, value = self._copy(value)
        np.add.at(out, self.index, value)
        return out

    def multiply(self, value, **_kw):
        out, value = self._copy(value)
        np.multiply.at(out, self.index, value)
        return out

    def get(self, **_kw):
        return self.array[self.index]


def _re(x):
    return np.real(x) if np.iscomplexobj(x) else x


class ShimArray(np.ndarray):
    """An ndarray with ``.at[...]`` updates and real-part comparisons."""

    @property
    def at(self):
        return _At(self)

    def __gt__(self, other):
        return np.greater(_re(np.asarray(self)), _re(np.asarray(other))).view(ShimArray)

    def __ge__(self, other):
        return np.greater_equal(_re(np.asarray(self)), _re(np.asarray(other))).view(ShimArray)

    def __lt__(self, other):
        return np.less(_re(np.asarray(self)), _re(np.asarray(other))).view(ShimArray)

    def __le__(self, other):
        return np.less_equal(_re(np.asarray(self)), _re(np.asarray(other))).view(ShimArray)

    def __abs__(self):
        return abs_(self)

    def __bool__(self):
        return bool(_re(np.asarray(self)))

    def __float__(self):
        return float(_re(np.asarray(self)))

    def block_until_ready(self):
        return self


def _wrap(x):
    if isinstance(x, np.ndarray):
        return x.view(ShimArray)
    if isinstance(x, (np.generic, float, int, complex, bool)):
        return np.asarray(x).view(ShimArray)
    return x


def _wrapped(fn):
    def call(*args, **kwargs):
        return _wrap(fn(*args, **kwargs))
    call.__name__ = getattr(fn, "__name__", "fn")
    return call


def asarray(a, dtype=None, **_kw):
    if dtype is not None and np.iscomplexobj(a) and not np.issubdtype(np.dtype(dtype), np.complexfloating):
        # A cast to real would drop a complex-step tangent: keep it (JAX's
        # asarray of a traced value keeps the tangent too).
        return np.asarray(a).view(ShimArray)
    return np.asarray(a, dtype=dtype).view(ShimArray)


array = asarray


def _tangent_select(cond, a, b):
    return np.where(cond, a, b)


def abs_(x):
    x = np.asarray(x)
    if np.iscomplexobj(x):
        return _wrap(np.where(np.real(x) >= 0.0, x, -x))
    return _wrap(np.abs(x))


abs = abs_  # noqa: A001
absolute = abs_


def maximum(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if np.iscomplexobj(a) or np.iscomplexobj(b):
        ra, rb = _re(a), _re(b)
        return _wrap(np.where(ra > rb, a, np.where(rb > ra, b, 0.5 * (a + b))))
    return _wrap(np.maximum(a, b))


def minimum(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if np.iscomplexobj(a) or np.iscomplexobj(b):
        ra, rb = _re(a), _re(b)
        return _wrap(np.where(ra < rb, a, np.where(rb < ra, b, 0.5 * (a + b))))
    return _wrap(np.minimum(a, b))


def clip(x, lo=None, hi=None):
    out = x
    if lo is not None:
        out = maximum(out, lo)
    if hi is not None:
        out = minimum(out, hi)
    return out


def sign(x):
    return _wrap(np.sign(_re(np.asarray(x))))


def hypot(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if np.iscomplexobj(a) or np.iscomplexobj(b):
        return _wrap(np.sqrt(a * a + b * b))
    return _wrap(np.hypot(a, b))


def arctan2(y, x):
    return _wrap(np.arctan2(_re(np.asarray(y)), _re(np.asarray(x))))


def isfinite(x):
    return _wrap(np.isfinite(np.asarray(x)))


def where(cond, a=None, b=None):
    if a is None:
        return np.where(np.asarray(cond))
    return _wrap(np.where(_re(np.asarray(cond)), a, b))


def pad(a, widths, mode="constant", **kw):
    return _wrap(np.pad(np.asarray(a), widths, mode=mode, **kw))


def max(a, axis=None, **kw):  # noqa: A001
    return _wrap(np.max(_re(np.asarray(a)), axis=axis, **kw))


def min(a, axis=None, **kw):  # noqa: A001
    return _wrap(np.min(_re(np.asarray(a)), axis=axis, **kw))


def argmax(a, axis=None):
    return _wrap(np.argmax(_re(np.asarray(a)), axis=axis))


def astype(x, dtype):
    return _wrap(np.asarray(x).astype(dtype))


for _name in ("sqrt", "sin", "cos", "tan", "arctan", "exp", "log", "tanh", "sinh", "cosh", "square",
              "concatenate", "stack", "zeros", "ones", "zeros_like", "ones_like", "full", "full_like",
              "empty", "empty_like", "broadcast_to", "sum", "prod", "mean", "all", "any", "tensordot",
              "einsum", "swapaxes", "moveaxis", "transpose", "repeat", "tile", "eye", "arange", "linspace",
              "reshape", "ravel", "take", "cumsum", "diff", "outer", "dot", "matmul", "vdot", "roll",
              "expand_dims", "squeeze", "floor", "ceil", "round", "real", "imag", "isnan", "logical_and",
              "logical_or", "logical_not", "nonzero", "flatnonzero", "argsort", "sort", "unique",
              "allclose", "array_equal", "isclose", "deg2rad", "rad2deg", "degrees", "radians", "atleast_1d",
              "atleast_2d", "meshgrid", "split", "cross", "power", "trace", "diag", "diagonal", "zeros_like",
              "count_nonzero", "nansum", "maximum_reduce", "column_stack", "vstack", "hstack", "fmax",
              "fmin", "floor_divide", "mod", "searchsorted", "interp", "std", "var", "cbrt", "log10",
              "exp2", "log2", "arccos", "arcsin", "abs", "shape", "ndim", "size"):
    if _name in globals() or not hasattr(np, _name):
        continue
    globals()[_name] = _wrapped(getattr(np, _name))


def _norm(x, ord=None, axis=None, **kw):
    x = np.asarray(x)
    if np.iscomplexobj(x):
        return _wrap(np.sqrt(np.sum(x * x, axis=axis)))
    return _wrap(np.linalg.norm(x, ord=ord, axis=axis, **kw))


linalg = types.SimpleNamespace(
    norm=_norm,
    inv=_wrapped(np.linalg.inv),
    solve=_wrapped(np.linalg.solve),
    lstsq=lambda a, b, rcond=None: tuple(_wrap(v) for v in np.linalg.lstsq(a, b, rcond=rcond)),
    det=_wrapped(np.linalg.det),
    eigvals=_wrapped(np.linalg.eigvals),
    svd=_wrapped(np.linalg.svd),
)
