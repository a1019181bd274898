"""Generated O- and C-grids round one airfoil, by hyperbolic marching.

The wall line (O-grid: the closed contour; C-grid: lower wake, contour, upper
wake) is distributed with Vinokur's two-sided stretching (J. Comput. Phys. 50
(1983) 215-234), clustered at both edges, then marched outward layer by layer.
Each layer solves the linearised orthogonality and cell-area conditions
``r_xi . r_eta = 0``, ``r_xi x r_eta = dV`` of Steger and Chaussee (SIAM J. Sci.
Stat. Comput. 1 (1980) 431-437) as a 2x2 block tridiagonal system in ``xi``,
with implicit second-difference smoothing of the step.  The same method as the
reference's generator (``src/jaxrans/mesh/generate.py:141-269``), written here
afresh; a grid is an input to both the device path and the oracle, so only its
validity (positive cells, point-matched cuts) matters, not bitwise agreement.

Normal steps either grow geometrically from the first cell to reach the far
field (``ratio=None``: the ratio solved for), or start at a given ``ratio``
that rises linearly along the line to the value that reaches the far field
(a 1.1 stretching kept over 96 cells reaches only ~0.1 chord, so it must give
way somewhere; rising linearly keeps the growth smooth).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy.optimize import brentq
from scipy.sparse import coo_matrix
from scipy.sparse.linalg import spsolve

from .geometry import Section

LE_SPACING = 2e-3
TE_SPACING = 2e-3
SMOOTHING = 3.0


# --- Segments and blocks -------------------------------------------------------------

SIDES = ("j_min", "j_max", "i_min", "i_max")
OUTWARD = {"j_min": -1, "j_max": 1, "i_min": -1, "i_max": 1}
CONDITION_KINDS = ("slip_wall", "no_slip_wall", "symmetry", "far_field", "inflow_total", "outflow_static")
WALL_KINDS = ("slip_wall", "no_slip_wall")


@dataclass(frozen=True)
class Patch:
    """Cells ``[start, stop)`` along a side on patch ``name``, condition ``kind``
    (``src/jaxrans/mesh/block.py:37-51``)."""

    name: str
    start: int
    stop: int
    kind: str | None = None


@dataclass(frozen=True)
class Cut:
    """Cells ``[start, stop)`` facing ``[partner_start, partner_start + n)`` of
    ``side`` of block ``block``, in order or reversed
    (``src/jaxrans/mesh/block.py:54-75``)."""

    start: int
    stop: int
    block: int
    side: str
    partner_start: int
    reversed: bool

    def partner(self, a: int) -> int:
        off = a - self.start
        return self.partner_start + (self.stop - self.start - 1 - off if self.reversed else off)


@dataclass
class Block:
    """Nodes ``(ni+1, nj+1)`` each and the segments tiling each side."""

    x: np.ndarray
    y: np.ndarray
    sides: dict = field(default_factory=dict)

    @property
    def ni(self) -> int:
        return self.x.shape[0] - 1

    @property
    def nj(self) -> int:
        return self.x.shape[1] - 1

    def length(self, side: str) -> int:
        return self.ni if side.startswith("j") else self.nj

    def patches(self) -> list:
        return [(side, s) for side in SIDES for s in self.sides[side] if isinstance(s, Patch)]

    def with_kinds(self, kinds: dict[str, str]) -> "Block":
        new = {side: [Patch(s.name, s.start, s.stop, kinds[s.name]) if isinstance(s, Patch) else s
                      for s in self.sides[side]] for side in SIDES}
        return Block(self.x, self.y, new)

    def check(self) -> None:
        for side in SIDES:
            n = self.length(side)
            stops = [0] + [s.stop for s in self.sides[side]]
            starts = [s.start for s in self.sides[side]] + [n]
            if stops != starts:
                raise ValueError(f"segments of {side} do not tile [0, {n})")


def patch_names(mesh) -> list[str]:
    out: list[str] = []
    for block in mesh:
        for _, seg in block.patches():
            if seg.name not in out:
                out.append(seg.name)
    return out


# --- Distributions ---------------------------------------------------------------------


def vinokur(n: int, ds0: float, ds1: float) -> np.ndarray:
    """``n + 1`` points on [0, 1], end intervals near ``ds0`` and ``ds1``
    (fractions): Vinokur's two-sided tanh/tan stretching."""
    xi = np.linspace(0.0, 1.0, n + 1)
    s0, s1 = 1.0 / (n * ds0), 1.0 / (n * ds1)
    a, b = np.sqrt(s0 / s1), np.sqrt(s0 * s1)
    if abs(b - 1.0) < 1e-6:
        u = xi
    elif b > 1.0:
        d = brentq(lambda d: np.sinh(d) / d - b, 1e-12, 50.0)
        u = 0.5 * (1.0 + np.tanh(d * (xi - 0.5)) / np.tanh(0.5 * d))
    else:
        d = brentq(lambda d: np.sin(d) / d - b, 1e-12, np.pi - 1e-12)
        u = 0.5 * (1.0 + np.tan(d * (xi - 0.5)) / np.tan(0.5 * d))
    s = u / (a + (1.0 - a) * u)
    s[0], s[-1] = 0.0, 1.0
    return s


def normal_steps(n: int, first: float, total: float, ratio: float | None = None) -> np.ndarray:
    """``n`` step lengths from ``first`` summing to ``total``: geometric with the
    ratio solved for, or starting at ``ratio`` and rising linearly to reach ``total``."""
    if first * n >= total:
        raise ValueError(f"a first step of {first:g} over {n} steps already exceeds {total:g}")
    if ratio is None:
        r = brentq(lambda r: first * (r ** n - 1.0) / (r - 1.0) - total, 1.0 + 1e-12, 10.0)
        return first * r ** np.arange(n)

    def steps(r_end: float) -> np.ndarray:
        rates = np.linspace(ratio, r_end, n - 1)
        return first * np.concatenate([[1.0], np.cumprod(rates)])

    if steps(ratio).sum() >= total:
        r = brentq(lambda r: first * (r ** n - 1.0) / (r - 1.0) - total, 1.0 + 1e-12, ratio)
        return first * r ** np.arange(n)
    r_end = brentq(lambda r: steps(r).sum() - total, ratio, 10.0)
    return steps(r_end)


def wall_arcs(section: Section, n: int) -> np.ndarray:
    """``n + 1`` arc lengths round the contour, ``n / 2`` cells each side of the nose."""
    if n % 2:
        raise ValueError(f"cells round the airfoil must be even, got {n}")
    s_le, total, c = float(section.arc[section.nose]), section.length, section.chord
    lower = s_le * vinokur(n // 2, TE_SPACING * c / s_le, LE_SPACING * c / s_le)
    upper = s_le + (total - s_le) * vinokur(n // 2, LE_SPACING * c / (total - s_le),
                                            TE_SPACING * c / (total - s_le))
    return np.concatenate([lower, upper[1:]])


# --- Marching ----------------------------------------------------------------------------


def _d1(r: np.ndarray, closed: bool) -> np.ndarray:
    if closed:
        return 0.5 * (np.roll(r, -1, axis=0) - np.roll(r, 1, axis=0))
    d = np.empty_like(r)
    d[1:-1] = 0.5 * (r[2:] - r[:-2])
    d[0], d[-1] = r[1] - r[0], r[-1] - r[-2]
    return d


def _d2(r: np.ndarray, closed: bool) -> np.ndarray:
    if closed:
        return np.roll(r, -1, axis=0) - 2.0 * r + np.roll(r, 1, axis=0)
    d = np.zeros_like(r)
    d[1:-1] = r[2:] - 2.0 * r[1:-1] + r[:-2]
    return d


def march(line: np.ndarray, steps: np.ndarray, closed: bool, outflow: np.ndarray | None = None,
          smoothing: float = SMOOTHING) -> np.ndarray:
    """Layers ``(n, len(steps) + 1, 2)`` marched from ``line (n, 2)``."""
    n = len(line)
    layers = np.empty((n, len(steps) + 1, 2))
    layers[:, 0] = r = line.copy()
    eye = np.eye(2)
    for k, ds in enumerate(steps):
        t = _d1(r, closed)
        t2 = np.sum(t * t, axis=1)
        area = ds * np.sqrt(t2)
        for _ in range(2):
            if closed:
                area = 0.5 * area + 0.25 * (np.roll(area, 1) + np.roll(area, -1))
            else:
                area[1:-1] = 0.5 * area[1:-1] + 0.25 * (area[:-2] + area[2:])
        # the orthogonal step of the target area, and C = A^-1 B of the linearisation
        eta = (area / t2)[:, None] * np.stack([-t[:, 1], t[:, 0]], axis=1)
        tx, ty, ex, ey = t[:, 0], t[:, 1], eta[:, 0], eta[:, 1]
        C = np.empty((n, 2, 2))
        C[:, 0, 0] = (tx * ex - ty * ey) / t2
        C[:, 0, 1] = (tx * ey + ty * ex) / t2
        C[:, 1, 0] = (ty * ex + tx * ey) / t2
        C[:, 1, 1] = (ty * ey - tx * ex) / t2
        rhs = r + eta + np.einsum("nab,nb->na", C, t) - smoothing * _d2(r, closed)
        # the entries row by row, each row's three 2x2 blocks left to right, zeros
        # dropped: the sparse matrix the solver sees is the same entry for entry
        i = np.arange(n) if closed else np.arange(1, n - 1)
        Ci = C[i]
        blocks = np.stack([-0.5 * Ci - smoothing * eye, np.broadcast_to((1.0 + 2.0 * smoothing) * eye, Ci.shape),
                           0.5 * Ci - smoothing * eye], axis=1)                    # (m, 3, 2, 2)
        j = np.stack([(i - 1) % n, i, (i + 1) % n], axis=1)                         # (m, 3)
        ab = np.arange(2)
        r_idx = np.broadcast_to(2 * i[:, None, None, None] + ab[None, None, :, None], blocks.shape)
        c_idx = np.broadcast_to(2 * j[:, :, None, None] + ab[None, None, None, :], blocks.shape)
        keep = blocks.ravel() != 0.0
        rows = list(r_idx.ravel()[keep])
        cols = list(c_idx.ravel()[keep])
        vals = list(blocks.ravel()[keep])

        def put(i, j, block):
            for a in range(2):
                for b in range(2):
                    if block[a, b] != 0.0:
                        rows.append(2 * i + a)
                        cols.append(2 * j + b)
                        vals.append(block[a, b])

        if not closed:
            w = outflow / np.linalg.norm(outflow)
            m = np.array([-w[1], w[0]])
            for end, inner in ((0, 1), (n - 1, n - 2)):
                put(end, end, np.stack([w, m]))
                put(end, inner, np.stack([np.zeros(2), -m]))
                rhs[end] = [w @ r[end], 0.0]
        A = coo_matrix((vals, (rows, cols)), shape=(2 * n, 2 * n)).tocsc()
        r = spsolve(A, rhs.ravel()).reshape(n, 2)
        layers[:, k + 1] = r
    return layers


def _reach(wall: np.ndarray, outer: np.ndarray) -> float:
    d = np.hypot(outer[:, None, 0] - wall[None, ::4, 0], outer[:, None, 1] - wall[None, ::4, 1])
    return float(d.min())


def _march_to(line, wall, cells_normal, first, far, ratio, **kw) -> np.ndarray:
    total = far
    for _ in range(5):
        layers = march(line, normal_steps(cells_normal, first, total, ratio), **kw)
        reach = _reach(wall, layers[:, -1])
        if abs(reach - far) <= 0.01 * far:
            break
        total *= far / reach
    return layers


def folded(x: np.ndarray, y: np.ndarray) -> bool:
    d1x, d1y = x[1:, 1:] - x[:-1, :-1], y[1:, 1:] - y[:-1, :-1]
    d2x, d2y = x[:-1, 1:] - x[1:, :-1], y[:-1, 1:] - y[1:, :-1]
    return not np.all(0.5 * (d1x * d2y - d1y * d2x) > 0.0)


def o_grid(section: Section, cells_airfoil: int, cells_normal: int, wall_spacing: float,
           far_field: float = 100.0, ratio: float | None = None) -> Block:
    """A single-block O-grid: ``i`` round the body from the trailing edge (lower
    surface first), ``j`` outward; wall on ``j_min``, far field on ``j_max``, the
    seam ``i_min`` <-> ``i_max``."""
    if not section.sharp:
        raise ValueError("o_grid: a blunt trailing edge is not implemented in jaxrans_b200; "
                         "use a sharp NACA section (domain.trailing_edge = \"close\")")
    c = section.chord
    x, y = section.at(wall_arcs(section, cells_airfoil))
    line = np.stack([x[:-1], y[:-1]], axis=1)
    layers = _march_to(line, line, cells_normal, wall_spacing * c, far_field * c, ratio, closed=True)
    layers = np.concatenate([layers, layers[:1]], axis=0)
    ni, nj = cells_airfoil, cells_normal
    sides = {"j_min": [Patch("wall", 0, ni)], "j_max": [Patch("farfield", 0, ni)],
             "i_min": [Cut(0, nj, 0, "i_max", 0, False)], "i_max": [Cut(0, nj, 0, "i_min", 0, False)]}
    block = Block(layers[..., 0].copy(), layers[..., 1].copy(), sides)
    if folded(block.x, block.y):
        raise ValueError(f"the generated O-grid folds ({cells_airfoil} x {cells_normal}); "
                         f"refine it or move the far field in")
    return block


def c_grid(section: Section, cells_airfoil: int, cells_wake: int, cells_normal: int, wall_spacing: float,
           far_field: float = 100.0, ratio: float | None = None) -> Block:
    """A single-block C-grid: ``i`` from the downstream end of the lower wake,
    round the airfoil (lower surface first) and out along the upper wake; the
    wake cut is ``j_min`` against itself, reversed."""
    if not section.sharp:
        raise ValueError("c_grid: a blunt trailing edge is not implemented in jaxrans_b200; "
                         "close it (domain.trailing_edge = \"close\")")
    c = section.chord
    x, y = section.at(wall_arcs(section, cells_airfoil))
    x[-1], y[-1] = x[0], y[0]
    first = np.hypot(x[1] - x[0], y[1] - y[0])
    fx, fy = section.splines()
    lower = np.array([fx(0.0, 1), fy(0.0, 1)])
    upper = -np.array([fx(section.length, 1), fy(section.length, 1)])
    direction = -(lower / np.linalg.norm(lower) + upper / np.linalg.norm(upper))
    direction /= np.linalg.norm(direction)
    s = np.concatenate([[0.0], np.cumsum(normal_steps(cells_wake, first, far_field * c))])
    wx, wy = x[0] + s * direction[0], y[0] + s * direction[1]
    line = np.stack([np.concatenate([wx[::-1], x[1:-1], wx]), np.concatenate([wy[::-1], y[1:-1], wy])], axis=1)
    layers = _march_to(line, np.stack([x, y], axis=1), cells_normal, wall_spacing * c, far_field * c, ratio,
                       closed=False, outflow=direction)
    ni, nj, nw = cells_airfoil + 2 * cells_wake, cells_normal, cells_wake
    sides = {"j_min": [Cut(0, nw, 0, "j_min", ni - nw, True), Patch("wall", nw, ni - nw),
                       Cut(ni - nw, ni, 0, "j_min", 0, True)],
             "j_max": [Patch("farfield", 0, ni)], "i_min": [Patch("farfield", 0, nj)],
             "i_max": [Patch("farfield", 0, nj)]}
    block = Block(layers[..., 0].copy(), layers[..., 1].copy(), sides)
    if folded(block.x, block.y):
        raise ValueError(f"the generated C-grid folds ({ni} x {nj}); refine it or move the far field in")
    return block
