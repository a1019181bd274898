"""3D structured blocks: their sides, a C-H wing block generated from a section, and
Plot3D files.

The block model follows the reference's (``src/jaxrans/mesh/block3d.py:1-151``): a
block of cells ``(ni, nj, nk)`` has six sides named by the index constant on them, in
the order ``j_min, j_max, i_min, i_max, k_min, k_max``; along a side run its other two
index directions in ascending order; each side is tiled by rectangles of cells
``[start, stop)`` in those running indices -- a named patch (``Rect3``) or cells facing
cells of a side of a block (``Cut3``, the partner's running position an affine map of
mine).

``wing_block`` builds the single-block C-H grid of a straight-tapered, swept wing that
spans the domain from a root symmetry plane to a tip plane (each spanwise station the
section's 2D C-grid scaled to the local chord and moved by the sweep): ``i`` round the
section and out along the wake, ``j`` from the wall out, ``k`` along the span from the
tip plane to the root plane (the order that makes the block right-handed).  x runs
chordwise, y along the span, z up, as in the reference's 3D cases.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .geometry import Section
from .grids import CONDITION_KINDS, WALL_KINDS, c_grid, normal_steps

SIDES_3D = ("j_min", "j_max", "i_min", "i_max", "k_min", "k_max")
KINDS_3D = ("slip_wall", "no_slip_wall", "symmetry", "far_field")   # the 3D path's conditions
AXIS = {"i": 0, "j": 1, "k": 2}


def normal_axis(side: str) -> int:
    return AXIS[side[0]]


def running_axes(side: str) -> tuple[int, int]:
    """The two index directions along a side, ascending."""
    n = normal_axis(side)
    return tuple(a for a in range(3) if a != n)


@dataclass(frozen=True)
class Rect3:
    """Cells ``[start, stop)`` (running indices) of a side on patch ``name``, condition
    ``kind``."""

    name: str
    start: tuple[int, int]
    stop: tuple[int, int]
    kind: str | None = None

    def __post_init__(self) -> None:
        if self.kind is not None and self.kind not in CONDITION_KINDS:
            raise ValueError(f"unknown boundary condition {self.kind!r}; known: {CONDITION_KINDS}")


@dataclass(frozen=True)
class Cut3:
    """Cells ``[start, stop)`` of a side facing side ``side`` of block ``block``: my
    running position ``a`` faces the partner's ``p[m] = origin[m] + s_m (a[axes[m]] -
    start[axes[m]])``, ``s_m = -1`` where ``flip[m]``, taken modulo ``period[m]`` where
    that is positive."""

    start: tuple[int, int]
    stop: tuple[int, int]
    block: int
    side: str
    origin: tuple[int, int]
    axes: tuple[int, int] = (0, 1)
    flip: tuple[bool, bool] = (False, False)
    period: tuple[int, int] = (0, 0)

    def partner(self, a) -> tuple[int, int]:
        out = []
        for m in range(2):
            d = a[self.axes[m]] - self.start[self.axes[m]]
            p = self.origin[m] + (-d if self.flip[m] else d)
            out.append(p % self.period[m] if self.period[m] else p)
        return tuple(out)


@dataclass
class Block3:
    """Nodes ``(3, ni+1, nj+1, nk+1)`` and the rectangles tiling each side."""

    nodes: np.ndarray
    sides: dict = field(default_factory=dict)

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(n - 1 for n in self.nodes.shape[1:])

    def extent(self, side: str) -> tuple[int, int]:
        a, b = running_axes(side)
        return self.shape[a], self.shape[b]

    def boundaries(self) -> list:
        return [(s, r) for s in SIDES_3D for r in self.sides[s] if isinstance(r, Rect3)]

    def patches(self) -> list:
        """``(side, Rect3)`` of every named patch (as ``grids.Block.patches``)."""
        return self.boundaries()

    def with_kinds(self, kinds: dict[str, str]) -> "Block3":
        new = {s: [Rect3(r.name, r.start, r.stop, kinds[r.name]) if isinstance(r, Rect3) else r
                   for r in self.sides[s]] for s in SIDES_3D}
        return Block3(self.nodes, new)

    def check(self) -> None:
        """Every side tiled exactly once."""
        for side in SIDES_3D:
            n = self.extent(side)
            count = np.zeros(n, dtype=np.int64)
            for r in self.sides[side]:
                if not all(0 <= r.start[m] < r.stop[m] <= n[m] for m in range(2)):
                    raise ValueError(f"rectangle {r} outside {side} of extent {n}")
                count[r.start[0]:r.stop[0], r.start[1]:r.stop[1]] += 1
            if np.any(count != 1):
                raise ValueError(f"the rectangles of {side} do not tile it exactly once")

    def walls(self) -> list:
        return [(s, r) for s, r in self.boundaries() if r.kind in WALL_KINDS]


def wing_block(section: Section, cells_airfoil: int, cells_wake: int, cells_normal: int, cells_span: int,
               wall_spacing: float, far_field: float, semispan: float, taper: float = 1.0,
               sweep_deg: float = 0.0) -> Block3:
    """The C-H block of a wing from its root section (chord 1 at the root): at spanwise
    station ``y`` the root's 2D C-grid scaled by the local chord ``1 - (1 - taper) y /
    semispan`` about the root leading edge and moved aft by ``y tan(sweep)``.  Sides:
    the wall and the two wake-cut halves on ``j_min`` (the cut facing itself, ``i``
    reversed), far field on ``j_max``, ``i_min``, ``i_max``, the tip plane ``k_min``
    (patch ``tip``), the root plane ``k_max`` (patch ``root``)."""
    base = c_grid(section, cells_airfoil, cells_wake, cells_normal, wall_spacing, far_field)
    x2, z2 = base.x, base.y
    nk = cells_span
    y = semispan * (1.0 - np.arange(nk + 1) / nk)            # tip (k = 0) to root (k = nk)
    chord = 1.0 - (1.0 - taper) * y / semispan
    shift = y * math.tan(math.radians(sweep_deg))
    nodes = np.empty((3,) + x2.shape + (nk + 1,))
    nodes[0] = x2[..., None] * chord + shift
    nodes[1] = np.broadcast_to(y, x2.shape + (nk + 1,))
    nodes[2] = z2[..., None] * chord
    ni, nj, nw = base.ni, base.nj, cells_wake
    sides = {
        "j_min": [Cut3((0, 0), (nw, nk), 0, "j_min", (ni - 1, 0), (0, 1), (True, False)),
                  Rect3("wall", (nw, 0), (ni - nw, nk)),
                  Cut3((ni - nw, 0), (ni, nk), 0, "j_min", (nw - 1, 0), (0, 1), (True, False))],
        "j_max": [Rect3("farfield", (0, 0), (ni, nk))],
        "i_min": [Rect3("farfield", (0, 0), (nj, nk))],
        "i_max": [Rect3("farfield", (0, 0), (nj, nk))],
        "k_min": [Rect3("tip", (0, 0), (ni, nj))],
        "k_max": [Rect3("root", (0, 0), (ni, nj))],
    }
    block = Block3(nodes, sides)
    block.check()
    return block


@dataclass(frozen=True)
class WingGrid:
    """A multi-block wing grid as a grid file holds it: node arrays and the box patch
    rules (``domain.patches`` entries) that name its boundary faces, and the wing's
    reference area (semispan planform), length (mean aerodynamic chord) and centre."""

    blocks: list
    patches: list
    reference_area: float
    reference_length: float
    moment_centre: tuple


def wing_ch_blocks(section: Section, cells_airfoil: int, cells_wake: int, cells_normal: int, cells_span: int,
                   cells_tip: int, wall_spacing: float, far_field: float, semispan: float, taper: float = 1.0,
                   sweep_deg: float = 0.0, cap_cells: int = 4, span_far: float | None = None) -> WingGrid:
    """The four point-matched blocks of a C-H grid round a straight-tapered, swept wing
    with its tip, from the root section (chord 1):

    * spanwise, the wing (root symmetry plane ``y = 0`` to the tip ``y = semispan``,
      ``cells_span`` stations closing in on the tip) and the region beyond the tip out
      to the far field ``y = semispan + span_far`` (``cells_tip`` stations, default
      ``span_far`` = ``far_field`` root chords);
    * round the section, the lower half (lower wake and lower surface up to the
      leading edge) and the upper half, ``(cells_airfoil / 2 + cells_wake)`` cells each.

    Each spanwise station is the root's 2D C-grid scaled by the local chord about the
    leading edge and moved aft by the sweep (beyond the tip, the tip's).  Past the tip
    the section closes over ``cap_cells`` stations (an elliptic tip cap: its thickness
    times ``sqrt(1 - (m / cap_cells)^2)``) and then continues as a sheet of zero thickness
    on the chord line, whose two sides face each other like the wake cut -- for a
    symmetric section, whose C-grid's lower and upper surfaces are mirror images.
    ``k`` runs from the spanwise far field to the root, which makes every block
    right-handed.  Patches by box rules: ``symmetry`` (the root plane), ``wall`` (the
    wing and its cap), ``farfield``."""
    if cells_airfoil % 2:
        raise ValueError(f"cells round the airfoil must be even, got {cells_airfoil}")
    if not 0 < cap_cells < cells_tip:
        raise ValueError(f"cap_cells must lie in (0, cells_tip), got {cap_cells} of {cells_tip}")
    base = c_grid(section, cells_airfoil, cells_wake, cells_normal, wall_spacing, far_field)
    x2, z2 = base.x, base.y
    ni, nw = base.ni, cells_wake
    if np.abs(z2[:, 0] + z2[::-1, 0]).max() > 1e-9 or np.abs(x2[:, 0] - x2[::-1, 0]).max() > 1e-9:
        raise ValueError("the tip region's sheet needs a symmetric section (mirror-image lower and upper surfaces)")
    # the chord-line section: the surface moved onto z = 0, the move fading out over half a chord
    reach = np.concatenate([np.zeros((ni + 1, 1)), np.cumsum(np.hypot(np.diff(x2, axis=1), np.diff(z2, axis=1)),
                                                             axis=1)], axis=1)
    fade = (1.0 - np.minimum(reach / 0.5, 1.0)) ** 2
    lift = np.zeros(ni + 1)
    lift[nw:ni - nw + 1] = z2[nw:ni - nw + 1, 0]
    move = lift[:, None] * fade                               # z of the sheet = z2 - move
    tip_chord = 1.0 - (1.0 - taper)
    half_thickness = 0.5 * float(np.ptp(z2[:, 0])) * tip_chord
    step = half_thickness / cap_cells                         # spanwise spacing at the tip and in the cap
    far = far_field if span_far is None else span_far
    y_wing = semispan - np.concatenate([[0.0], np.cumsum(normal_steps(cells_span, step, semispan))])[::-1]
    beyond = np.concatenate([np.full(cap_cells, step), normal_steps(cells_tip - cap_cells, step,
                                                                    far - cap_cells * step)])
    y_tip = semispan + np.concatenate([[0.0], np.cumsum(beyond)])
    shift = math.tan(math.radians(sweep_deg))

    def stations(y, thickness):
        chord = 1.0 - (1.0 - taper) * np.minimum(y, semispan) / semispan
        dx = np.minimum(y, semispan) * shift
        nodes = np.empty((3,) + x2.shape + (len(y),))
        z = z2[..., None] - (1.0 - thickness) * move[..., None]
        nodes[0] = x2[..., None] * chord + dx
        nodes[1] = np.broadcast_to(y, x2.shape + (len(y),))
        nodes[2] = z * chord
        return nodes[..., ::-1]                               # k from the far side toward the root

    m = np.arange(cells_tip + 1)
    cap = np.sqrt(np.clip(1.0 - (m / cap_cells) ** 2, 0.0, None))
    wing = stations(y_wing, np.ones(cells_span + 1))
    tip = stations(y_tip, cap)
    lo, hi = slice(0, ni // 2 + 1), slice(ni // 2, ni + 1)
    blocks = [np.ascontiguousarray(b[:, s]) for b in (wing, tip) for s in (lo, hi)]
    reach_x = float(x2[nw:ni - nw + 1, 0].max()) + semispan * shift + 1.0
    patches = [{"name": "symmetry", "y_max": 1e-9 * semispan},
               {"name": "wall", "x_min": -1.0, "x_max": reach_x, "y_max": semispan + (cap_cells + 0.5) * step,
                "z_min": -1.0, "z_max": 1.0},
               {"name": "farfield"}]
    area = 0.5 * semispan * (1.0 + taper)
    mac = (2.0 / 3.0) * (1.0 + taper + taper * taper) / (1.0 + taper)
    return WingGrid(blocks, patches, area, mac, (0.25, 0.0, 0.0))


# --- Plot3D ------------------------------------------------------------------------------


def write_plot3d(path: str | Path, blocks: list[np.ndarray]) -> None:
    """Unformatted (Fortran records, little endian), multi-block 3D, FP64: the block
    count, the node dimensions, then each block's x, y, z with ``i`` fastest."""
    def record(payload: bytes) -> bytes:
        n = np.array([len(payload)], dtype="<i4").tobytes()
        return n + payload + n
    out = [record(np.array([len(blocks)], dtype="<i4").tobytes()),
           record(np.array([b.shape[1:] for b in blocks], dtype="<i4").ravel().tobytes())]
    for b in blocks:
        out.append(record(np.concatenate([np.asarray(b[c], dtype="<f8").ravel(order="F") for c in range(3)])
                          .tobytes()))
    Path(path).write_bytes(b"".join(out))


def read_plot3d(path: str | Path) -> list[np.ndarray]:
    """The node arrays ``(3, ni+1, nj+1, nk+1)`` of a 3D Plot3D file: formatted, or
    unformatted (Fortran records in either byte order, FP64 or FP32), with or without
    the block count, with or without iblank."""
    from .gridfile import read_plot3d_blocks
    blocks = read_plot3d_blocks(path)
    if any(len(b) != 3 for b in blocks):
        raise ValueError(f"{Path(path).name}: a 2D grid, not a 3D one")
    return [np.stack(b) for b in blocks]
