"""2D structured grid files: Plot3D read to blocks of nodes, and assembled into a mesh
of blocks with cuts and named patches.

The assembly follows the reference's (``src/jaxrans/mesh/assemble.py:97-315``), so that
a case directory with ``"grid": "file"`` loads to the same mesh:

1. every block made right-handed (``i`` reversed if its areas are negative);
2. coincident faces -- both end nodes within ``pair_tol`` of the smaller of the face's
   length and its cell's width across it -- matched into cuts, between blocks or within
   one (an O-grid's seam, a C-grid's wake cut);
3. every other face named by the case's patch rules (boxes; the first that contains
   the face's midpoint), else by the boundary loop it lies on: walked with the fluid on
   the left, a counter-clockwise loop is ``farfield``, a clockwise one (a body) ``wall``.

The Plot3D reader takes formatted (text) and unformatted (Fortran records, either byte
order) files, single or multi-block, with or without iblank, 2D or a thin 3D extrusion
of a 2D grid (the first plane of the thin index, in its two varying coordinates).
"""

from __future__ import annotations

import gzip
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .grids import SIDES, Block, Cut, Patch


@dataclass(frozen=True)
class PatchRule:
    """Boundary faces whose midpoints lie inside the box get the patch ``name``; a
    missing bound is unbounded (``src/jaxrans/mesh/assemble.py:37-52``)."""

    name: str
    x_min: float = -np.inf
    x_max: float = np.inf
    y_min: float = -np.inf
    y_max: float = np.inf
    z_min: float = -np.inf
    z_max: float = np.inf

    def contains(self, x, y, z=None):
        inside = (x >= self.x_min) & (x <= self.x_max) & (y >= self.y_min) & (y <= self.y_max)
        return inside if z is None else inside & (z >= self.z_min) & (z <= self.z_max)


# --- Plot3D ---------------------------------------------------------------------------------


def _raw(path: Path) -> bytes:
    data = path.read_bytes()
    return gzip.decompress(data) if data[:2] == b"\x1f\x8b" else data


def _binary(raw: bytes) -> bool:
    return any(b < 9 or 13 < b < 32 for b in raw[:4096])


def _blocks_from(values: np.ndarray, dims: np.ndarray, ndim: int, iblank: bool):
    out, at = [], 0
    for shape in dims:
        n = int(np.prod(shape))
        coords = []
        for _ in range(ndim):
            coords.append(values[at:at + n].reshape(tuple(shape), order="F"))
            at += n
        if iblank:
            at += n
        out.append(coords)
    return out if at == values.size else None


def _formatted(raw: bytes):
    text = raw.decode(errors="replace").replace("D", "E").replace("d", "e")
    tokens = text.split()
    try:
        numbers = np.array([float(t) for t in tokens])
    except ValueError:
        return None
    for multi in (True, False):
        for ndim in (2, 3):
            head = 1 if multi else 0
            if numbers.size <= head:
                continue
            nblocks = int(numbers[0]) if multi else 1
            if multi and (numbers[0] != nblocks or nblocks < 1):
                continue
            dims = numbers[head:head + ndim * nblocks]
            if dims.size < ndim * nblocks or np.any(dims != np.round(dims)) or np.any(dims < 1):
                continue
            dims = dims.astype(np.int64).reshape(nblocks, ndim)
            values = numbers[head + ndim * nblocks:]
            n = int(dims.prod(axis=1).sum())
            for iblank in (False, True):
                if values.size == n * (ndim + iblank):
                    return _blocks_from(values, dims, ndim, iblank)
    return None


def _records(raw: bytes, order: str):
    out, at = [], 0
    while at < len(raw):
        if at + 4 > len(raw):
            return None
        n = int(np.frombuffer(raw, order + "i4", 1, at)[0])
        if n < 0 or at + 8 + n > len(raw) or int(np.frombuffer(raw, order + "i4", 1, at + 4 + n)[0]) != n:
            return None
        out.append(raw[at + 4:at + 4 + n])
        at += n + 8
    return out


def _unformatted(raw: bytes):
    for order in ("<", ">"):
        records = _records(raw, order)
        if not records:
            continue
        for multi in (True, False):
            k = 0
            if multi:
                if len(records[0]) != 4:
                    continue
                nblocks, k = int(np.frombuffer(records[0], order + "i4")[0]), 1
            else:
                nblocks = 1
            if k >= len(records):
                continue
            dims = np.frombuffer(records[k], order + "i4")
            for ndim in (2, 3):
                if dims.size != ndim * nblocks or np.any(dims < 1) or len(records) != k + 1 + nblocks:
                    continue
                blocks = []
                for shape, rec in zip(dims.reshape(nblocks, ndim), records[k + 1:]):
                    n = int(np.prod(shape))
                    for fmt in ("f8", "f4"):
                        size = np.dtype(fmt).itemsize
                        if len(rec) in (n * ndim * size, n * (ndim * size + 4)):
                            v = np.frombuffer(rec, order + fmt, n * ndim).astype(np.float64)
                            blocks.append([v[c * n:(c + 1) * n].reshape(tuple(shape), order="F") for c in range(ndim)])
                            break
                    else:
                        break
                if len(blocks) == nblocks:
                    return blocks
    return None


def _plane(coords):
    """A 2D block of nodes ``(x, y)``: as given, or of a 3D block the first plane of a
    thin index (one or two planes) in the two coordinates that vary across it."""
    if len(coords) == 2:
        return np.ascontiguousarray(coords[0]), np.ascontiguousarray(coords[1])
    scale = max(float(np.abs(c).max()) for c in coords) or 1.0
    shape = coords[0].shape
    for axis in range(3):
        if shape[axis] > 2:
            continue
        first = [np.take(c, 0, axis) for c in coords]
        last = [np.take(c, -1, axis) for c in coords]
        same = [np.abs(a - b).max() <= 1e-10 * scale for a, b in zip(first, last)]
        flat = [np.ptp(a) <= 1e-10 * scale for a in first]
        in_plane = [k for k in range(3) if same[k] and not flat[k]]
        if len(in_plane) == 2:
            return tuple(np.ascontiguousarray(first[k]) for k in in_plane)
    raise ValueError(f"a 3D block of {shape} nodes is not a 2D plane extruded along a thin index")


def read_plot3d_blocks(path: str | Path) -> list[list[np.ndarray]]:
    """Every block of a Plot3D file as its coordinate arrays, two (2D) or three (3D),
    each of the block's node shape."""
    path = Path(path)
    raw = _raw(path)
    blocks = _unformatted(raw) if _binary(raw) else _formatted(raw)
    if blocks is None:
        raise ValueError(f"{path.name}: not a Plot3D grid this reader understands (formatted or unformatted, "
                         f"2D or 3D, single or multi-block, with or without iblank)")
    return blocks


def read_plot3d_2d(path: str | Path) -> list[tuple[np.ndarray, np.ndarray]]:
    """Every block of a Plot3D file as 2D node arrays ``(x, y)``, ``(ni+1, nj+1)`` each."""
    return [_plane(b) for b in read_plot3d_blocks(path)]


def write_plot3d_2d(path: str | Path, blocks: list[tuple[np.ndarray, np.ndarray]]) -> None:
    """A formatted multi-block 2D Plot3D file (``.p2dfmt``)."""
    lines = [str(len(blocks))]
    lines += [f"{x.shape[0]} {x.shape[1]}" for x, _ in blocks]
    for x, y in blocks:
        for c in (x, y):
            vals = np.asarray(c, dtype=np.float64).ravel(order="F")
            lines += [" ".join(f"{v:.17e}" for v in vals[s:s + 4]) for s in range(0, len(vals), 4)]
    Path(path).write_text("\n".join(lines) + "\n")


# --- assembly -----------------------------------------------------------------------------


def _right_handed(x, y):
    d1x, d1y = x[1:, 1:] - x[:-1, :-1], y[1:, 1:] - y[:-1, :-1]
    d2x, d2y = x[:-1, 1:] - x[1:, :-1], y[:-1, 1:] - y[1:, :-1]
    area = 0.5 * (d1x * d2y - d1y * d2x)
    if np.all(area > 0.0):
        return x, y
    if not np.all(area < 0.0):
        raise ValueError(f"a block of {x.shape} nodes folds over: cell areas of both signs")
    return x[::-1].copy(), y[::-1].copy()


def _widths(x, y):
    """Cell extent along each index direction, between opposite face midpoints."""
    mx_i, my_i = 0.5 * (x[:, :-1] + x[:, 1:]), 0.5 * (y[:, :-1] + y[:, 1:])
    mx_j, my_j = 0.5 * (x[:-1, :] + x[1:, :]), 0.5 * (y[:-1, :] + y[1:, :])
    return (np.hypot(mx_i[1:] - mx_i[:-1], my_i[1:] - my_i[:-1]),
            np.hypot(mx_j[:, 1:] - mx_j[:, :-1], my_j[:, 1:] - my_j[:, :-1]))


def _side_nodes(x, y, side):
    index = {"j_min": (slice(None), 0), "j_max": (slice(None), -1),
             "i_min": (0, slice(None)), "i_max": (-1, slice(None))}[side]
    return x[index], y[index]


@dataclass
class _Faces:
    block: np.ndarray
    side: np.ndarray
    cell: np.ndarray
    a: np.ndarray
    b: np.ndarray
    width: np.ndarray

    @property
    def length(self):
        return np.hypot(*(self.b - self.a).T)

    @property
    def mid(self):
        return 0.5 * (self.a + self.b)


def _faces(blocks) -> _Faces:
    parts = {k: [] for k in ("block", "side", "cell", "a", "b", "width")}
    for k, (x, y) in enumerate(blocks):
        wi, wj = _widths(x, y)
        across = {"j_min": wj[:, 0], "j_max": wj[:, -1], "i_min": wi[0, :], "i_max": wi[-1, :]}
        for s, side in enumerate(SIDES):
            sx, sy = _side_nodes(x, y, side)
            n = sx.size - 1
            parts["block"].append(np.full(n, k))
            parts["side"].append(np.full(n, s))
            parts["cell"].append(np.arange(n))
            parts["a"].append(np.stack([sx[:-1], sy[:-1]], axis=1))
            parts["b"].append(np.stack([sx[1:], sy[1:]], axis=1))
            parts["width"].append(across[side])
    return _Faces(*(np.concatenate(parts[k]) for k in ("block", "side", "cell", "a", "b", "width")))


def _match(faces: _Faces, pair_tol: float):
    """For every face the coincident face (-1: none) and whether it runs the other way:
    a sweep over the midpoints sorted by x, then both end nodes compared."""
    mid, tol = faces.mid, pair_tol * np.minimum(faces.length, faces.width)
    order = np.argsort(mid[:, 0])
    xs = mid[order, 0]
    lo = np.searchsorted(xs, mid[:, 0] - tol, side="left")
    hi = np.searchsorted(xs, mid[:, 0] + tol, side="right")
    me = np.repeat(np.arange(len(mid)), hi - lo)
    other = order[np.concatenate([np.arange(l, h) for l, h in zip(lo, hi)])] if len(me) else me
    keep = other != me
    me, other = me[keep], other[keep]

    def close(p, q):
        return np.hypot(*(p - q).T) <= tol[me]

    same = close(faces.a[me], faces.a[other]) & close(faces.b[me], faces.b[other])
    flipped = close(faces.a[me], faces.b[other]) & close(faces.b[me], faces.a[other])
    hit = same | flipped
    me, other, flipped = me[hit], other[hit], flipped[hit]
    if np.unique(me).size != me.size:
        raise ValueError("a face coincides with more than one other face")
    partner = np.full(len(mid), -1)
    reverse = np.zeros(len(mid), dtype=bool)
    partner[me], reverse[me] = other, flipped
    return partner, reverse


def _by_loop(faces: _Faces, boundary: np.ndarray) -> np.ndarray:
    """``farfield`` or ``wall`` for every boundary face by the orientation of its loop,
    walked with the fluid on the left (a face on no closed loop is ``wall``)."""
    names = np.full(len(boundary), None, dtype=object)
    rows = np.flatnonzero(boundary)
    if not rows.size:
        return names
    forward = np.isin(faces.side[rows], (SIDES.index("j_min"), SIDES.index("i_max")))
    a = np.where(forward[:, None], faces.a[rows], faces.b[rows])
    b = np.where(forward[:, None], faces.b[rows], faces.a[rows])
    tol = 1e-3 * np.hypot(*(b - a).T).min()

    def key(p):
        return tuple(np.round(p / tol).astype(np.int64))

    starts = {key(p): n for n, p in enumerate(a)}
    following = np.array([starts.get(key(p), -1) for p in b])
    seen = np.zeros(len(rows), dtype=bool)
    for start in range(len(rows)):
        if seen[start]:
            continue
        loop, face = [], start
        while face >= 0 and not seen[face]:
            seen[face] = True
            loop.append(face)
            face = following[face]
        closed = face == start
        area = 0.5 * np.sum(a[loop, 0] * b[loop, 1] - b[loop, 0] * a[loop, 1])
        names[rows[loop]] = "farfield" if closed and area > 0.0 else "wall"
    return names


def _segments(targets: list) -> list:
    """Per-cell targets along a side (a patch name, or ``(block, side, cell, reversed)``)
    to patches and cuts."""
    out, k = [], 0
    while k < len(targets):
        t = targets[k]
        stop = k + 1
        if isinstance(t, str):
            while stop < len(targets) and targets[stop] == t:
                stop += 1
            out.append(Patch(t, k, stop))
        else:
            block, side, cell, rev = t
            step = -1 if rev else 1
            while (stop < len(targets) and not isinstance(targets[stop], str)
                   and targets[stop][:2] == (block, side) and targets[stop][3] == rev
                   and targets[stop][2] == targets[stop - 1][2] + step):
                stop += 1
            last = targets[stop - 1][2]
            out.append(Cut(k, stop, block, side, min(cell, last), rev))
        k = stop
    return out


def assemble(raw, rules=(), pair_tol: float = 0.05) -> list[Block]:
    """Blocks of nodes ``(x, y)`` as read -> blocks with cuts and named patches."""
    blocks = [_right_handed(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)) for x, y in raw]
    faces = _faces(blocks)
    partner, reverse = _match(faces, pair_tol)
    names = _by_loop(faces, partner < 0)
    named = np.zeros(len(names), dtype=bool)
    for rule in rules:
        hit = ~named & rule.contains(faces.mid[:, 0], faces.mid[:, 1])
        names[hit], named[hit] = rule.name, True
    names[partner >= 0] = None
    mesh = []
    for k, (x, y) in enumerate(blocks):
        sides = {}
        for side in SIDES:
            rows = np.flatnonzero((faces.block == k) & (faces.side == SIDES.index(side)))
            rows = rows[np.argsort(faces.cell[rows])]
            targets = [names[r] if partner[r] < 0 else
                       (int(faces.block[partner[r]]), SIDES[faces.side[partner[r]]], int(faces.cell[partner[r]]),
                        bool(reverse[r])) for r in rows]
            sides[side] = _segments(targets)
        block = Block(x, y, sides)
        block.check()
        mesh.append(block)
    return mesh


def load_grid(path: str | Path, coordinate_scale: float = 1.0, rules=(), pair_tol: float = 0.05) -> list[Block]:
    """Read and assemble a 2D Plot3D file."""
    raw = [(coordinate_scale * x, coordinate_scale * y) for x, y in read_plot3d_2d(path)]
    return assemble(raw, tuple(rules), pair_tol)
