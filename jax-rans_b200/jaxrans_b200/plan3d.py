"""The static plan of a 3D mesh: the canvas the 3D kernels run on.

Every block, with a ring of ``g = 2`` ghost cells, is a tile of one 3D canvas
``(NI, NJ, NK)``; block ``b``'s cell ``(i, j, k)`` sits at flat index
``((oi + g + i) NJ + (oj + g + j)) NK + (ok + g + k)``.  The tables mean what the
reference's 3D atlas makes them mean (``src/jaxrans/mesh/atlas3d.py:119-287``), so that
results can be compared entry by entry:

* the canvas geometry: each tile's nodes grown by ``g`` linearly extrapolated layers,
  its metrics (volume, face area vectors of the three families toward increasing
  index, centres), the block's own cells inside; gaps between tiles a lattice of unit
  cells that nothing reads;
* the ghost fill as three gather stages per pass, each block's side pairs in its
  ``fill_order`` (the wall-normal pair first), every side extended over the ghosts of
  the stages before it; the stages repeat until no read is of an unfilled ghost
  (``passes``: one on a single block);
* ghost centres reflected through physical faces and copied across cuts;
* line chains along each block's wall-normal index; wall faces; the wall distance.

The metrics follow the reference's formulas (``src/jaxrans/mesh/block.py:225-275``): a
quadrilateral face's vector area is half the cross product of its diagonals (the six
of a cell close exactly), the volume is a third of the outward flux of the position
through the faces, the centre the mean of the eight nodes.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .grid3d import SIDES_3D, Block3, Cut3, normal_axis, running_axes
from .grids import WALL_KINDS

G = 2
MAX_PASSES = 4


def metrics3d(nodes: np.ndarray):
    """``(centres (3, ni, nj, nk), volume (ni, nj, nk), faces)`` of nodes ``(3, ni+1, nj+1,
    nk+1)``; ``faces[a]`` is ``(3, ...)`` with one more entry along axis ``a``."""
    faces = []
    for axis in range(3):
        a1, a2 = (axis + 1) % 3, (axis + 2) % 3
        n = np.moveaxis(nodes, (1 + axis, 1 + a1, 1 + a2), (1, 2, 3))
        p00, p10, p11, p01 = n[:, :, :-1, :-1], n[:, :, 1:, :-1], n[:, :, 1:, 1:], n[:, :, :-1, 1:]
        S = 0.5 * np.cross(p11 - p00, p01 - p10, axis=0)
        mid = 0.25 * (p00 + p10 + p11 + p01)
        faces.append((np.moveaxis(S, (1, 2, 3), (1 + axis, 1 + a1, 1 + a2)),
                      np.moveaxis(mid, (1, 2, 3), (1 + axis, 1 + a1, 1 + a2))))
    volume = 0.0
    for axis, (S, mid) in enumerate(faces):
        flux = np.sum(S * mid, axis=0)
        hi = np.take(flux, range(1, flux.shape[axis]), axis=axis)
        lo = np.take(flux, range(0, flux.shape[axis] - 1), axis=axis)
        volume = volume + (hi - lo)
    volume = volume / 3.0
    ni, nj, nk = nodes.shape[1] - 1, nodes.shape[2] - 1, nodes.shape[3] - 1
    corners = [nodes[:, i:i + ni, j:j + nj, k:k + nk] for i in (0, 1) for j in (0, 1) for k in (0, 1)]
    centres = sum(corners) / 8.0
    return centres, volume, tuple(S for S, _ in faces)


def extended_nodes(nodes: np.ndarray, g: int) -> np.ndarray:
    """Nodes grown by ``g`` linearly extrapolated layers on every side, axis by axis."""
    for axis in range(1, 4):
        a = np.moveaxis(nodes, axis, 0)
        lo = [a[0] - (k + 1) * (a[1] - a[0]) for k in range(g)][::-1]
        hi = [a[-1] + (k + 1) * (a[-1] - a[-2]) for k in range(g)]
        nodes = np.moveaxis(np.concatenate([np.stack(lo), a, np.stack(hi)]), 0, axis)
    return nodes


def cell_on(side: str, a, layer: int, shape, inward: bool) -> tuple[int, int, int]:
    """The cell ``layer`` cells inward from (or outward beyond) ``side`` at running
    position ``a``."""
    n = normal_axis(side)
    out = [0, 0, 0]
    for m, axis in enumerate(running_axes(side)):
        out[axis] = a[m]
    low = side.endswith("min")
    if inward:
        out[n] = layer if low else shape[n] - 1 - layer
    else:
        out[n] = -1 - layer if low else shape[n] + layer
    return tuple(out)


def side_geometry(nodes: np.ndarray, faces, shape, side: str):
    """Outward unit normals and midpoints ``(3, na, nb)`` of a side's faces (a collapsed
    face has a zero normal)."""
    n = normal_axis(side)
    index = 0 if side.endswith("min") else shape[n]
    S = np.take(faces[n], index, axis=1 + n)
    plane = np.take(nodes, index, axis=1 + n)
    length = np.linalg.norm(S, axis=0)
    sign = -1.0 if side.endswith("min") else 1.0
    normal = np.where(length > 0.0, sign * S / np.where(length > 0.0, length, 1.0), 0.0)
    mid = 0.25 * (plane[:, :-1, :-1] + plane[:, 1:, :-1] + plane[:, :-1, 1:] + plane[:, 1:, 1:])
    return normal, mid


def line_axis(block: Block3) -> int:
    """The direction of a block's line chains: the normal of most of its wall faces,
    else of its far-field faces, else ``j``."""
    for kinds in (WALL_KINDS, ("far_field",)):
        count = [0, 0, 0]
        for side, r in block.boundaries():
            if r.kind in kinds:
                count[normal_axis(side)] += (r.stop[0] - r.start[0]) * (r.stop[1] - r.start[1])
        if max(count):
            return int(np.argmax(count))
    return 1


def fill_order(block: Block3) -> tuple[int, int, int]:
    first = line_axis(block)
    return (first, *(a for a in range(3) if a != first))


@dataclass
class Stage3:
    """A gather stage: ``index`` (one per canvas cell) is the cell itself, the cell a
    ghost copies across a cut, or ``n_canvas + r`` for condition row ``r``; rows are
    grouped by condition kind in first-seen order, each with its source cell, outward
    unit normal and face midpoint.  Every read of a stage precedes its writes."""

    index: np.ndarray
    conditions: tuple          # (kind, source (n,), normal (3, n), midpoint (3, n))


@dataclass
class Lines3:
    cells: np.ndarray
    up_face: np.ndarray
    up_sign: np.ndarray
    down_face: np.ndarray
    down_sign: np.ndarray


@dataclass
class WallQuads:
    """Every wall face: block, side (index into ``SIDES_3D``), running position
    ``(n, 2)`` and corners ``(n, 4, 3)`` in running order."""

    block: np.ndarray
    side: np.ndarray
    cell: np.ndarray
    corners: np.ndarray


@dataclass
class Walls3:
    quads: WallQuads
    cell: np.ndarray
    family: np.ndarray
    face: np.ndarray
    into_fluid: np.ndarray


@dataclass
class Plan3:
    mesh: list
    g: int
    origins: list
    shape: tuple
    interior: np.ndarray        # (NI, NJ, NK) bool
    volume: np.ndarray          # (NI, NJ, NK)
    faces: tuple                # 3 x (3, ...): family a has one more entry along a
    centres: np.ndarray         # (3, NI+2, NJ+2, NK+2)
    stages: list                # the stages of every pass, in order
    neighbours: np.ndarray
    lines: Lines3
    walls: Walls3
    distance: np.ndarray | None = None
    extras: dict = field(default_factory=dict)
    dim = 3

    @property
    def n_canvas(self) -> int:
        return int(np.prod(self.shape))

    @property
    def cells(self) -> int:
        return int(self.interior.sum())

    def windows(self):
        return [tuple(slice(o + self.g, o + self.g + n) for o, n in zip(origin, b.shape))
                for b, origin in zip(self.mesh, self.origins)]

    def pack(self, blocks, fill=0.0) -> np.ndarray:
        lead = blocks[0].shape[:-3]
        out = np.full(lead + self.shape, fill, dtype=np.float64)
        for value, w in zip(blocks, self.windows()):
            out[(Ellipsis,) + w] = value
        return out

    def unpack(self, canvas: np.ndarray) -> list:
        """Each block's cells of a canvas field ``(..., NI, NJ, NK)``."""
        return [canvas[(Ellipsis,) + w] for w in self.windows()]


def _pack2(shapes):
    """First fit in columns: the plane as tall as the tallest tile; tiles taken tallest
    first (then widest), each stacked on the first column at least as wide as it with
    room left, else starting a new column (as wide as that tile) to the right."""
    height = max(h for _, h in shapes)
    origins = [None] * len(shapes)
    columns = []                            # [x, width, height used]
    for k in sorted(range(len(shapes)), key=lambda k: (-shapes[k][1], -shapes[k][0])):
        w, h = shapes[k]
        col = next((c for c in columns if w <= c[1] and c[2] + h <= height), None)
        if col is None:
            col = [columns[-1][0] + columns[-1][1] if columns else 0, w, 0]
            columns.append(col)
        origins[k] = (col[0], col[2])
        col[2] += h
    return origins, (columns[-1][0] + columns[-1][1], height)


def pack_tiles(tiles):
    """Origins and canvas shape: tiles packed in the plane of two axes, as deep as the
    deepest along the third, the depth axis the one giving the smallest canvas."""
    best = None
    for depth in range(3):
        a, b = (x for x in range(3) if x != depth)
        flat, (na, nb) = _pack2([(t[a], t[b]) for t in tiles])
        shape = [0, 0, 0]
        shape[a], shape[b], shape[depth] = na, nb, max(t[depth] for t in tiles)
        if best is None or np.prod(shape) < np.prod(best[1]):
            origins = []
            for x, y in flat:
                o = [0, 0, 0]
                o[a], o[b] = x, y
                origins.append(tuple(o))
            best = (origins, tuple(shape))
    return best


def build_plan3d(mesh, g: int = G, with_distance: bool = True, distance_on: str = "auto") -> Plan3:
    """Pack ``mesh`` (3D blocks whose patches carry conditions) and build every table.
    The wall distance is computed on the device (``jr_wall_distance3d``) when
    ``distance_on`` is ``"device"``, or ``"auto"`` with a CUDA device present; on the
    host (NumPy) otherwise."""
    if distance_on not in ("auto", "device", "host"):
        raise ValueError(f"distance_on must be auto, device or host, got {distance_on!r}")
    mesh = list(mesh)
    for block in mesh:
        block.check()
        unset = sorted({r.name for _, r in block.boundaries() if r.kind is None})
        if unset:
            raise ValueError(f"patch(es) {unset} have no boundary condition")
    origins, canvas = pack_tiles([tuple(n + 2 * g for n in b.shape) for b in mesh])
    NI, NJ, NK = canvas
    n_canvas = NI * NJ * NK

    def pos(b, i, j, k):
        oi, oj, ok = origins[b]
        return ((oi + g + i) * NJ + (oj + g + j)) * NK + (ok + g + k)

    windows = [tuple(slice(o + g, o + g + n) for o, n in zip(origins[b], block.shape))
               for b, block in enumerate(mesh)]
    interior = np.zeros(canvas, dtype=bool)
    for w in windows:
        interior[w] = True
    lattice = np.stack(np.meshgrid(*(np.arange(n, dtype=np.float64) for n in canvas), indexing="ij"))
    centres, volume = 1e3 + 10.0 * lattice, np.ones(canvas)
    faces = [np.zeros((3,) + tuple(n + (a == x) for x, n in enumerate(canvas))) for a in range(3)]
    block_geometry = []
    for block, origin, window in zip(mesh, origins, windows):
        tc, tv, tf = metrics3d(extended_nodes(np.asarray(block.nodes, dtype=np.float64), g))
        tile = tuple(slice(o, o + n) for o, n in zip(origin, tv.shape))
        centres[(slice(None),) + tile] = tc
        volume[tile] = np.where(np.abs(tv) > 1e-300, tv, 1.0)
        bc, bv, bf = metrics3d(np.asarray(block.nodes, dtype=np.float64))
        volume[window] = bv
        for a, f in enumerate(tf):
            faces[a][(slice(None),) + tuple(slice(o, o + n) for o, n in zip(origin, f.shape[1:]))] = f
        block_geometry.append((bc, bv, bf))

    def stage(layers: int, which: int) -> Stage3:
        index = np.arange(n_canvas)
        entries: dict[str, list] = {}
        for b, block in enumerate(mesh):
            shape = block.shape
            order = fill_order(block)
            handled = set(order[:which])
            name = "ijk"[order[which]]
            for side in (f"{name}_min", f"{name}_max"):
                normal, mid = side_geometry(block.nodes, block_geometry[b][2], shape, side)
                axes = running_axes(side)
                n = tuple(shape[a] for a in axes)
                for rect in block.sides[side]:
                    ranges = []
                    for m, axis in enumerate(axes):
                        ext = layers if axis in handled else 0
                        lo = rect.start[m] - (ext if rect.start[m] == 0 else 0)
                        hi = rect.stop[m] + (ext if rect.stop[m] == n[m] else 0)
                        ranges.append(range(lo, hi))
                    for a in ((x, y) for x in ranges[0] for y in ranges[1]):
                        for layer in range(layers):
                            ghost = pos(b, *cell_on(side, a, layer, shape, inward=False))
                            if isinstance(rect, Cut3):
                                partner = mesh[rect.block].shape
                                p = list(rect.partner(a))
                                for m, axis in enumerate(running_axes(rect.side)):
                                    corner = layers if axes[rect.axes[m]] in handled else 0
                                    p[m] = min(max(p[m], -corner), partner[axis] - 1 + corner)
                                index[ghost] = pos(rect.block, *cell_on(rect.side, p, layer, partner, inward=True))
                            else:
                                read = layer if rect.kind in (*WALL_KINDS, "symmetry") else 0
                                source = pos(b, *cell_on(side, a, read, shape, inward=True))
                                f = tuple(min(max(a[m], 0), n[m] - 1) for m in range(2))
                                entries.setdefault(rect.kind, []).append(
                                    (ghost, source, *normal[:, f[0], f[1]], *mid[:, f[0], f[1]]))
        conditions, offset = [], n_canvas
        for kind, rows in entries.items():
            rows = np.array(rows)
            index[rows[:, 0].astype(np.int64)] = offset + np.arange(len(rows))
            offset += len(rows)
            conditions.append((kind, rows[:, 1].astype(np.int64), rows[:, 2:5].T.copy(), rows[:, 5:8].T.copy()))
        return Stage3(index, tuple(conditions))

    plans = {layers: [stage(layers, s) for s in range(3)] for layers in (g, 1)}
    passes = {layers: count_passes(p, interior.ravel()) for layers, p in plans.items()}
    flat = centres.reshape(3, -1)
    for st in plans[1] * passes[1]:
        flat = reflect(st, flat)
    centres = np.pad(flat.reshape((3,) + canvas), ((0, 0), (1, 1), (1, 1), (1, 1)), mode="edge")
    plan = Plan3(mesh, g, origins, canvas, interior, volume, tuple(faces), centres, plans[g] * passes[g],
                 _neighbours(mesh, pos, n_canvas), _lines(mesh, origins, g, canvas),
                 _walls(mesh, origins, pos, g, canvas))
    if with_distance:
        centres_of = [c for c, _, _ in block_geometry]
        if _on_device(distance_on):
            from .native3d import wall_distance_device
            points = np.concatenate([np.moveaxis(c, 0, -1).reshape(-1, 3) for c in centres_of])
            flat = wall_distance_device(points, plan.walls.quads.corners) if len(plan.walls.quads.corners) \
                else np.full(len(points), np.inf)
            parts, at = [], 0
            for b in mesh:
                n = int(np.prod(b.shape))
                parts.append(flat[at:at + n].reshape(b.shape))
                at += n
        else:
            parts = [wall_distance3d(b, plan.walls.quads, c) for b, c in zip(mesh, centres_of)]
        plan.distance = plan.pack(parts, 1.0)
    return plan


def _on_device(distance_on: str) -> bool:
    if distance_on != "auto":
        return distance_on == "device"
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def reflect(stage: Stage3, centres: np.ndarray) -> np.ndarray:
    """A stage applied to centres ``(3, n)``: copies across cuts, reflections through
    physical faces."""
    parts = [centres]
    for _, source, normal, midpoint in stage.conditions:
        x = centres[:, source]
        d = np.sum((x - midpoint) * normal, axis=0)
        parts.append(x - 2.0 * d * normal)
    return np.concatenate(parts, axis=1)[:, stage.index]


def count_passes(stages, interior: np.ndarray) -> int:
    """How many times the stages run so that the last pass reads filled cells only."""
    filled = interior.copy()
    for passes in range(1, MAX_PASSES + 1):
        clean = True
        for st in stages:
            written = st.index != np.arange(len(filled))
            read = np.concatenate([filled] + [filled[s] for _, s, _, _ in st.conditions])[st.index]
            clean &= bool(np.all(read[written]))
            filled = np.where(written, read, filled)
        if clean:
            return passes
    raise ValueError(f"the ghost fill does not settle in {MAX_PASSES} passes: a cut map is inconsistent")


def _neighbours(mesh, pos, n_canvas: int) -> np.ndarray:
    """Across every block face, the cell on the other side, or the cell itself."""
    index = np.arange(n_canvas)
    for b, block in enumerate(mesh):
        for side in SIDES_3D:
            for rect in block.sides[side]:
                for a in ((x, y) for x in range(rect.start[0], rect.stop[0])
                          for y in range(rect.start[1], rect.stop[1])):
                    ghost = pos(b, *cell_on(side, a, 0, block.shape, inward=False))
                    if isinstance(rect, Cut3):
                        partner = mesh[rect.block].shape
                        index[ghost] = pos(rect.block, *cell_on(rect.side, rect.partner(a), 0, partner, inward=True))
                    else:
                        index[ghost] = pos(b, *cell_on(side, a, 0, block.shape, inward=True))
    return index


def _lines(mesh, origins, g: int, canvas) -> Lines3:
    """A chain per block and pair of the other indices, along its line axis; link faces
    are flat indices into the three face families concatenated."""
    dims = [tuple(n + (a == x) for x, n in enumerate(canvas)) for a in range(3)]
    offsets = np.cumsum([0] + [int(np.prod(d)) for d in dims])
    chains, links = [], []
    for block, origin in zip(mesh, origins):
        axis = line_axis(block)
        cells = np.stack(np.meshgrid(*(o + g + np.arange(n) for o, n in zip(origin, block.shape)), indexing="ij"))
        cells = np.moveaxis(cells, 1 + axis, -1).reshape(3, -1, block.shape[axis])
        above = cells.copy()
        above[axis] += 1
        chains.append(np.ravel_multi_index(tuple(cells), canvas))
        links.append(offsets[axis] + np.ravel_multi_index(tuple(above), dims[axis]))
    length = max(c.shape[1] for c in chains)

    def pad(a, fill):
        return np.pad(a, ((0, 0), (0, length - a.shape[1])), constant_values=fill)

    cells = np.concatenate([pad(c, -1) for c in chains]).astype(np.int64)
    up_sign = ((cells >= 0) & (np.roll(cells, -1, axis=1) >= 0)).astype(np.int64)
    up_sign[:, -1] = 0
    face = np.where(up_sign != 0, np.concatenate([pad(f, 0) for f in links]), 0).astype(np.int64)
    return Lines3(cells, face, up_sign, face.copy(), -up_sign)


def wall_quads(mesh) -> WallQuads:
    rows = []
    for b, block in enumerate(mesh):
        for side, rect in block.walls():
            n = normal_axis(side)
            plane = np.take(block.nodes, 0 if side.endswith("min") else block.shape[n], axis=1 + n)
            for x in range(rect.start[0], rect.stop[0]):
                for y in range(rect.start[1], rect.stop[1]):
                    quad = np.stack([plane[:, x, y], plane[:, x + 1, y], plane[:, x + 1, y + 1], plane[:, x, y + 1]])
                    rows.append((b, SIDES_3D.index(side), x, y, quad))
    if not rows:
        empty = np.zeros(0, dtype=np.int64)
        return WallQuads(empty, empty, np.zeros((0, 2), np.int64), np.zeros((0, 4, 3)))
    return WallQuads(np.array([r[0] for r in rows]), np.array([r[1] for r in rows]),
                     np.array([r[2:4] for r in rows]), np.stack([r[4] for r in rows]))


def _walls(mesh, origins, pos, g: int, canvas) -> Walls3:
    quads = wall_quads(mesh)
    cell, family, face, sign = [], [], [], []
    for b, s, a in zip(quads.block, quads.side, quads.cell):
        side = SIDES_3D[s]
        c = cell_on(side, tuple(a), 0, mesh[b].shape, inward=True)
        cell.append(pos(b, *c))
        n = normal_axis(side)
        f = [o + g + x for o, x in zip(origins[b], c)]
        f[n] += side.endswith("max")
        dims = list(canvas)
        dims[n] += 1
        family.append(n)
        face.append((f[0] * dims[1] + f[1]) * dims[2] + f[2])
        sign.append(1.0 if side.endswith("min") else -1.0)
    return Walls3(quads, np.array(cell, dtype=np.int64), np.array(family, dtype=np.int64),
                  np.array(face, dtype=np.int64), np.array(sign))


# --- Wall distance ------------------------------------------------------------------------
# The exact distance from a point to the bilinear patch of a wall face: every face is
# first ranked by the distance to its two triangles (point-triangle distance by
# barycentric projection and the three edges, Ericson, Real-Time Collision Detection,
# 2005, 5.1.5), then the patch distance (Newton on |x(u, v) - p|^2 from the patch
# centre, kept if it lands inside, and the four edges) is taken over the nearest
# CANDIDATES faces -- the method of the reference (src/jaxrans/mesh/wall3d.py:1-158).

CANDIDATES = 16
NEWTON_ITERATIONS = 12


def _dot(u, v):
    return np.sum(u * v, axis=-1)


def triangle_distance(p, a, b, c):
    ab, ac = b - a, c - a
    n = np.cross(ab, ac)
    nn = _dot(n, n)
    ap = p - a
    safe = np.where(nn > 0.0, nn, 1.0)
    v = _dot(np.cross(ap, ac), n) / safe
    w = _dot(np.cross(ab, ap), n) / safe
    inside = (nn > 0.0) & (v >= 0.0) & (w >= 0.0) & (v + w <= 1.0)
    best = np.where(inside, np.abs(_dot(ap, n)) / np.sqrt(safe), np.inf)
    for s, e in ((a, b), (b, c), (c, a)):
        best = np.minimum(best, _segment_distance(p, s, e))
    return best


def _segment_distance(p, s, e):
    edge = e - s
    t = np.clip(_dot(p - s, edge) / np.maximum(_dot(edge, edge), 1e-300), 0.0, 1.0)
    r = p - s - t[..., None] * edge
    return np.sqrt(_dot(r, r))


def patch_distance(p, quads):
    a, b, c, d = (quads[..., k, :] for k in range(4))
    eu, ev, w = b - a, d - a, a - b + c - d
    u = np.full(p.shape[:-1], 0.5)
    v = np.full(p.shape[:-1], 0.5)
    for _ in range(NEWTON_ITERATIONS):
        x_u = eu + v[..., None] * w
        x_v = ev + u[..., None] * w
        r = a + u[..., None] * eu + v[..., None] * ev + (u * v)[..., None] * w - p
        g_u, g_v = _dot(r, x_u), _dot(r, x_v)
        h_uu, h_vv = _dot(x_u, x_u), _dot(x_v, x_v)
        h_uv = _dot(x_u, x_v) + _dot(r, w)
        det = h_uu * h_vv - h_uv * h_uv
        ok = np.abs(det) > 1e-300
        safe = np.where(ok, det, 1.0)
        u = np.where(ok, u - (h_vv * g_u - h_uv * g_v) / safe, u)
        v = np.where(ok, v - (h_uu * g_v - h_uv * g_u) / safe, v)
        u, v = np.clip(u, -0.5, 1.5), np.clip(v, -0.5, 1.5)
    r = a + u[..., None] * eu + v[..., None] * ev + (u * v)[..., None] * w - p
    inside = (u >= 0.0) & (u <= 1.0) & (v >= 0.0) & (v <= 1.0)
    best = np.where(inside, np.sqrt(_dot(r, r)), np.inf)
    for s, e in ((a, b), (b, c), (c, d), (d, a)):
        best = np.minimum(best, _segment_distance(p, s, e))
    return best


def wall_distance3d(block: Block3, quads: WallQuads, centres: np.ndarray, chunk: int = 256) -> np.ndarray:
    """Distance from every cell centre of ``block`` to the nearest wall face."""
    if not len(quads.corners):
        return np.full(block.shape, np.inf)
    q = quads.corners
    k = min(CANDIDATES, q.shape[0])
    points = np.moveaxis(centres, 0, -1).reshape(-1, 3)
    out = np.empty(len(points))
    for s in range(0, len(points), chunk):
        p = points[s:s + chunk, None, :]
        tri = np.minimum(triangle_distance(p, q[None, :, 0], q[None, :, 1], q[None, :, 2]),
                         triangle_distance(p, q[None, :, 0], q[None, :, 2], q[None, :, 3]))
        nearest = np.argsort(tri, axis=1, kind="stable")[:, :k]
        out[s:s + chunk] = patch_distance(p, q[nearest]).min(axis=1)
    return out.reshape(block.shape)
