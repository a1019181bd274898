"""The static plan of a mesh: the canvas the device kernels run on.

Every block, with a ring of ``g = 2`` ghost cells, is packed into one 2D canvas
``(NI, NJ)``; block ``b``'s cell ``(i, j)`` (ghosts included, ``-g <= i < ni+g``)
sits at flat index ``(oi_b + g + i) * NJ + (oj_b + g + j)``.  Fields are stored
variable-major ``(nvar, NI * NJ)`` in FP64.  The plan holds, in NumPy, every
table the kernels read, with the meaning the reference's atlas gives them
(``src/jaxrans/mesh/atlas.py:97-489``):

* the canvas geometry: volumes, face area vectors toward increasing index
  (i-faces ``(2, NI+1, NJ)``, j-faces ``(2, NI, NJ+1)``), cell centres with one
  layer of reflected ghost centres;
* the ghost fill as two gather stages (``j`` sides, then ``i`` sides with the
  corners), each a list of records ``(ghost, source, kind, normal, midpoint)``;
* the neighbour map behind face averages;
* the line chains through a block's own ``j`` cut (the C-grid wake);
* the wall faces, grouped into bodies, and the wall distance.

The layout and the tables are alike in both codes because the device results
are compared with the reference's canvas arrays entry by entry.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .grids import SIDES, OUTWARD, WALL_KINDS, Block, Cut, Patch

G = 2

# Ghost-record kinds (the C-ABI's codes): a copy across a cut, or a condition.
KIND_CODES = {"copy": 0, "slip_wall": 1, "no_slip_wall": 2, "symmetry": 3, "far_field": 4,
              "inflow_total": 5, "outflow_static": 6}


def metrics(x: np.ndarray, y: np.ndarray):
    """``(centres (2, ni, nj), area (ni, nj), faces_i (2, ni+1, nj), faces_j (2, ni, nj+1))``
    from nodes ``(ni+1, nj+1)``: the area is half the cross product of the
    diagonals, a face's vector its edge turned clockwise, so it points toward
    increasing index (``src/jaxrans/mesh/block.py:225-252``)."""
    x1, y1, x2, y2 = x[:-1, :-1], y[:-1, :-1], x[1:, :-1], y[1:, :-1]
    x3, y3, x4, y4 = x[1:, 1:], y[1:, 1:], x[:-1, 1:], y[:-1, 1:]
    d1x, d1y, d2x, d2y = x3 - x1, y3 - y1, x4 - x2, y4 - y2
    area = 0.5 * (d1x * d2y - d1y * d2x)
    centres = np.stack([0.25 * (x1 + x2 + x3 + x4), 0.25 * (y1 + y2 + y3 + y4)])
    ex_i, ey_i = x[:, 1:] - x[:, :-1], y[:, 1:] - y[:, :-1]
    ex_j, ey_j = x[1:, :] - x[:-1, :], y[1:, :] - y[:-1, :]
    return centres, area, np.stack([ey_i, -ex_i]), np.stack([-ey_j, ex_j])


def _extended(a: np.ndarray, g: int) -> np.ndarray:
    """Node array grown by ``g`` linearly extrapolated layers on every side."""
    for axis in (0, 1):
        a = np.moveaxis(a, axis, 0)
        lo = [a[0] - (k + 1) * (a[1] - a[0]) for k in range(g)][::-1]
        hi = [a[-1] + (k + 1) * (a[-1] - a[-2]) for k in range(g)]
        a = np.moveaxis(np.concatenate([np.stack(lo), a, np.stack(hi)]), 0, axis)
    return a


def _interior_cell(side, a, layer, ni, nj):
    return {"j_min": (a, layer), "j_max": (a, nj - 1 - layer),
            "i_min": (layer, a), "i_max": (ni - 1 - layer, a)}[side]


def _ghost_cell(side, a, layer, ni, nj):
    return {"j_min": (a, -1 - layer), "j_max": (a, nj + layer),
            "i_min": (-1 - layer, a), "i_max": (ni + layer, a)}[side]


def _side_faces(block: Block, side: str, faces_i, faces_j):
    """Outward unit normals and midpoints of a side's faces."""
    if side.startswith("j"):
        j = 0 if side == "j_min" else block.nj
        sx, sy = faces_j[0][:, j], faces_j[1][:, j]
        x, y = block.x[:, j], block.y[:, j]
    else:
        i = 0 if side == "i_min" else block.ni
        sx, sy = faces_i[0][i, :], faces_i[1][i, :]
        x, y = block.x[i, :], block.y[i, :]
    length = np.hypot(sx, sy)
    sign = OUTWARD[side]
    return sign * sx / length, sign * sy / length, 0.5 * (x[:-1] + x[1:]), 0.5 * (y[:-1] + y[1:])


@dataclass
class Stage:
    """One gather stage: per ghost, its source cell, the kind (a code of
    ``KIND_CODES``), the outward unit normal and the face midpoint.  All
    sources are read before any ghost of the stage is written."""

    ghost: np.ndarray
    source: np.ndarray
    kind: np.ndarray
    normal: np.ndarray      # (2, n)
    midpoint: np.ndarray    # (2, n)
    order: tuple = ()       # condition kinds in first-seen order (the reference's value layout)


@dataclass
class Chains:
    """Line chains ``(n_lines, L)`` of flat canvas cells, ``-1`` padded, with the
    link faces and outward signs of ``src/jaxrans/mesh/atlas.py:59-76``."""

    cells: np.ndarray
    up_face: np.ndarray
    up_sign: np.ndarray
    down_face: np.ndarray
    down_sign: np.ndarray

    @property
    def lengths(self) -> np.ndarray:
        return (self.cells >= 0).sum(axis=1)


@dataclass
class Walls:
    cell: np.ndarray
    family: np.ndarray
    face: np.ndarray
    into_fluid: np.ndarray
    body: np.ndarray
    a: np.ndarray
    b: np.ndarray

    @property
    def bodies(self) -> int:
        return int(self.body.max()) + 1 if self.body.size else 0

    @property
    def mid(self) -> np.ndarray:
        return 0.5 * (self.a + self.b)


@dataclass
class Plan:
    mesh: list
    g: int
    origins: list
    NI: int
    NJ: int
    interior: np.ndarray          # (NI, NJ) bool
    volume: np.ndarray            # (NI, NJ)
    faces_i: np.ndarray           # (2, NI+1, NJ)
    faces_j: np.ndarray           # (2, NI, NJ+1)
    centres: np.ndarray           # (2, NI+2, NJ+2): one ghost layer beyond the canvas
    stages: list
    neighbours: np.ndarray        # (NI*NJ,)
    chains: Chains
    walls: Walls
    quarter_chord: tuple
    distance: np.ndarray | None = None   # (NI, NJ), 1.0 off the blocks
    extras: dict = field(default_factory=dict)

    @property
    def shape(self) -> tuple[int, int]:
        return (self.NI, self.NJ)

    @property
    def n_canvas(self) -> int:
        return self.NI * self.NJ

    @property
    def cells(self) -> int:
        return int(self.interior.sum())

    def windows(self):
        return [(slice(oi + self.g, oi + self.g + b.ni), slice(oj + self.g, oj + self.g + b.nj))
                for b, (oi, oj) in zip(self.mesh, self.origins)]

    def pack(self, blocks, fill=0.0) -> np.ndarray:
        lead = blocks[0].shape[:-2]
        out = np.full(lead + self.shape, fill, dtype=np.float64)
        for value, (wi, wj) in zip(blocks, self.windows()):
            out[..., wi, wj] = value
        return out

    def unpack(self, canvas: np.ndarray) -> list:
        return [canvas[..., wi, wj] for wi, wj in self.windows()]


def _pack(shapes):
    """Tiles placed side by side along ``i``, the canvas as tall as the tallest."""
    origins, x = [], 0
    for w, _ in shapes:
        origins.append((x, 0))
        x += w
    return origins, (x, max(h for _, h in shapes))


def build_plan(mesh, g: int = G, with_distance: bool = False) -> Plan:
    """Pack ``mesh`` (blocks whose patches carry conditions) and build every table."""
    mesh = list(mesh)
    for block in mesh:
        block.check()
        unset = [s.name for _, s in block.patches() if s.kind is None]
        if unset:
            raise ValueError(f"patch(es) {sorted(set(unset))} have no boundary condition")
    shapes = [(b.ni + 2 * g, b.nj + 2 * g) for b in mesh]
    origins, (NI, NJ) = _pack(shapes)

    def pos(b, i, j):
        oi, oj = origins[b]
        return (oi + g + i) * NJ + (oj + g + j)

    interior = np.zeros((NI, NJ), dtype=bool)
    area = np.ones((NI, NJ))
    li, lj = np.meshgrid(np.arange(NI), np.arange(NJ), indexing="ij")
    xc, yc = 1e3 + 10.0 * li, 1e3 + 10.0 * lj
    fi = np.zeros((2, NI + 1, NJ))
    fj = np.zeros((2, NI, NJ + 1))
    block_faces = []
    for b, block in enumerate(mesh):
        oi, oj = origins[b]
        ti, tj = shapes[b]
        c_t, a_t, fi_t, fj_t = metrics(_extended(block.x, g), _extended(block.y, g))
        area[oi:oi + ti, oj:oj + tj] = np.where(np.abs(a_t) > 1e-300, a_t, 1.0)
        xc[oi:oi + ti, oj:oj + tj], yc[oi:oi + ti, oj:oj + tj] = c_t
        fi[:, oi:oi + ti + 1, oj:oj + tj] = fi_t
        fj[:, oi:oi + ti, oj:oj + tj + 1] = fj_t
        c_b, a_b, fi_b, fj_b = metrics(block.x, block.y)
        block_faces.append((fi_b, fj_b))
        wi = slice(oi + g, oi + g + block.ni)
        wj = slice(oj + g, oj + g + block.nj)
        interior[wi, wj] = True
        area[wi, wj] = a_b
        fi[:, wi.start:wi.stop + 1, wj] = fi_b
        fj[:, wi, wj.start:wj.stop + 1] = fj_b
        xc[wi, wj], yc[wi, wj] = c_b

    def stage(layers: int, sides, corners: bool) -> Stage:
        records: dict[str, list] = {}
        copies = []
        for b, block in enumerate(mesh):
            ni, nj = block.ni, block.nj
            for side in sides:
                segs = block.sides[side]
                n = block.length(side)
                ext = layers if corners else 0
                nx, ny, mx, my = _side_faces(block, side, *block_faces[b])
                for k, seg in enumerate(segs):
                    lo = seg.start - (ext if k == 0 else 0)
                    hi = seg.stop + (ext if k == len(segs) - 1 else 0)
                    for a in range(lo, hi):
                        for layer in range(layers):
                            ghost = pos(b, *_ghost_cell(side, a, layer, ni, nj))
                            if isinstance(seg, Cut):
                                partner = mesh[seg.block]
                                span = partner.length(seg.side)
                                c = layers if (corners and seg.side.startswith("i")) else 0
                                p = min(max(seg.partner(a), -c), span - 1 + c)
                                src = pos(seg.block, *_interior_cell(seg.side, p, layer, partner.ni, partner.nj))
                                copies.append((ghost, src))
                            else:
                                read = layer if seg.kind in (*WALL_KINDS, "symmetry") else 0
                                src = pos(b, *_interior_cell(side, a, read, ni, nj))
                                f = min(max(a, 0), n - 1)
                                records.setdefault(seg.kind, []).append((ghost, src, nx[f], ny[f], mx[f], my[f]))
        order = tuple(records)
        rows = [(gh, s, KIND_CODES["copy"], 0.0, 0.0, 0.0, 0.0) for gh, s in copies]
        for kind in order:
            rows += [(r[0], r[1], KIND_CODES[kind], *r[2:]) for r in records[kind]]
        arr = np.array(rows, dtype=np.float64).reshape(-1, 7)
        return Stage(arr[:, 0].astype(np.int64), arr[:, 1].astype(np.int64), arr[:, 2].astype(np.int32),
                     arr[:, 3:5].T.copy(), arr[:, 5:7].T.copy(), order)

    # Reflected ghost centres (one layer), then the canvas edge copied once more.
    centres = np.stack([xc.ravel(), yc.ravel()])
    for st in (stage(1, ("j_min", "j_max"), False), stage(1, ("i_min", "i_max"), True)):
        centres = reflect(st, centres)
    centres = centres.reshape(2, NI, NJ)
    padded = np.stack([np.pad(c, 1, mode="edge") for c in centres])
    stages = [stage(g, ("j_min", "j_max"), False), stage(g, ("i_min", "i_max"), True)]

    plan = Plan(mesh, g, origins, NI, NJ, interior, area, fi, fj, padded, stages,
                _neighbours(mesh, pos, NI * NJ), _chains(mesh, pos, origins, g, NI, NJ),
                _walls(mesh, pos, origins, g, NI, NJ), (0.25, 0.0))
    plan.quarter_chord = _quarter_chord(plan.walls)
    if with_distance:
        plan.distance = plan.pack(wall_distance(mesh, plan.walls), 1.0)
    return plan


def reflect(stage: Stage, centres: np.ndarray) -> np.ndarray:
    """A stage applied to cell centres ``(2, n)``: copies across cuts,
    reflections through every physical face (``atlas.py:370-378``)."""
    out = centres.copy()
    copy = stage.kind == KIND_CODES["copy"]
    out[:, stage.ghost[copy]] = centres[:, stage.source[copy]]
    cond = ~copy
    x = centres[:, stage.source[cond]]
    n, m = stage.normal[:, cond], stage.midpoint[:, cond]
    d = np.sum((x - m) * n, axis=0)
    out[:, stage.ghost[cond]] = x - 2.0 * d * n
    return out


def _neighbours(mesh, pos, n_canvas: int) -> np.ndarray:
    index = np.arange(n_canvas)
    for b, block in enumerate(mesh):
        for side in SIDES:
            for seg in block.sides[side]:
                for a in range(seg.start, seg.stop):
                    ghost = pos(b, *_ghost_cell(side, a, 0, block.ni, block.nj))
                    if isinstance(seg, Cut):
                        partner = mesh[seg.block]
                        index[ghost] = pos(seg.block, *_interior_cell(seg.side, seg.partner(a), 0,
                                                                      partner.ni, partner.nj))
                    else:
                        index[ghost] = pos(b, *_interior_cell(side, a, 0, block.ni, block.nj))
    return index


def _chains(mesh, pos, origins, g, NI, NJ) -> Chains:
    """Cells linked along ``j``, through a block's own ``j``-side cut, as paths
    walked from their ends (``atlas.py:398-470``)."""

    def jface(b, i, j):
        oi, oj = origins[b]
        return (NI + 1) * NJ + (oi + g + i) * (NJ + 1) + (oj + g + j)

    links: dict[tuple, dict[str, tuple]] = {}

    def link(cell, direction, other, face, sign):
        links.setdefault(cell, {})[direction] = (other, face, sign)

    for b, block in enumerate(mesh):
        ni, nj = block.ni, block.nj
        for i in range(ni):
            for j in range(nj - 1):
                link((b, i, j), "up", (b, i, j + 1), jface(b, i, j + 1), 1)
                link((b, i, j + 1), "down", (b, i, j), jface(b, i, j + 1), -1)
        for side, j, direction, face_j, sign in (("j_min", 0, "down", 0, -1), ("j_max", nj - 1, "up", nj, 1)):
            for seg in block.sides[side]:
                if not isinstance(seg, Cut) or not seg.side.startswith("j") or seg.block != b:
                    continue
                partner = mesh[seg.block]
                for a in range(seg.start, seg.stop):
                    p = seg.partner(a)
                    pj = 0 if seg.side == "j_min" else partner.nj - 1
                    link((b, a, j), direction, (seg.block, p, pj), jface(b, a, face_j), sign)

    def around(cell):
        return [v[0] for v in links.get(cell, {}).values()]

    seen: set = set()
    chains = []
    cells = [(b, i, j) for b, block in enumerate(mesh) for i in range(block.ni) for j in range(block.nj)]
    ends = [c for c in cells if len(around(c)) < 2]
    for start in ends + cells:
        if start in seen:
            continue
        chain, previous, cell = [], None, start
        while cell is not None and cell not in seen:
            seen.add(cell)
            chain.append(cell)
            nxt = [c for c in around(cell) if c != previous and c not in seen]
            previous, cell = cell, (nxt[0] if nxt else None)
        chains.append(chain)
    L = max(len(c) for c in chains)
    shape = (len(chains), L)
    out = {k: np.full(shape, fill, dtype=np.int64) for k, fill in
           (("cells", -1), ("up_face", 0), ("up_sign", 0), ("down_face", 0), ("down_sign", 0))}
    for n, chain in enumerate(chains):
        for k, cell in enumerate(chain):
            out["cells"][n, k] = pos(*cell)
            if k + 1 < len(chain):
                nxt = chain[k + 1]
                for record in links[cell].values():
                    if record[0] == nxt:
                        out["up_face"][n, k], out["up_sign"][n, k] = record[1], record[2]
                for record in links[nxt].values():
                    if record[0] == cell:
                        out["down_face"][n, k], out["down_sign"][n, k] = record[1], record[2]
    return Chains(out["cells"], out["up_face"], out["up_sign"], out["down_face"], out["down_sign"])


def _wall_rows(mesh):
    rows = []
    for k, block in enumerate(mesh):
        for side in SIDES:
            for seg in block.sides[side]:
                if not (isinstance(seg, Patch) and seg.kind in WALL_KINDS):
                    continue
                lo, hi = seg.start, seg.stop + 1
                index = {"j_min": (slice(lo, hi), 0), "j_max": (slice(lo, hi), -1),
                         "i_min": (0, slice(lo, hi)), "i_max": (-1, slice(lo, hi))}[side]
                p = np.stack([block.x[index], block.y[index]], axis=1)
                forward = side in ("j_min", "i_max")
                for n in range(seg.stop - seg.start):
                    a, b = (p[n], p[n + 1]) if forward else (p[n + 1], p[n])
                    rows.append((k, SIDES.index(side), seg.start + n, *a, *b))
    return rows


def _walls(mesh, pos, origins, g, NI, NJ) -> Walls:
    """Wall faces chained into bodies, each closed loop from its trailing edge
    (largest ``x``), bodies by leading-edge ``x`` (``mesh/mesh.py:487-536``)."""
    rows = _wall_rows(mesh)
    if not rows:
        z = np.zeros(0, dtype=np.int64)
        return Walls(z, z, z, np.zeros(0), z, np.zeros((0, 2)), np.zeros((0, 2)))
    rows = np.array(rows)
    a, b = rows[:, 3:5], rows[:, 5:7]
    tol = 1e-3 * np.hypot(*(b - a).T).min()

    def key(p):
        return tuple(np.round(p / tol).astype(np.int64))

    starts = {key(p): n for n, p in enumerate(a)}
    if len(starts) != len(a):
        raise ValueError("two wall faces start at the same node")
    following = np.array([starts.get(key(p), -1) for p in b])
    has_pred = np.zeros(len(a), dtype=bool)
    has_pred[following[following >= 0]] = True
    body = np.full(len(a), -1)
    loops = []
    for start in [*np.flatnonzero(~has_pred), *range(len(a))]:
        if body[start] >= 0:
            continue
        loop, f = [], start
        while f >= 0 and body[f] < 0:
            body[f] = len(loops)
            loop.append(f)
            f = following[f]
        if f == start:
            t = int(np.argmax(a[loop, 0]))
            loop = loop[t:] + loop[:t]
        elif f >= 0:
            raise ValueError("wall faces chain into one another inconsistently")
        loops.append(loop)
    loops.sort(key=lambda lp: a[lp, 0].min())
    order = np.concatenate(loops)
    for n, lp in enumerate(loops):
        body[lp] = n
    cell, family, face, sign = [], [], [], []
    for blk, s, c in zip(rows[order, 0].astype(int), rows[order, 1].astype(int), rows[order, 2].astype(int)):
        block, side = mesh[blk], SIDES[s]
        i, j = _interior_cell(side, c, 0, block.ni, block.nj)
        cell.append(pos(blk, i, j))
        ci, cj = origins[blk][0] + g + i, origins[blk][1] + g + j
        if side.startswith("j"):
            family.append(1)
            face.append(ci * (NJ + 1) + cj + (side == "j_max"))
        else:
            family.append(0)
            face.append((ci + (side == "i_max")) * NJ + cj)
        sign.append(1.0 if side in ("j_min", "i_min") else -1.0)
    return Walls(np.array(cell, dtype=np.int64), np.array(family, dtype=np.int64), np.array(face, dtype=np.int64),
                 np.array(sign), body[order], a[order], b[order])


def _quarter_chord(walls: Walls) -> tuple[float, float]:
    if walls.bodies == 0:
        return (0.25, 0.0)
    best = None
    for k in range(walls.bodies):
        nodes = walls.a[walls.body == k]
        te = nodes[0]
        le = nodes[np.argmax(np.hypot(*(nodes - te).T))]
        chord = np.hypot(*(te - le))
        if best is None or chord > best[0]:
            best = (chord, le[0] + 0.25 * (te[0] - le[0]), le[1] + 0.25 * (te[1] - le[1]))
    return float(best[1]), float(best[2])


def wall_distance(mesh, walls: Walls, chunk: int = 4096) -> list:
    """Exact distance from every cell centre to the nearest wall face: the
    clamped projection on each face (``mesh/mesh.py:539-568``)."""
    if not walls.a.size:
        return [np.full((b.ni, b.nj), np.inf) for b in mesh]
    ax, ay = walls.a.T
    ex, ey = (walls.b - walls.a).T
    length2 = ex ** 2 + ey ** 2
    out = []
    for block in mesh:
        c, _, _, _ = metrics(block.x, block.y)
        px, py = c[0].ravel(), c[1].ravel()
        d = np.empty_like(px)
        for s in range(0, px.size, chunk):
            qx = px[s:s + chunk, None] - ax[None, :]
            qy = py[s:s + chunk, None] - ay[None, :]
            t = np.clip((qx * ex + qy * ey) / length2, 0.0, 1.0)
            d[s:s + chunk] = np.sqrt(np.min((qx - t * ex) ** 2 + (qy - t * ey) ** 2, axis=1))
        out.append(d.reshape(block.ni, block.nj))
    return out


def block_from_record(x: np.ndarray, y: np.ndarray, sides: dict) -> Block:
    """A block from nodes and a JSON-style side record (the golden fixtures' form)."""
    out = {}
    for side in SIDES:
        segs = []
        for rec in sides[side]:
            if rec[0] == "interface":
                segs.append(Cut(int(rec[1]), int(rec[2]), int(rec[3]), rec[4], int(rec[5]), bool(rec[6])))
            else:
                segs.append(Patch(rec[3], int(rec[1]), int(rec[2]), rec[4]))
        out[side] = segs
    return Block(np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64), out)
