"""The 3D path through the C ABI: a 3D plan's descriptor, its ghost records, and a plan
object with the residual and J.v of one 3D case (``jr_plan3d_*``, ``jr_residual3d``,
``jr_jvp3d``).

The plan (``jaxrans_b200.plan3d``) keeps the reference's ghost stages in gather form
(``src/jaxrans/mesh/atlas3d.py:166-210``: per canvas cell the cell itself, a cell to
copy, or a condition row); the device runs them as records, one per ghost the stage
writes (a later write of the same ghost wins, as in the gather form).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .native import FLUX_CODES, LIMITER_CODES, NativeError, _check, _f64p, _i32p, _u8p, load_library
from .grid3d import KINDS_3D
from .plan3d import Plan3

KIND3 = {k: n + 1 for n, k in enumerate(KINDS_3D)}   # 0: a copy


class Plan3Desc(C.Structure):
    """``jr_plan3d_desc`` (include/jaxrans_b200.h)."""

    _fields_ = [
        ("NI", C.c_int32), ("NJ", C.c_int32), ("NK", C.c_int32), ("nvar", C.c_int32),
        ("interior", _u8p), ("volume", _f64p), ("faces", _f64p * 3), ("centres", _f64p), ("distance", _f64p),
        ("n_stages", C.c_int32), ("stage_records", _i32p),
        ("ghost", _i32p), ("source", _i32p), ("kind", _i32p), ("normal", _f64p),
        ("gamma", C.c_double), ("mu_inf", C.c_double), ("sutherland", C.c_double), ("kappa", C.c_double),
        ("flux", C.c_int32), ("limiter", C.c_int32),
        ("q_inf", C.c_double * 6),
        ("neighbours", _i32p), ("n_chains", C.c_int32), ("chain_L", C.c_int32), ("chain_cells", _i32p),
        ("chain_up_face", _i32p), ("chain_up_sign", _i32p),
        ("cfl_max", C.c_double), ("cfl_growth", C.c_double), ("cfl_cutback", C.c_double), ("cfl_min", C.c_double),
        ("krylov_tol", C.c_double), ("krylov_success", C.c_double), ("max_relative_update", C.c_double),
        ("krylov_subspace", C.c_int32), ("krylov_restarts", C.c_int32), ("preconditioner", C.c_int32),
        ("n_walls", C.c_int32), ("wall_cell", _i32p), ("wall_family", _i32p), ("wall_face", _i32p),
        ("wall_into", _f64p), ("wall_mid", _f64p), ("line_precision", C.c_int32), ("c_cr1", C.c_double),
    ]


@dataclass
class Records:
    """Every stage's ghost records, stage after stage."""

    counts: np.ndarray      # (n_stages,)
    ghost: np.ndarray
    source: np.ndarray
    kind: np.ndarray
    normal: np.ndarray      # (n, 3)


def records_of(plan: Plan3) -> Records:
    """The stages of ``plan`` as records: for each ghost a stage writes, a copy of the cell
    it gathers, or the condition row it gathers (its kind, source cell and normal)."""
    n = plan.n_canvas
    counts, ghost, source, kind, normal = [], [], [], [], []
    for st in plan.stages:
        written = np.flatnonzero(st.index != np.arange(n))
        target = st.index[written]
        copy = target < n
        row = target - n
        kinds = np.zeros(len(written), dtype=np.int32)
        src = np.where(copy, target, 0).astype(np.int64)
        nrm = np.zeros((len(written), 3))
        offset = 0
        for name, cond_source, cond_normal, _ in st.conditions:
            m = (~copy) & (row >= offset) & (row < offset + len(cond_source))
            kinds[m] = KIND3[name]
            src[m] = cond_source[row[m] - offset]
            nrm[m] = cond_normal[:, row[m] - offset].T
            offset += len(cond_source)
        if np.any((~copy) & (row >= offset)):
            raise ValueError("a stage gathers a condition row it does not have")
        counts.append(len(written))
        ghost.append(written)
        source.append(src)
        kind.append(kinds)
        normal.append(nrm)
    return Records(np.array(counts, dtype=np.int32), np.concatenate(ghost).astype(np.int32),
                   np.concatenate(source).astype(np.int32), np.concatenate(kind).astype(np.int32),
                   np.concatenate(normal))


def apply_records(records: Records, q: np.ndarray) -> np.ndarray:
    """The records run on the host as the device runs them (every read of a stage before
    its writes), with copies only: the fill's index logic, for checking ``records_of``."""
    flat = q.reshape(q.shape[0], -1).copy()
    at = 0
    for count in records.counts:
        g, s = records.ghost[at:at + count], records.source[at:at + count]
        new = flat.copy()
        new[:, g] = flat[:, s]
        flat = new
        at += count
    return flat.reshape(q.shape)


def describe(plan: Plan3, q_inf, gamma: float, flux: str, limiter: str, kappa: float = 0.0,
             mu_inf: float | None = None, sutherland: float | None = None, implicit=None, c_cr1: float = 0.0):
    """``(jr_plan3d_desc, arrays it points into)`` for ``plan``, the physics and the
    implicit solver's settings (``config.ImplicitConfig``; its defaults if None); keep
    the arrays alive while the descriptor is used."""
    rec = records_of(plan)
    keep = []

    def arr(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a

    def ptr(a, t):
        return a.ctypes.data_as(t)

    nvar = len(q_inf)
    d = Plan3Desc()
    d.NI, d.NJ, d.NK = plan.shape
    d.nvar = nvar
    d.interior = ptr(arr(plan.interior, np.uint8), _u8p)
    d.volume = ptr(arr(plan.volume, np.float64), _f64p)
    for a in range(3):
        d.faces[a] = ptr(arr(plan.faces[a], np.float64), _f64p)
    d.centres = ptr(arr(plan.centres, np.float64), _f64p)
    d.distance = ptr(arr(plan.distance, np.float64), _f64p) if plan.distance is not None else None
    d.n_stages = len(rec.counts)
    d.stage_records = ptr(arr(rec.counts, np.int32), _i32p)
    d.ghost = ptr(arr(rec.ghost, np.int32), _i32p)
    d.source = ptr(arr(rec.source, np.int32), _i32p)
    d.kind = ptr(arr(rec.kind, np.int32), _i32p)
    d.normal = ptr(arr(rec.normal, np.float64), _f64p)
    d.gamma = gamma
    d.mu_inf = 0.0 if mu_inf is None else mu_inf
    d.sutherland = -1.0 if sutherland is None else sutherland
    d.kappa = kappa
    d.flux = FLUX_CODES[flux]
    d.limiter = 4 if kappa != 0.0 else LIMITER_CODES[limiter]
    for v in range(6):
        d.q_inf[v] = float(q_inf[v]) if v < nvar else 0.0
    d.neighbours = ptr(arr(plan.neighbours, np.int32), _i32p)
    lines = plan.lines
    d.n_chains, d.chain_L = lines.cells.shape
    d.chain_cells = ptr(arr(lines.cells, np.int32), _i32p)
    d.chain_up_face = ptr(arr(lines.up_face, np.int32), _i32p)
    d.chain_up_sign = ptr(arr(lines.up_sign, np.int32), _i32p)
    from .config import ImplicitConfig
    imp = implicit if implicit is not None else ImplicitConfig()
    d.cfl_max, d.cfl_growth, d.cfl_cutback, d.cfl_min = imp.cfl_max, imp.cfl_growth, imp.cfl_cutback, imp.cfl_min
    d.krylov_tol, d.krylov_success = imp.krylov_tol, imp.krylov_success
    d.max_relative_update = -1.0 if imp.max_relative_update is None else imp.max_relative_update
    d.krylov_subspace, d.krylov_restarts = imp.krylov_subspace, imp.krylov_restarts
    d.preconditioner = {"none": 0, "line_j": 1, "line_j_coupled": 2}[imp.preconditioner]
    d.line_precision = 1 if imp.precision == "mixed" else 0
    d.c_cr1 = float(c_cr1)
    W = plan.walls
    d.n_walls = len(W.cell)
    d.wall_cell = ptr(arr(W.cell, np.int32), _i32p)
    d.wall_family = ptr(arr(W.family, np.int32), _i32p)
    d.wall_face = ptr(arr(W.face, np.int32), _i32p)
    d.wall_into = ptr(arr(W.into_fluid, np.float64), _f64p)
    d.wall_mid = ptr(arr(W.quads.corners.mean(axis=1), np.float64), _f64p)
    return d, keep


class DevicePlan3:
    """One 3D case on the device: residual and J.v of canvas fields (``(nvar, NI, NJ,
    NK)`` float64 NumPy arrays in and out)."""

    def __init__(self, plan: Plan3, q_inf, gamma: float, flux: str, limiter: str, kappa: float = 0.0,
                 mu_inf: float | None = None, sutherland: float | None = None, implicit=None, library=None,
                 c_cr1: float = 0.0):
        self.lib = load_library(library)
        self.plan = plan
        self.q_inf, self.gamma, self.flux, self.limiter = np.asarray(q_inf, dtype=np.float64), gamma, flux, limiter
        self.mu_inf, self.sutherland = mu_inf, sutherland
        from .config import ImplicitConfig
        self.implicit = implicit if implicit is not None else ImplicitConfig()
        self.nvar = len(q_inf)
        self.shape = (self.nvar,) + plan.shape
        d, keep = describe(plan, q_inf, gamma, flux, limiter, kappa, mu_inf, sutherland, implicit, c_cr1)
        handle = C.c_void_p()
        _check(self.lib, self.lib.jr_plan3d_create(C.byref(d), C.byref(handle)), "jr_plan3d_create")
        self.handle = handle

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.jr_plan3d_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def _run(self, name, *arrays):
        import torch
        if not torch.cuda.is_available():
            raise NativeError("the 3D path runs on a CUDA device (there is no CPU fallback)")
        ins = [torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda") for a in arrays]
        out = torch.empty(self.shape, dtype=torch.float64, device="cuda")
        return ins, out

    def residual(self, U, first_order: bool = False) -> np.ndarray:
        (u,), out = self._run("jr_residual3d", U)
        _check(self.lib, self.lib.jr_residual3d(self.handle, u.data_ptr(), out.data_ptr(), int(first_order)),
               "jr_residual3d")
        return out.cpu().numpy()

    def jvp(self, U, v) -> np.ndarray:
        (u, t), out = self._run("jr_jvp3d", U, v)
        _check(self.lib, self.lib.jr_jvp3d(self.handle, u.data_ptr(), t.data_ptr(), out.data_ptr()), "jr_jvp3d")
        return out.cpu().numpy()

    def wave_speeds(self, U) -> list:
        """lambda per face family (three arrays of the families' face shapes)."""
        import torch
        (u,), _ = self._run("jr_wave_speeds3d", U)
        shapes = [tuple(n + (a == x) for x, n in enumerate(self.plan.shape)) for a in range(3)]
        out = torch.empty(sum(int(np.prod(s)) for s in shapes), dtype=torch.float64, device="cuda")
        _check(self.lib, self.lib.jr_wave_speeds3d(self.handle, u.data_ptr(), out.data_ptr()), "jr_wave_speeds3d")
        flat, parts, at = out.cpu().numpy(), [], 0
        for s in shapes:
            parts.append(flat[at:at + int(np.prod(s))].reshape(s))
            at += int(np.prod(s))
        return parts

    def newton_steps(self, U, n_steps: int, cfl: float, residual_norm: float = float("inf")):
        """``(U, cfl, |R| before the last accepted step, history)`` after ``n_steps``
        pseudo-transient Newton steps from ``U`` (``jr_newton_steps3d``)."""
        (u,), _ = self._run("jr_newton_steps3d", U)
        c, r = C.c_double(cfl), C.c_double(residual_norm)
        hist = np.zeros(n_steps)
        _check(self.lib, self.lib.jr_newton_steps3d(self.handle, u.data_ptr(), int(n_steps), C.byref(c), C.byref(r),
                                                     hist.ctypes.data), "jr_newton_steps3d")
        return u.cpu().numpy(), c.value, r.value, hist

    def time_kernels(self, U, reps: int = 5) -> dict:
        """Average ms per call at ``U`` (``jr_time_kernels3d``, CUDA events on the plan's
        stream): the residual R2, the J.v of R1 and the line preconditioner."""
        (u,), _ = self._run("jr_time_kernels3d", U)
        ms = np.zeros(3)
        _check(self.lib, self.lib.jr_time_kernels3d(self.handle, u.data_ptr(), int(reps), ms.ctypes.data_as(_f64p)),
               "jr_time_kernels3d")
        return dict(zip(("residual3d", "jvp3d", "line_precondition3d"), ms.tolist()))

    # -- a state kept on the device between calls (the march's blocks)
    def set_state(self, U, cfl: float, residual_norm: float = float("inf")) -> None:
        """Keep ``U`` on the device with the step's CFL and previous |R|."""
        (u,), _ = self._run("set_state", U)
        self._state = [u, float(cfl), float(residual_norm)]

    def get_state(self):
        """``(U, cfl, residual_norm)`` of the kept state."""
        u, cfl, res = self._state
        return u.cpu().numpy(), cfl, res

    def newton_block(self, n_steps: int) -> np.ndarray:
        """``n_steps`` Newton steps on the kept state; |R| before each."""
        u, cfl, res = self._state
        c, r = C.c_double(cfl), C.c_double(res)
        hist = np.zeros(n_steps)
        _check(self.lib, self.lib.jr_newton_steps3d(self.handle, u.data_ptr(), int(n_steps), C.byref(c), C.byref(r),
                                                     hist.ctypes.data), "jr_newton_steps3d")
        self._state = [u, c.value, r.value]
        return hist

    def state_wall_loads(self) -> np.ndarray:
        """Per wall face of the kept state: gauge pressure, area vector into the fluid (3),
        laminar viscous force (3) (``jr_wall_loads3d``)."""
        out = np.zeros((len(self.plan.walls.cell), 7))
        _check(self.lib, self.lib.jr_wall_loads3d(self.handle, self._state[0].data_ptr(), out.ctypes.data),
               "jr_wall_loads3d")
        return out

    def state_forces(self, area: float, length: float = 1.0, centre=(0.25, 0.0, 0.0)) -> np.ndarray:
        """``(cl, cd, cm, cd_friction)`` of the kept state."""
        return self._forces_at(self._state[0], area, length, centre)

    def forces(self, U, area: float, length: float = 1.0, centre=(0.25, 0.0, 0.0)) -> np.ndarray:
        """``(cl, cd, cm, cd_friction)`` at ``U`` (``jr_forces3d``)."""
        (u,), _ = self._run("jr_forces3d", U)
        return self._forces_at(u, area, length, centre)

    def _forces_at(self, u, area, length, centre) -> np.ndarray:
        c = np.ascontiguousarray(centre, dtype=np.float64)
        out = np.zeros(4)
        _check(self.lib, self.lib.jr_forces3d(self.handle, u.data_ptr(), float(area), float(length), c.ctypes.data,
                                               out.ctypes.data), "jr_forces3d")
        return out

    def precondition(self, U, cfl: float, r) -> np.ndarray:
        """z = M^-1 r of line_j at (U, cfl)."""
        (u, rr), out = self._run("jr_precondition3d", U, r)
        _check(self.lib, self.lib.jr_precondition3d(self.handle, u.data_ptr(), float(cfl), rr.data_ptr(),
                                                     out.data_ptr()), "jr_precondition3d")
        return out.cpu().numpy()


def wall_distance_device(points: np.ndarray, faces: np.ndarray, library=None) -> np.ndarray:
    """The distance of every point ``(..., 3)`` to the nearest wall face ``(m, 4, 3)`` on
    the device (``jr_wall_distance3d``)."""
    import torch
    if not torch.cuda.is_available():
        raise NativeError("the device wall distance runs on a CUDA device")
    lib = load_library(library)
    pts = torch.as_tensor(np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3), device="cuda")
    q = torch.as_tensor(np.ascontiguousarray(faces, dtype=np.float64).reshape(-1, 4, 3), device="cuda")
    out = torch.empty(pts.shape[0], dtype=torch.float64, device="cuda")
    _check(lib, lib.jr_wall_distance3d(pts.data_ptr(), int(pts.shape[0]), q.data_ptr(), int(q.shape[0]),
                                       out.data_ptr()), "jr_wall_distance3d")
    return out.cpu().numpy().reshape(np.shape(points)[:-1])
