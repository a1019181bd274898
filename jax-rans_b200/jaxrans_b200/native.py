"""The C-ABI library: loading it, and a plan object over ``jr_plan``.

The library (``lib/libjaxrans_b200.so``, built by ``jaxrans_b200.build``) holds the
sm_100a kernels.  There is no CPU fallback: without the library, or without a CUDA
device, every entry point raises.  Device buffers are passed as raw pointers; the
helpers here take ``torch`` CUDA tensors (torch is only the allocator) or NumPy arrays,
which are copied to the device and back.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .config import FlowConditions, ImplicitConfig, NumericsConfig, freestream_primitive
from .plan import Plan

LIB_NAME = "libjaxrans_b200.so"
LIB_PATH = Path(__file__).resolve().parent / "lib" / LIB_NAME

FLUX_CODES = {"hllc": 0, "roe": 1}
LIMITER_CODES = {"none": 0, "minmod": 1, "van_albada": 2, "van_albada_smooth": 3}
FAR_FIELD_CODES = {"characteristic": 0, "characteristic_point_vortex": 1}

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


class PlanDesc(C.Structure):
    """``jr_plan_desc`` (include/jaxrans_b200.h)."""

    _fields_ = [
        ("NI", C.c_int32), ("NJ", C.c_int32), ("nvar", C.c_int32),
        ("interior", _u8p), ("volume", _f64p), ("faces_i", _f64p), ("faces_j", _f64p),
        ("centres", _f64p), ("distance", _f64p), ("neighbours", _i32p),
        ("n_ghost", C.c_int32 * 2), ("ghost", _i32p * 2), ("source", _i32p * 2), ("kind", _i32p * 2),
        ("geom", _f64p * 2),
        ("n_walls", C.c_int32), ("wall_cell", _i32p), ("wall_family", _i32p), ("wall_face", _i32p),
        ("wall_into", _f64p), ("wall_mid", _f64p),
        ("n_chains", C.c_int32), ("chain_L", C.c_int32), ("chain_cells", _i32p), ("chain_len", _i32p),
        ("chain_up_face", _i32p), ("chain_up_sign", _i32p), ("chain_down_face", _i32p),
        ("chain_down_sign", _i32p),
        ("gamma", C.c_double), ("mu_inf", C.c_double), ("sutherland", C.c_double), ("c_cr1", C.c_double),
        ("kappa", C.c_double),
        ("flux", C.c_int32), ("limiter", C.c_int32), ("far_field", C.c_int32),
        ("q_inf", C.c_double * 5), ("quarter_chord", C.c_double * 2),
        ("cfl", C.c_double), ("cfl_max", C.c_double), ("cfl_growth", C.c_double), ("cfl_cutback", C.c_double),
        ("cfl_min", C.c_double), ("krylov_tol", C.c_double), ("krylov_success", C.c_double),
        ("max_relative_update", C.c_double),
        ("krylov_subspace", C.c_int32), ("krylov_restarts", C.c_int32), ("preconditioner", C.c_int32),
        ("precision", C.c_int32),
        ("force_length", C.c_double), ("moment_centre", C.c_double * 2),
    ]


EXPORTS = ("jr_plan_create", "jr_plan_destroy", "jr_last_error", "jr_plan_sizes", "jr_plan_stream",
           "jr_synchronize", "jr_residual", "jr_jvp", "jr_wave_speeds", "jr_precond_factor", "jr_precond_apply",
           "jr_state_set", "jr_state_get", "jr_state_device", "jr_newton_steps", "jr_newton_steps_async",
           "jr_forces", "jr_state_set_device", "jr_graph_kernels", "jr_time_kernels", "jr_plan_set_stream",
           "jr_batch_create", "jr_plan_cases", "jr_case_sizes", "jr_case_enable", "jr_case_set_inflow",
           "jr_case_state_set", "jr_case_state_get", "jr_residual_noalloc", "jr_case_load",
           "jr_launch_count", "jr_autotune", "jr_line_schedule", "jr_wait_limit_check", "jr_wall_loads",
           "jr_plan3d_create", "jr_plan3d_destroy", "jr_residual3d", "jr_jvp3d", "jr_wave_speeds3d",
           "jr_precondition3d", "jr_newton_steps3d", "jr_forces3d", "jr_wall_distance3d",
           "jr_launches3d", "jr_wall_loads3d", "jr_monitor_set", "jr_monitor_blocks", "jr_monitor_get", "jr_norm",
           "jr_time_kernels3d")

TIMED_KERNELS = ("residual_tile", "jvp_tile", "ghosts_tangent", "line_apply", "line_factor", "cgs2_full_basis",
                 "linearize")

_LIB = None


# return codes and status bits of the C ABI (include/jaxrans_b200.h)
JR_OK, JR_EINVAL, JR_ENOMEM, JR_ECUDA, JR_EMISMATCH, JR_ETIMEOUT = 0, 1, 2, 3, 4, 5
JR_STATUS_NONFINITE, JR_STATUS_REJECTED, JR_STATUS_GMRES_BREAKDOWN, JR_STATUS_WAIT_LIMIT = 1, 2, 4, 8


class NativeError(RuntimeError):
    """A failure reported by the C-ABI library (``code``: its return code)."""

    def __init__(self, message: str, code: int = JR_ECUDA):
        super().__init__(message)
        self.code = code


class DeviceTimeout(NativeError):
    """A device-side wait gave up (``JR_ETIMEOUT``): a case's status has
    ``JR_STATUS_WAIT_LIMIT``; its last steps are not to be trusted."""


def load_library(path: Path | None = None) -> C.CDLL:
    """The C-ABI library; raises if it has not been built."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    path = Path(path) if path is not None else LIB_PATH
    if not path.is_file():
        raise NativeError(f"{path} is missing: build it with `python -m jaxrans_b200.build` "
                          f"(there is no CPU fallback)")
    lib = C.CDLL(str(path))
    vp = C.c_void_p
    sig = {
        "jr_plan_create": (C.c_int, [C.POINTER(PlanDesc), C.POINTER(vp)]),
        "jr_plan_destroy": (C.c_int, [vp]),
        "jr_last_error": (C.c_char_p, []),
        "jr_plan_sizes": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "jr_plan_stream": (vp, [vp]),
        "jr_synchronize": (C.c_int, [vp]),
        "jr_residual": (C.c_int, [vp, vp, vp, C.c_int]),
        "jr_residual_noalloc": (C.c_int, [vp, vp, vp, C.c_int]),
        "jr_jvp": (C.c_int, [vp, vp, vp, vp]),
        "jr_wave_speeds": (C.c_int, [vp, vp, vp]),
        "jr_precond_factor": (C.c_int, [vp, vp, C.c_double]),
        "jr_precond_apply": (C.c_int, [vp, vp, vp]),
        "jr_state_set": (C.c_int, [vp, vp, C.c_double, C.c_double]),
        "jr_state_get": (C.c_int, [vp, vp, _f64p, _f64p, _i32p]),
        "jr_state_device": (vp, [vp]),
        "jr_newton_steps": (C.c_int, [vp, C.c_int32, vp]),
        "jr_newton_steps_async": (C.c_int, [vp, C.c_int32, vp]),
        "jr_forces": (C.c_int, [vp, vp, vp]),
        "jr_state_set_device": (C.c_int, [vp, vp, C.c_double, C.c_double]),
        "jr_graph_kernels": (C.c_int, [vp, C.POINTER(C.c_int64)]),
        "jr_launch_count": (C.c_int, [vp, C.POINTER(C.c_int64)]),
        "jr_autotune": (C.c_int, [vp, C.c_int32, _i32p]),
        "jr_line_schedule": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32]),
        "jr_wait_limit_check": (C.c_int, [C.c_int32, _i32p]),
        "jr_plan3d_create": (C.c_int, [vp, C.POINTER(vp)]),
        "jr_plan3d_destroy": (C.c_int, [vp]),
        "jr_residual3d": (C.c_int, [vp, vp, vp, C.c_int32]),
        "jr_jvp3d": (C.c_int, [vp, vp, vp, vp]),
        "jr_wave_speeds3d": (C.c_int, [vp, vp, vp]),
        "jr_precondition3d": (C.c_int, [vp, vp, C.c_double, vp, vp]),
        "jr_newton_steps3d": (C.c_int, [vp, vp, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), vp]),
        "jr_forces3d": (C.c_int, [vp, vp, C.c_double, C.c_double, vp, vp]),
        "jr_wall_distance3d": (C.c_int, [vp, C.c_int64, vp, C.c_int32, vp]),
        "jr_launches3d": (C.c_int, [vp]),
        "jr_time_kernels3d": (C.c_int, [vp, vp, C.c_int32, _f64p]),
        "jr_wall_loads3d": (C.c_int, [vp, vp, vp]),
        "jr_wall_loads": (C.c_int, [vp, vp, vp]),
        "jr_time_kernels": (C.c_int, [vp, C.c_int32, _f64p]),
        "jr_plan_set_stream": (C.c_int, [vp, vp]),
        "jr_batch_create": (C.c_int, [C.POINTER(PlanDesc), C.c_int32, C.POINTER(vp)]),
        "jr_plan_cases": (C.c_int, [vp]),
        "jr_case_sizes": (C.c_int, [vp, C.c_int32] + [C.POINTER(C.c_int64)] * 4),
        "jr_case_enable": (C.c_int, [vp, C.c_int32, C.c_int32]),
        "jr_case_set_inflow": (C.c_int, [vp, C.c_int32, _f64p]),
        "jr_case_load": (C.c_int, [vp, C.c_int32, C.POINTER(PlanDesc)]),
        "jr_case_state_set": (C.c_int, [vp, C.c_int32, vp, C.c_double, C.c_double]),
        "jr_case_state_get": (C.c_int, [vp, C.c_int32, vp, _f64p, _f64p, _i32p]),
        "jr_monitor_set": (C.c_int, [vp, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32]),
        "jr_monitor_blocks": (C.c_int, [vp, C.c_int32, C.c_int32, vp]),
        "jr_monitor_get": (C.c_int, [vp, C.c_int32, _i32p, _i32p, _f64p, vp]),
        "jr_norm": (C.c_int, [vp, vp, C.c_int32, _f64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    if path == LIB_PATH:
        _LIB = lib
    return lib


def _check(lib, rc: int, what: str) -> None:
    if rc != 0:
        msg = lib.jr_last_error().decode(errors="replace")
        cls = DeviceTimeout if rc == JR_ETIMEOUT else NativeError
        raise cls(f"{what} failed (code {rc}): {msg}", rc)


def _ptr(a: np.ndarray, kind):
    return a.ctypes.data_as(kind)


def fill_desc(d: PlanDesc, plan: Plan, flow: FlowConditions, numerics: NumericsConfig, implicit: ImplicitConfig,
              force_length: float, moment_centre, keep: list) -> None:
    """``d`` for one case; the arrays it points into are appended to ``keep``."""
    nvar = flow.nvar
    if nvar == 5 and plan.distance is None:
        raise ValueError("the SA model needs the plan's wall distance (build_plan(..., with_distance=True))")

    def arr(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a

    d.NI, d.NJ, d.nvar = plan.NI, plan.NJ, nvar
    d.interior = _ptr(arr(plan.interior, np.uint8), _u8p)
    d.volume = _ptr(arr(plan.volume, np.float64), _f64p)
    d.faces_i = _ptr(arr(plan.faces_i, np.float64), _f64p)
    d.faces_j = _ptr(arr(plan.faces_j, np.float64), _f64p)
    d.centres = _ptr(arr(plan.centres, np.float64), _f64p)
    d.distance = _ptr(arr(plan.distance, np.float64), _f64p) if (nvar == 5) else _f64p()
    d.neighbours = _ptr(arr(plan.neighbours, np.int32), _i32p)
    for s, st in enumerate(plan.stages):
        d.n_ghost[s] = len(st.ghost)
        d.ghost[s] = _ptr(arr(st.ghost, np.int32), _i32p)
        d.source[s] = _ptr(arr(st.source, np.int32), _i32p)
        d.kind[s] = _ptr(arr(st.kind, np.int32), _i32p)
        d.geom[s] = _ptr(arr(np.stack([st.normal[0], st.normal[1], st.midpoint[0], st.midpoint[1]], axis=1),
                             np.float64), _f64p)
    W = plan.walls
    d.n_walls = len(W.cell)
    d.wall_cell = _ptr(arr(W.cell, np.int32), _i32p)
    d.wall_family = _ptr(arr(W.family, np.int32), _i32p)
    d.wall_face = _ptr(arr(W.face, np.int32), _i32p)
    d.wall_into = _ptr(arr(W.into_fluid, np.float64), _f64p)
    d.wall_mid = _ptr(arr(W.mid if len(W.cell) else np.zeros((0, 2)), np.float64), _f64p)
    ch = plan.chains
    d.n_chains, d.chain_L = ch.cells.shape
    d.chain_cells = _ptr(arr(ch.cells.T, np.int32), _i32p)
    d.chain_len = _ptr(arr(ch.lengths, np.int32), _i32p)
    d.chain_up_face = _ptr(arr(ch.up_face.T, np.int32), _i32p)
    d.chain_up_sign = _ptr(arr(ch.up_sign.T, np.int32), _i32p)
    d.chain_down_face = _ptr(arr(ch.down_face.T, np.int32), _i32p)
    d.chain_down_sign = _ptr(arr(ch.down_sign.T, np.int32), _i32p)
    d.gamma = flow.gamma
    d.mu_inf = 0.0 if flow.inviscid else flow.mu_inf
    d.sutherland = -1.0 if flow.sutherland_ratio is None else flow.sutherland_ratio
    d.c_cr1 = 0.3 if flow.turbulence == "sa_noft2_qcr" else 0.0
    d.kappa = numerics.kappa
    d.flux = FLUX_CODES[numerics.flux]
    d.limiter = 4 if numerics.kappa != 0.0 else LIMITER_CODES[numerics.limiter]
    d.far_field = FAR_FIELD_CODES[numerics.far_field]
    for k, v in enumerate(freestream_primitive(flow)):
        d.q_inf[k] = v
    d.quarter_chord[0], d.quarter_chord[1] = plan.quarter_chord
    imp = implicit
    d.cfl, d.cfl_max, d.cfl_growth = imp.cfl, imp.cfl_max, imp.cfl_growth
    d.cfl_cutback, d.cfl_min = imp.cfl_cutback, imp.cfl_min
    d.krylov_tol, d.krylov_success = imp.krylov_tol, imp.krylov_success
    d.max_relative_update = -1.0 if imp.max_relative_update is None else imp.max_relative_update
    d.krylov_subspace, d.krylov_restarts = imp.krylov_subspace, imp.krylov_restarts
    d.preconditioner = {"none": 0, "line_j": 1, "line_j_coupled": 2}[imp.preconditioner]
    d.precision = 1 if imp.precision == "mixed" else 0
    d.force_length = force_length
    d.moment_centre[0], d.moment_centre[1] = moment_centre[0], moment_centre[1]


class DevicePlan:
    """Cases on the device: ``jr_plan`` with their tables, buffers and state.

    ``DevicePlan(plan, flow, ...)`` is one case; ``DevicePlan.batch(plans, flows, ...)``
    advances several at once (a polar: one grid, one flow per angle).  For a single case
    fields have the case's shape ``(nvar, NI, NJ)``; for a batch, arrays that span the
    batch are flat, the cases back to back (``offsets``), and the ``case_*`` methods
    read or write one case."""

    def __init__(self, plan: Plan, flow: FlowConditions, numerics: NumericsConfig,
                 implicit: ImplicitConfig | None = None, force_length: float = 1.0,
                 moment_centre=(0.25, 0.0), library: Path | None = None):
        self._create([plan], [flow], numerics, implicit, force_length, moment_centre, library)

    @classmethod
    def batch(cls, plans, flows, numerics: NumericsConfig, implicit: ImplicitConfig | None = None,
              force_length: float = 1.0, moment_centre=(0.25, 0.0), library: Path | None = None) -> "DevicePlan":
        if isinstance(plans, Plan):
            plans = [plans] * len(flows)
        if len(plans) != len(flows) or not flows:
            raise ValueError("a batch needs one plan per flow, and at least one case")
        self = cls.__new__(cls)
        self._create(list(plans), list(flows), numerics, implicit, force_length, moment_centre, library)
        return self

    def _create(self, plans, flows, numerics, implicit, force_length, moment_centre, library):
        """``numerics``, ``implicit``, ``force_length`` and ``moment_centre`` are one for
        every case or a list with one per case."""
        n = len(plans)

        def per_case(x, single=lambda x: False):
            return list(x) if isinstance(x, (list, tuple)) and not single(x) else [x] * n

        nums = per_case(numerics)
        imps = [i or ImplicitConfig() for i in per_case(implicit)]
        lengths = per_case(force_length)
        centres = per_case(moment_centre, lambda x: len(x) in (2, 3) and np.isscalar(x[0]))
        self.lib = load_library(library)
        self.plans, self.flows, self.numerics = plans, flows, nums[0]
        self.plan, self.flow = plans[0], flows[0]
        self.implicit = imps[0]
        keep: list = []
        descs = (PlanDesc * n)()
        for k, (plan, flow) in enumerate(zip(plans, flows)):
            fill_desc(descs[k], plan, flow, nums[k], imps[k], lengths[k], centres[k], keep)
        handle = C.c_void_p()
        if len(plans) == 1:
            _check(self.lib, self.lib.jr_plan_create(descs, C.byref(handle)), "jr_plan_create")
        else:
            _check(self.lib, self.lib.jr_batch_create(descs, len(plans), C.byref(handle)), "jr_batch_create")
        self.handle = handle
        self.n_cases = len(plans)
        self.nvar = flows[0].nvar
        self.shapes = [(self.nvar, p.NI, p.NJ) for p in plans]
        self.shape = self.shapes[0]
        sizes = [self.nvar * p.NI * p.NJ for p in plans]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.n_vec = int(self.offsets[-1])
        faces = [(p.NI + 1) * p.NJ + p.NI * (p.NJ + 1) for p in plans]
        self.face_offsets = np.concatenate([[0], np.cumsum(faces)]).astype(np.int64)
        self.n_faces = int(self.face_offsets[-1])

    def _field_shape(self):
        return self.shape if self.n_cases == 1 else (self.n_vec,)

    # -- lifetime ---------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.jr_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- device buffers ---------------------------------------------------------------
    @staticmethod
    def _device(a):
        """A CUDA float64 tensor of ``a``; torch's stream is drained so the plan's
        own stream sees the data."""
        import torch
        if isinstance(a, torch.Tensor):
            if a.device.type != "cuda" or a.dtype != torch.float64 or not a.is_contiguous():
                raise ValueError("device buffers must be contiguous float64 CUDA tensors")
            t = a
        else:
            t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
        torch.cuda.synchronize()
        return t

    @staticmethod
    def _like_input(x, t):
        import torch
        return t if isinstance(x, torch.Tensor) else t.cpu().numpy()

    def _empty(self, n):
        import torch
        return torch.empty(n, dtype=torch.float64, device="cuda")

    def sync(self) -> None:
        _check(self.lib, self.lib.jr_synchronize(self.handle), "jr_synchronize")

    # -- entry points --------------------------------------------------------------------
    def residual(self, U, first_order: bool = False):
        u = self._device(U)
        out = self._empty(self._field_shape())
        _check(self.lib, self.lib.jr_residual(self.handle, u.data_ptr(), out.data_ptr(), int(first_order)),
               "jr_residual")
        self.sync()
        return self._like_input(U, out)

    def jvp(self, U, v):
        u, t = self._device(U), self._device(v)
        out = self._empty(self._field_shape())
        _check(self.lib, self.lib.jr_jvp(self.handle, u.data_ptr(), t.data_ptr(), out.data_ptr()), "jr_jvp")
        self.sync()
        return self._like_input(U, out)

    def norm(self, R, variable: int = 0):
        """The volume-weighted L2 norm of row ``variable`` over the block cells, on the
        device: a float, or one per case for a batch."""
        keep = self._device(R)
        out = np.empty(self.n_cases)
        _check(self.lib, self.lib.jr_norm(self.handle, keep.data_ptr(), int(variable), _ptr(out, _f64p)), "jr_norm")
        return float(out[0]) if self.n_cases == 1 else out

    def wave_speeds(self, U):
        u = self._device(U)
        out = self._empty(self.n_faces)
        _check(self.lib, self.lib.jr_wave_speeds(self.handle, u.data_ptr(), out.data_ptr()), "jr_wave_speeds")
        self.sync()
        lam = self._like_input(U, out)
        if self.n_cases > 1:
            return lam
        nfi = (self.plan.NI + 1) * self.plan.NJ
        return (lam[:nfi].reshape(self.plan.NI + 1, self.plan.NJ),
                lam[nfi:].reshape(self.plan.NI, self.plan.NJ + 1))

    def precondition(self, U, cfl: float, r):
        u, rr = self._device(U), self._device(r)
        out = self._empty(self._field_shape())
        _check(self.lib, self.lib.jr_precond_factor(self.handle, u.data_ptr(), float(cfl)), "jr_precond_factor")
        _check(self.lib, self.lib.jr_precond_apply(self.handle, rr.data_ptr(), out.data_ptr()), "jr_precond_apply")
        self.sync()
        return self._like_input(r, out)

    def set_state(self, U=None, cfl: float | None = None, residual_norm: float = float("inf")) -> None:
        """Every case's state (``U``: the case's shape, or the batch back to back) with one
        CFL and previous |R|."""
        cfl = self.implicit.cfl if cfl is None else cfl
        ptr = None
        if U is not None:
            U = np.ascontiguousarray(U, dtype=np.float64)
            if U.size != self.n_vec or (self.n_cases == 1 and U.shape != self.shape):
                raise ValueError(f"state must be {self._field_shape()}, got {U.shape}")
            ptr = U.ctypes.data
        _check(self.lib, self.lib.jr_state_set(self.handle, ptr, float(cfl), float(residual_norm)), "jr_state_set")

    def get_state(self):
        """``(U, cfl, |R| before the last accepted step, status)``; for a batch U is flat
        and the scalars are arrays over the cases."""
        U = np.empty(self._field_shape())
        cfl, res = np.empty(self.n_cases), np.empty(self.n_cases)
        status = np.empty(self.n_cases, dtype=np.int32)
        _check(self.lib, self.lib.jr_state_get(self.handle, U.ctypes.data, _ptr(cfl, _f64p), _ptr(res, _f64p),
                                                _ptr(status, _i32p)), "jr_state_get")
        if self.n_cases == 1:
            return U, float(cfl[0]), float(res[0]), int(status[0])
        return U, cfl, res, status

    def case_state(self, k: int):
        """Case k: ``(U (nvar, NI, NJ), cfl, |R|, status)``."""
        U = np.empty(self.shapes[k])
        cfl, res, status = C.c_double(), C.c_double(), C.c_int32()
        _check(self.lib, self.lib.jr_case_state_get(self.handle, int(k), U.ctypes.data, C.byref(cfl), C.byref(res),
                                                     C.byref(status)), "jr_case_state_get")
        return U, cfl.value, res.value, status.value

    def set_case_state(self, k: int, U=None, cfl: float | None = None, residual_norm: float = float("inf")) -> None:
        cfl = self.implicit.cfl if cfl is None else cfl
        ptr = None
        if U is not None:
            U = np.ascontiguousarray(U, dtype=np.float64)
            if U.shape != self.shapes[k]:
                raise ValueError(f"case {k} state must be {self.shapes[k]}, got {U.shape}")
            ptr = U.ctypes.data
        _check(self.lib, self.lib.jr_case_state_set(self.handle, int(k), ptr, float(cfl), float(residual_norm)),
               "jr_case_state_set")

    def enable(self, k: int, enabled: bool = True) -> None:
        _check(self.lib, self.lib.jr_case_enable(self.handle, int(k), int(bool(enabled))), "jr_case_enable")

    def load_case(self, k: int, plan: Plan, flow: FlowConditions, numerics: NumericsConfig,
                  implicit: ImplicitConfig | None = None, force_length: float = 1.0,
                  moment_centre=(0.25, 0.0)) -> None:
        """Slot k takes a new case of the same shape (grid size and topology); its state
        is set afterwards (``set_case_state``)."""
        keep: list = []
        d = PlanDesc()
        fill_desc(d, plan, flow, numerics, implicit or self.implicit, force_length, moment_centre, keep)
        _check(self.lib, self.lib.jr_case_load(self.handle, int(k), C.byref(d)), "jr_case_load")
        self.plans[k], self.flows[k] = plan, flow
        if k == 0:
            self.plan, self.flow = plan, flow

    def set_inflow(self, k: int, q_inf) -> None:
        """Case k's freestream primitives (rho, u, v, p[, nu_hat])."""
        q = np.zeros(5)
        q[: self.nvar] = np.asarray(q_inf, dtype=np.float64)[: self.nvar]
        _check(self.lib, self.lib.jr_case_set_inflow(self.handle, int(k), _ptr(q, _f64p)), "jr_case_set_inflow")

    def newton_steps(self, n: int) -> np.ndarray:
        """|R| before each step: ``(n,)``, or ``(n, n_cases)`` for a batch."""
        hist = np.empty(n if self.n_cases == 1 else (n, self.n_cases))
        _check(self.lib, self.lib.jr_newton_steps(self.handle, int(n), hist.ctypes.data), "jr_newton_steps")
        return hist

    # the exit test on the device (jr_monitor_*): reasons by code
    MONITOR_REASONS = ("running", "converged", "settled", "max_iters", "non_finite", "stalled")
    MONITOR_BLOCKS = 1024

    def monitor_set(self, k: int, tol: float, forces_tol, max_blocks: int, release: bool = True) -> None:
        """Case k's exit test on the device (``jr_monitor_set``); enables the case."""
        ft = -1.0 if forces_tol is None else float(forces_tol)
        _check(self.lib, self.lib.jr_monitor_set(self.handle, int(k), float(tol), ft, int(max_blocks),
                                                 int(bool(release))), "jr_monitor_set")

    def monitor_blocks(self, n_blocks: int, block_iters: int) -> np.ndarray:
        """n_blocks blocks of Newton steps with the exit tests on the device; |R| before
        each step, ``(n_blocks * block_iters, n_cases)``."""
        hist = np.empty((n_blocks * block_iters, self.n_cases))
        _check(self.lib, self.lib.jr_monitor_blocks(self.handle, int(n_blocks), int(block_iters), hist.ctypes.data),
               "jr_monitor_blocks")
        return hist

    def monitor_get(self, k: int):
        """Case k's monitor: ``(reason, blocks, peak, coefficients (blocks, 3))``."""
        reason, blocks, peak = C.c_int32(), C.c_int32(), C.c_double()
        coef = np.empty((self.MONITOR_BLOCKS, 3))
        _check(self.lib, self.lib.jr_monitor_get(self.handle, int(k), C.byref(reason), C.byref(blocks),
                                                 C.byref(peak), coef.ctypes.data), "jr_monitor_get")
        n = min(int(blocks.value), self.MONITOR_BLOCKS)
        return self.MONITOR_REASONS[reason.value], int(blocks.value), peak.value, coef[:n].copy()

    def newton_steps_async(self, n: int, history_device=None) -> None:
        ptr = None if history_device is None else history_device.data_ptr()
        _check(self.lib, self.lib.jr_newton_steps_async(self.handle, int(n), ptr), "jr_newton_steps_async")

    def set_state_device(self, U_device, cfl: float | None = None, residual_norm: float = float("inf")) -> None:
        """The state from a device tensor (no host copy)."""
        cfl = self.implicit.cfl if cfl is None else cfl
        _check(self.lib, self.lib.jr_state_set_device(self.handle, U_device.data_ptr(), float(cfl),
                                                       float(residual_norm)), "jr_state_set_device")

    def kernels_per_step(self) -> int:
        n = C.c_int64()
        _check(self.lib, self.lib.jr_graph_kernels(self.handle, C.byref(n)), "jr_graph_kernels")
        return int(n.value)

    def autotune(self, reps: int = 10) -> dict:
        """Pick the line factor's and line solve's block sizes, and whether the solve
        stages its factor in shared memory, by timing them (results do not depend on the
        choice)."""
        out = np.zeros(3, dtype=np.int32)
        _check(self.lib, self.lib.jr_autotune(self.handle, int(reps), _ptr(out, _i32p)), "jr_autotune")
        return {"line_factor_threads": int(out[0]), "line_apply_threads": int(out[1]),
                "line_apply_stage": int(out[2])}

    def line_schedule(self, factor_threads: int = 128, apply_threads: int = 128, stage: int = 0) -> None:
        """Set the line-solve schedule by hand (``jr_line_schedule``): ``stage`` 0 reads
        the factor from global memory, 1..4 stage it in shared memory from level
        ``stage - 1`` of the longest chain."""
        _check(self.lib, self.lib.jr_line_schedule(self.handle, int(factor_threads), int(apply_threads),
                                                   int(stage)), "jr_line_schedule")

    def launch_count(self) -> int:
        """Kernels launched by this plan's Newton steps so far (skipped cycles not counted)."""
        n = C.c_int64()
        _check(self.lib, self.lib.jr_launch_count(self.handle, C.byref(n)), "jr_launch_count")
        return int(n.value)

    def time_kernels(self, reps: int = 20) -> dict:
        """Average ms per launch of the hot kernels at the current state (CUDA events
        on the plan's stream)."""
        out = np.zeros(len(TIMED_KERNELS))
        _check(self.lib, self.lib.jr_time_kernels(self.handle, int(reps), _ptr(out, _f64p)), "jr_time_kernels")
        return dict(zip(TIMED_KERNELS, out.tolist()))

    def stream_handle(self) -> int:
        return int(self.lib.jr_plan_stream(self.handle) or 0)

    def state_device_ptr(self) -> int:
        return int(self.lib.jr_state_device(self.handle))

    def wall_loads(self, U=None):
        """Per wall face (n_walls, 5): gauge pressure, area vector into the fluid (x, y),
        viscous force (x, y); a list with one array per case for a batch."""
        n = [len(p.walls.cell) for p in self.plans]
        out = np.empty((max(1, sum(n)), 5))
        keep = self._device(U) if U is not None else None
        ptr = None if keep is None else keep.data_ptr()
        _check(self.lib, self.lib.jr_wall_loads(self.handle, ptr, out.ctypes.data), "jr_wall_loads")
        parts = np.split(out[: sum(n)], np.cumsum(n)[:-1])
        return parts[0] if self.n_cases == 1 else parts

    def forces(self, U=None) -> np.ndarray:
        """cl, cd, cm, cd_friction, fx, fy: ``(6,)``, or ``(n_cases, 6)`` for a batch."""
        out = np.empty(6 if self.n_cases == 1 else (self.n_cases, 6))
        ptr = None
        keep = None
        if U is not None:
            keep = self._device(U)
            ptr = keep.data_ptr()
        _check(self.lib, self.lib.jr_forces(self.handle, ptr, out.ctypes.data), "jr_forces")
        return out
