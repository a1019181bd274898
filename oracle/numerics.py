"""The residual ``R(U)`` and its exact first-order JVP, restated in NumPy (oracle).

Follows ``src/jaxrans/numerics/residual.py:46-334`` and the modules it calls:
reconstruction (``reconstruction.py:29-80``), limiters (``limiters.py:61-116``),
Riemann fluxes (``riemann.py:47-203``), face gradients (``gradients.py:26-95``),
the SA row (``turbulence.py:38-156``, ``physics/spalart_allmaras.py:66-216``),
the viscous flux (``physics/navier_stokes.py:49-116``) and the ghost fill
(``boundary.py:54-267``).  Everything runs on the canvas of a plan
(``jaxrans_b200.plan``), variable-major ``(nvar, NI, NJ)``.

Complex-safe throughout, for the complex-step JVP (module ``oracle``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

PR_LAM, PR_TURB = 0.72, 0.9
STEP = 1e-100

# --- complex-step primitives with JAX's JVP rules ----------------------------------


def re(x):
    return np.real(x) if np.iscomplexobj(x) else x


def jabs(x):
    return np.where(re(x) >= 0.0, x, -x)


def jmax(a, b):
    a, b = np.asarray(a), np.asarray(b)
    ra, rb = re(a), re(b)
    return np.where(ra > rb, a, np.where(rb > ra, b, 0.5 * (a + b)))


def jmin(a, b):
    a, b = np.asarray(a), np.asarray(b)
    ra, rb = re(a), re(b)
    return np.where(ra < rb, a, np.where(rb < ra, b, 0.5 * (a + b)))


def jhypot(a, b):
    if np.iscomplexobj(a) or np.iscomplexobj(b):
        return np.sqrt(a * a + b * b)
    return np.hypot(a, b)


def dot2(a, b):
    """``a_x b_x + a_y b_y`` in index order (``core/state.py:67-73``)."""
    return a[0] * b[0] + a[1] * b[1]


# --- the model of one case ---------------------------------------------------------


@dataclass
class SAConst:
    """SA-noft2 / SA-neg constants (``physics/spalart_allmaras.py:66-89``)."""

    c_b1: float = 0.1355
    sigma: float = 2.0 / 3.0
    c_b2: float = 0.622
    kappa: float = 0.41
    c_w2: float = 0.3
    c_w3: float = 2.0
    c_v1: float = 7.1
    c_2: float = 0.7
    c_3: float = 0.9
    c_n1: float = 16.0
    r_max: float = 10.0

    @property
    def c_w1(self) -> float:
        return self.c_b1 / self.kappa ** 2 + (1.0 + self.c_b2) / self.sigma


SA = SAConst()


@dataclass
class Model:
    """Everything the residual of one case needs besides the state."""

    plan: object
    q_inf: np.ndarray               # (nvar,) primitive freestream
    gamma: float = 1.4
    flux: str = "hllc"
    limiter: str = "minmod"
    kappa: float = 0.0
    mu_inf: float | None = None     # None: inviscid
    sutherland: float | None = None
    sa: bool = False
    c_cr1: float = 0.0
    far_field: str = "characteristic"
    distance: np.ndarray | None = None   # (NI, NJ)

    @property
    def nvar(self) -> int:
        return 5 if self.sa else 4

    @property
    def viscous(self) -> bool:
        return self.mu_inf is not None

    def mu(self, T):
        """Sutherland's law or a constant (``navier_stokes.py:49-69``)."""
        s = self.sutherland
        if s is None:
            return self.mu_inf
        return self.mu_inf * T * np.sqrt(T) * (1.0 + s) / (T + s)

    @property
    def U0(self) -> np.ndarray:
        return initial_state(self)


# --- state conversions (core/state.py:88-93, residual.py:46-51) --------------------


def prim(U, gamma: float):
    rho = U[0]
    u, v = U[1] / rho, U[2] / rho
    p = (gamma - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v))
    rows = [rho, u, v, p]
    if U.shape[0] > 4:
        rows.append(U[4] / rho)
    return np.stack(rows)


def conservative(q, gamma: float):
    rho, u, v, p = q[0], q[1], q[2], q[3]
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    rows = [rho, rho * u, rho * v, E]
    if q.shape[0] > 4:
        rows.append(rho * q[4])
    return np.stack(rows)


def initial_state(model: Model) -> np.ndarray:
    """The freestream on every canvas cell (``residual.py:245-258``)."""
    q = np.asarray(model.q_inf, dtype=np.float64)
    shape = model.plan.shape
    ones = np.ones(shape)
    rho, u, v, p = q[0], q[1], q[2], q[3]
    E = p / (model.gamma - 1.0) + 0.5 * (rho * ones) * ((u * ones) * (u * ones) + (v * ones) * (v * ones))
    rows = [rho * ones, (rho * ones) * (u * ones), (rho * ones) * (v * ones), E]
    if q.shape[0] > 4:
        rows.append((q[0] * q[4]) * ones)
    return np.stack(rows)


# --- boundary conditions (boundary.py:54-158) ---------------------------------------


def _mirror(u, v, nx, ny):
    vn = u * nx + v * ny
    return u - 2.0 * vn * nx, v - 2.0 * vn * ny


def characteristic(edge, nx, ny, qf, gamma: float):
    """Riemann-invariant far field (``boundary.py:91-122``); ``qf`` the reference
    state per face ``(nvar, n)``."""
    rho_i, u_i, v_i, p_i = edge[0], edge[1], edge[2], edge[3]
    rho_f, u_f, v_f, p_f = qf[0], qf[1], qf[2], qf[3]
    a_i = np.sqrt(gamma * p_i / rho_i)
    a_f = np.sqrt(gamma * p_f / rho_f)
    two = 2.0 / (gamma - 1.0)
    vn_i = u_i * nx + v_i * ny
    vn_f = u_f * nx + v_f * ny
    rp = vn_i + two * a_i
    rm = vn_f - two * a_f
    vn_b = 0.5 * (rp + rm)
    a_b = 0.25 * (gamma - 1.0) * (rp - rm)
    out = re(vn_b) > 0.0
    s_b = np.where(out, p_i / rho_i ** gamma, p_f / rho_f ** gamma)
    tu = np.where(out, u_i - vn_i * nx, u_f - vn_f * nx)
    tv = np.where(out, v_i - vn_i * ny, v_f - vn_f * ny)
    rho_b = (a_b * a_b / (gamma * s_b)) ** (1.0 / (gamma - 1.0))
    p_b = rho_b * a_b * a_b / gamma
    rows = [rho_b, vn_b * nx + tu, vn_b * ny + tv, p_b]
    if edge.shape[0] > 4:
        rows.append(np.where(out, edge[4], qf[4]))
    return np.stack(rows)


def point_vortex(dx, dy, q_inf, gamma: float, circulation):
    """Compressible point vortex plus freestream (``boundary.py:181-212``)."""
    rho_f, u_f, v_f, p_f = q_inf[0], q_inf[1], q_inf[2], q_inf[3]
    a2 = gamma * p_f / rho_f
    speed2 = u_f * u_f + v_f * v_f
    mach2 = speed2 / a2
    alpha = np.arctan2(v_f, u_f)
    r = np.hypot(dx, dy)
    theta = np.arctan2(dy, dx)
    strength = circulation * np.sqrt(1.0 - mach2) / (2.0 * np.pi * r * (1.0 - mach2 * np.sin(theta - alpha) ** 2))
    u = u_f + strength * np.sin(theta)
    v = v_f - strength * np.cos(theta)
    ratio = 1.0 + 0.5 * (gamma - 1.0) * (speed2 - u * u - v * v) / a2
    rho = rho_f * ratio ** (1.0 / (gamma - 1.0))
    p = p_f * ratio ** (gamma / (gamma - 1.0))
    rows = [rho, u, v, p]
    if q_inf.shape[0] > 4:
        rows.append(np.broadcast_to(q_inf[4], np.shape(dx)))
    return np.stack([np.broadcast_to(r_, np.shape(dx)) for r_ in rows])


def wall_values(plan, fields):
    """A per-family canvas face field at every wall face (``atlas.py:153-161``)."""
    W = plan.walls
    out = None
    for a, f in enumerate(fields):
        flat = f.reshape(f.shape[:-2] + (-1,))
        picked = flat[..., np.where(W.family == a, W.face, 0)]
        out = picked if out is None else np.where(W.family == a, picked, out)
    return out


def wall_vectors(plan):
    return plan.walls.into_fluid * wall_values(plan, (plan.faces_i, plan.faces_j))


def circulation(q, model: Model):
    """Kutta-Joukowski circulation of the wall pressure lift (``boundary.py:227-240``)."""
    plan = model.plan
    p = q[3].reshape(-1)[plan.walls.cell] - model.q_inf[3]
    S = wall_vectors(plan)
    fx, fy = -np.sum(p * S[0]), -np.sum(p * S[1])
    u_f, v_f = model.q_inf[1], model.q_inf[2]
    speed = np.hypot(u_f, v_f)
    return (fy * u_f - fx * v_f) / speed / (model.q_inf[0] * speed)


def _condition(kind: int, q, nx, ny, mx, my, model: Model, reference):
    g = model.gamma
    if kind in (1, 3):                        # slip wall / symmetry: mirror the velocity
        u, v = _mirror(q[1], q[2], nx, ny)
        rows = [q[0], u, v, q[3]]
        if q.shape[0] > 4:
            rows.append(-q[4] if kind == 1 else q[4])
        return np.stack(rows)
    if kind == 2:                             # no-slip wall: velocity and scalars reversed
        rows = [q[0], -q[1], -q[2], q[3]]
        if q.shape[0] > 4:
            rows.append(-q[4])
        return np.stack(rows)
    if kind == 4:                             # far field
        return characteristic(q, nx, ny, reference(mx, my, q.shape[0]), g)
    if kind == 5:                             # total-condition inflow (boundary.py:130-147)
        g1 = g - 1.0
        qf = model.q_inf
        t_f = g * qf[3] / qf[0]
        speed_f = np.hypot(qf[1], qf[2])
        t_total = t_f + 0.5 * g1 * speed_f * speed_f
        p_total = qf[3] * (t_total / t_f) ** (g / g1)
        p_b = q[3]
        mach2 = jmax(2.0 / g1 * ((p_total / p_b) ** (g1 / g) - 1.0), 0.0)
        t_b = t_total / (1.0 + 0.5 * g1 * mach2)
        speed = np.sqrt(mach2 * t_b)
        rows = [g * p_b / t_b, speed * qf[1] / speed_f, speed * qf[2] / speed_f, p_b]
        if q.shape[0] > 4:
            rows.append(np.broadcast_to(qf[4], p_b.shape) * np.ones_like(p_b))
        return np.stack(rows)
    if kind == 6:                             # static-pressure outflow
        out = q.copy()
        out[3] = model.q_inf[3]
        return out
    raise ValueError(f"unknown condition code {kind}")


def fill_ghosts(q, model: Model, far_field: str | None = None):
    """Every ghost of a primitive canvas by the plan's two gather stages
    (``boundary.py:257-267``, ``atlas.py:331-367``)."""
    plan = model.plan
    far_field = far_field or model.far_field
    flat = q.reshape(q.shape[0], -1)
    nv = q.shape[0]
    if far_field == "characteristic_point_vortex":
        circ = circulation(q, model)
        xc, yc = plan.quarter_chord

        def reference(mx, my, rows):
            return point_vortex(mx - xc, my - yc, model.q_inf[:rows], model.gamma, circ)
    else:
        def reference(mx, my, rows):
            return np.broadcast_to(model.q_inf[:rows, None], (rows, mx.shape[0]))
    for st in plan.stages:
        new = flat.copy()
        copy = st.kind == 0
        new[:, st.ghost[copy]] = flat[:, st.source[copy]]
        for kind in np.unique(st.kind[~copy]):
            m = st.kind == kind
            src = flat[:, st.source[m]]
            new[:, st.ghost[m]] = _condition(int(kind), src, st.normal[0, m], st.normal[1, m],
                                             st.midpoint[0, m], st.midpoint[1, m], model, reference)[:nv]
        flat = new
    return flat.reshape(q.shape)


# --- limiters and reconstruction (limiters.py:61-116, reconstruction.py:29-80) --------


def limit(a, b, name: str):
    if name == "none":
        return 0.5 * (a + b)
    if name == "minmod":
        return np.where(re(a * b) > 0.0, np.sign(re(a)) * jmin(jabs(a), jabs(b)), 0.0)
    if name == "van_albada":
        same = re(a * b) > 0.0
        denom = np.where(same, a * a + b * b, 1.0)
        return np.where(same, a * b * (a + b) / denom, 0.0)
    if name == "van_albada_smooth":
        e = 1e-12
        return ((b * b + e) * a + (a * a + e) * b) / (a * a + b * b + 2.0 * e)
    raise KeyError(name)


def _windows(padded, g: int, shape, axis: int):
    out = []
    for off in range(4):
        idx = [slice(None), slice(g, g + shape[0]), slice(g, g + shape[1])]
        idx[1 + axis] = slice(g - 2 + off, g - 2 + off + shape[axis] + 1)
        out.append(padded[tuple(idx)])
    return out


def face_states(padded, g, shape, axis, model: Model, first_order: bool):
    q_mm, q_m, q_p, q_pp = _windows(padded, g, shape, axis)
    if first_order:
        return q_m, q_p
    d_minus, d_mid, d_plus = q_m - q_mm, q_p - q_m, q_pp - q_p
    if model.kappa != 0.0:
        lo, hi = 0.25 * (1.0 - model.kappa), 0.25 * (1.0 + model.kappa)
        return q_m + lo * d_minus + hi * d_mid, q_p - lo * d_plus - hi * d_mid
    return q_m + 0.5 * limit(d_minus, d_mid, model.limiter), q_p - 0.5 * limit(d_mid, d_plus, model.limiter)


# --- Riemann fluxes (riemann.py:47-203, physics/euler.py:43-94) ------------------------


def sound(rho, p, g):
    return np.sqrt(g * p / rho)


def normal_flux(q, nx, ny, g):
    rho, u, v, p = q[0], q[1], q[2], q[3]
    vn = u * nx + v * ny
    E = p / (g - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.stack([rho * vn, rho * u * vn + p * nx, rho * v * vn + p * ny, (E + p) * vn])


def roe_average(qL, qR, g):
    rho_l, u_l, v_l, p_l = qL[0], qL[1], qL[2], qL[3]
    rho_r, u_r, v_r, p_r = qR[0], qR[1], qR[2], qR[3]
    h_l = g / (g - 1.0) * p_l / rho_l + 0.5 * (u_l * u_l + v_l * v_l)
    h_r = g / (g - 1.0) * p_r / rho_r + 0.5 * (u_r * u_r + v_r * v_r)
    w = np.sqrt(rho_r / rho_l)
    den = 1.0 + w
    rho = np.sqrt(rho_l * rho_r)
    u = (u_l + w * u_r) / den
    v = (v_l + w * v_r) / den
    H = (h_l + w * h_r) / den
    a2 = (g - 1.0) * (H - 0.5 * (u * u + v * v))
    return rho, u, v, H, np.sqrt(jmax(a2, 1e-30))


def _normal(sx, sy):
    length = np.hypot(sx, sy)
    safe = np.maximum(length, 1e-300)
    return length, sx / safe, sy / safe


def roe_flux(qL, qR, sx, sy, g):
    length, nx, ny = _normal(sx, sy)
    rho, u, v, H, a = roe_average(qL, qR, g)
    vn = u * nx + v * ny
    d_rho, d_p = qR[0] - qL[0], qR[3] - qL[3]
    du, dv = qR[1] - qL[1], qR[2] - qL[2]
    d_vn = du * nx + dv * ny
    dut, dvt = du - d_vn * nx, dv - d_vn * ny
    a2 = a * a
    al_m = (d_p - rho * a * d_vn) / (2.0 * a2)
    al_e = d_rho - d_p / a2
    al_p = (d_p + rho * a * d_vn) / (2.0 * a2)
    lm, l0, lp = jabs(vn - a), jabs(vn), jabs(vn + a)
    kin = 0.5 * (u * u + v * v)
    one = np.ones_like(rho)
    r_m = [one, u - a * nx, v - a * ny, H - a * vn]
    r_e = [one, u, v, kin]
    shear = [np.zeros_like(rho), rho * dut, rho * dvt, rho * (u * dut + v * dvt)]
    r_p = [one, u + a * nx, v + a * ny, H + a * vn]
    diss = [lm * al_m * r_m[k] + l0 * al_e * r_e[k] + l0 * shear[k] + lp * al_p * r_p[k] for k in range(4)]
    central = 0.5 * (normal_flux(qL, nx, ny, g) + normal_flux(qR, nx, ny, g))
    return length * (central - 0.5 * np.stack(diss))


def hllc_flux(qL, qR, sx, sy, g):
    length, nx, ny = _normal(sx, sy)
    rho_l, u_l, v_l, p_l = qL[0], qL[1], qL[2], qL[3]
    rho_r, u_r, v_r, p_r = qR[0], qR[1], qR[2], qR[3]
    vn_l, vn_r = u_l * nx + v_l * ny, u_r * nx + v_r * ny
    a_l, a_r = sound(rho_l, p_l, g), sound(rho_r, p_r, g)
    _, u_ro, v_ro, _, a_ro = roe_average(qL, qR, g)
    vn_ro = u_ro * nx + v_ro * ny
    s_l = jmin(vn_l - a_l, vn_ro - a_ro)
    s_r = jmax(vn_r + a_r, vn_ro + a_ro)
    m_l = rho_l * (s_l - vn_l)
    m_r = rho_r * (s_r - vn_r)
    s_m = (p_r - p_l + m_l * vn_l - m_r * vn_r) / jmin(m_l - m_r, -1e-300)

    def star(rho, u, v, p, vn, s_k, f_k, u_k, wide):
        p_star = p + rho * (vn - s_k) * (vn - s_m)
        rho_star = rho * (s_k - vn) / wide
        e_star = ((s_k - vn) * u_k[3] - p * vn + p_star * s_m) / wide
        us = np.stack([rho_star, rho_star * (u + (s_m - vn) * nx), rho_star * (v + (s_m - vn) * ny), e_star])
        return f_k + s_k * (us - u_k)

    U_l, U_r = conservative(qL[:4], g), conservative(qR[:4], g)
    f_l, f_r = normal_flux(qL, nx, ny, g), normal_flux(qR, nx, ny, g)
    st_l = star(rho_l, u_l, v_l, p_l, vn_l, s_l, f_l, U_l, jmin(s_l - s_m, -1e-300))
    st_r = star(rho_r, u_r, v_r, p_r, vn_r, s_r, f_r, U_r, jmax(s_r - s_m, 1e-300))
    f = np.where(re(s_l) >= 0.0, f_l, np.where(re(s_m) >= 0.0, st_l, np.where(re(s_r) >= 0.0, st_r, f_r)))
    return length * f


# --- gradients and the viscous flux (gradients.py:26-95, navier_stokes.py:86-116) ------


def _corners(a):
    return 0.25 * (a[..., :-1, :-1] + a[..., 1:, :-1] + a[..., :-1, 1:] + a[..., 1:, 1:])


def face_gradients(phi, centres):
    """Diamond gradients ``(2, nphi, face)`` per family from one-ghost-layer fields."""
    shape = (centres.shape[1] - 2, centres.shape[2] - 2)
    xn, pn = _corners(centres), _corners(phi)
    out = []
    for a in range(2):
        def cell(off):
            idx = [slice(1, 1 + n) for n in shape]
            idx[a] = slice(off, off + shape[a] + 1)
            return (slice(None),) + tuple(idx)

        def node(shift):
            idx = []
            for b in range(2):
                start = 0 if b == a else shift
                idx.append(slice(start, start + shape[b] + (b == a)))
            return (slice(None),) + tuple(idx)

        dc = centres[cell(1)] - centres[cell(0)]
        dpc = phi[cell(1)] - phi[cell(0)]
        dn = xn[node(1)] - xn[node(0)]
        dpn = pn[node(1)] - pn[node(0)]
        d1x, d1y, d2x, d2y = dc[0], dc[1], dn[0], dn[1]
        det = d1x * d2y - d2x * d1y
        out.append(np.stack([(dpc * d2y - dpn * d1y) / det, (d1x * dpn - d2x * dpc) / det]))
    return out


def _sides(p1, a):
    """Cells before and after every face of family ``a`` of a one-ghost field."""
    n0, n1 = p1.shape[-2], p1.shape[-1]
    if a == 0:
        return p1[..., 0:n0 - 1, 1:-1], p1[..., 1:n0, 1:-1]
    return p1[..., 1:-1, 0:n1 - 1], p1[..., 1:-1, 1:n1]


def face_avg(p1, a):
    lo, hi = _sides(p1, a)
    return 0.5 * (lo + hi)


def qcr(gv, mu_t, c_cr1):
    """QCR2000 addition to the stress (``spalart_allmaras.py:197-216``)."""
    square = gv[0][0] * gv[0][0] + gv[0][1] * gv[0][1] + gv[1][0] * gv[1][0] + gv[1][1] * gv[1][1]
    pos = re(square) > 0.0
    norm = np.where(pos, np.sqrt(np.where(pos, square, 1.0)), 1.0)
    rot = [[(gv[i][k] - gv[k][i]) / norm for k in range(2)] for i in range(2)]
    div = gv[0][0] + gv[1][1]
    tau = [[mu_t * (gv[i][k] + gv[k][i] - (2.0 / 3.0) * div * (1.0 if i == k else 0.0)) for k in range(2)]
           for i in range(2)]
    prod = [[rot[i][0] * tau[j][0] + rot[i][1] * tau[j][1] for j in range(2)] for i in range(2)]
    return [[-c_cr1 * (prod[i][j] + prod[j][i]) for j in range(2)] for i in range(2)]


def viscous_flux(vel, gv, gt, sx, sy, mu, k, extra=None):
    div = gv[0][0] + gv[1][1]
    ttd = (2.0 / 3.0) * div

    def tau(a, b):
        lin = mu * (2.0 * gv[a][a] - ttd) if a == b else mu * (gv[0][1] + gv[1][0])
        return lin if extra is None else lin + extra[a][b]

    fx = tau(0, 0) * sx + tau(0, 1) * sy
    fy = tau(1, 0) * sx + tau(1, 1) * sy
    energy = (vel[0] * fx + vel[1] * fy) + k * (gt[0] * sx + gt[1] * sy)
    return np.stack([np.zeros_like(energy), fx, fy, energy])


def eddy(rho, nu_tilde, nu):
    """``mu_t = rho nu~ f_v1``, zero where ``nu~ <= 0`` (``spalart_allmaras.py:128-131``)."""
    pos = re(nu_tilde) > 0.0
    chi = np.where(pos, nu_tilde / nu, 0.0)
    chi3 = chi * chi * chi
    return np.where(pos, rho * nu_tilde * (chi3 / (chi3 + SA.c_v1 ** 3)), 0.0)


def temperature(q, g):
    return g * q[3] / q[0]


def viscous_fluxes(p1, centres, faces, model: Model, mu_t=None, grads=None):
    g = model.gamma
    if grads is None:
        phi = np.concatenate([p1[1:3], temperature(p1, g)[None]])
        grads = face_gradients(phi, centres)
    out = []
    for a in range(2):
        lo, hi = _sides(p1, a)
        vel = 0.5 * (lo[1:3] + hi[1:3])
        T = 0.5 * (temperature(lo, g) + temperature(hi, g))
        mu = model.mu(T)
        k = mu / (PR_LAM * (g - 1.0))
        extra = None
        if mu_t is not None:
            mu = mu + mu_t[a]
            k = k + mu_t[a] / (PR_TURB * (g - 1.0))
        G = grads[a]
        gv = [[G[0, 0], G[1, 0]], [G[0, 1], G[1, 1]]]     # gv[comp][dir]
        if mu_t is not None and model.c_cr1:
            extra = qcr(gv, mu_t[a], model.c_cr1)
        out.append(viscous_flux(vel, gv, G[:, 2], faces[a][0], faces[a][1], mu, k, extra))
    return out


# --- the SA row (turbulence.py:56-151, spalart_allmaras.py:119-195) ---------------------


def divergence(fluxes):
    f0, f1 = fluxes
    return (f0[..., 1:, :] - f0[..., :-1, :]) + (f1[..., :, 1:] - f1[..., :, :-1])


def green_gauss(phi_faces, faces, volume):
    return np.stack([divergence([phi_faces[0] * faces[0][c], phi_faces[1] * faces[1][c]]) / volume
                     for c in range(2)])


def vorticity_abs(gx):
    return jabs(gx[0, 1] - gx[1, 0])


def s_tilde(omega, nu_tilde, nu, d):
    chi = nu_tilde / nu
    chi3 = chi * chi * chi
    fv1 = chi3 / (chi3 + SA.c_v1 ** 3)
    fv2 = 1.0 - chi / (1.0 + chi * fv1)
    kd = SA.kappa * d
    s_bar = nu_tilde * fv2 / (kd * kd)
    ordinary = re(s_bar) >= re(-SA.c_2 * omega)
    den = np.where(ordinary, 1.0, (SA.c_3 - 2.0 * SA.c_2) * omega - s_bar)
    clipped = omega + omega * (SA.c_2 ** 2 * omega + SA.c_3 * s_bar) / den
    return np.where(ordinary, omega + s_bar, clipped)


def ipow6(x):
    """``x**6`` as JAX's ``integer_pow`` evaluates it: ``x^2 (x^2)^2``."""
    x2 = x * x
    return x2 * (x2 * x2)


def f_w(r):
    gg = r + SA.c_w2 * (ipow6(r) - r)
    g6 = ipow6(gg)
    c6 = SA.c_w3 ** 6
    return gg * ((1.0 + c6) / (g6 + c6)) ** (1.0 / 6.0)


def r_of(nu_tilde, s_t, d):
    kd = SA.kappa * d
    den = s_t * (kd * kd)
    ok = re(den) > 0.0
    safe = np.where(ok, den, 1.0)
    return np.where(ok, jmin(nu_tilde / safe, SA.r_max), SA.r_max)


def sa_source(nu_tilde, nu, omega, d):
    pos = re(nu_tilde) >= 0.0
    s_t = s_tilde(omega, np.where(pos, nu_tilde, 0.0), nu, d)
    wall = (nu_tilde / d) * (nu_tilde / d)
    production = np.where(pos, SA.c_b1 * s_t, SA.c_b1 * omega) * nu_tilde
    destruction = np.where(pos, SA.c_w1 * f_w(r_of(nu_tilde, s_t, d)), -SA.c_w1) * wall
    return production, destruction


def f_n(nu_tilde, nu):
    pos = re(nu_tilde) >= 0.0
    ratio = nu_tilde / nu
    chi3 = np.where(pos, 0.0, ratio * ratio * ratio)
    return np.where(pos, 1.0, (SA.c_n1 + chi3) / (SA.c_n1 - chi3))


def diffusion(rho, nu_tilde, mu):
    nu = mu / rho
    return (mu + rho * nu_tilde * f_n(nu_tilde, nu)) / SA.sigma


def sa_row(p1, mass, grad_nu, faces, volume, model: Model):
    g, nu_inf = model.gamma, model.mu_inf
    nu_hat = p1[4]
    fl = []
    for a in range(2):
        lo, hi = _sides(nu_hat, a)
        up = np.where(re(mass[a]) > 0.0, lo, hi)
        fa = face_avg(p1, a)
        mu = model.mu(temperature(fa, g))
        coef = diffusion(fa[0], fa[4] * nu_inf, mu)
        fl.append(mass[a] * up - coef * (grad_nu[a][0] * faces[a][0] + grad_nu[a][1] * faces[a][1]))
    cell = p1[:, 1:-1, 1:-1]
    rho = cell[0]
    mu = model.mu(temperature(cell, g))
    vel_faces = [face_avg(p1[1:3], a) for a in range(2)]
    omega = vorticity_abs(green_gauss(vel_faces, faces, volume))
    P, D = sa_source(cell[4] * nu_inf, mu / rho, omega, model.distance)
    grad = green_gauss([face_avg(nu_hat, a) for a in range(2)], faces, volume)
    src = rho * ((P - D) / nu_inf + SA.c_b2 / SA.sigma * nu_inf * (grad[0] * grad[0] + grad[1] * grad[1]))
    return divergence(fl) - src * volume


# --- the residual (residual.py:54-91, 273-334) ----------------------------------------


def net_flux(padded, model: Model, first_order: bool):
    plan = model.plan
    g, gamma = plan.g, model.gamma
    shape = plan.shape
    faces = [plan.faces_i, plan.faces_j]
    flow = padded[:4]
    fluxes = []
    for a in range(2):
        qL, qR = face_states(flow, g, shape, a, model, first_order)
        F = hllc_flux if model.flux == "hllc" else roe_flux
        fluxes.append(F(qL, qR, faces[a][0], faces[a][1], gamma))
    sa = None
    if model.viscous:
        p1 = padded[:, g - 1:padded.shape[1] - (g - 1), g - 1:padded.shape[2] - (g - 1)]
        if not model.sa:
            visc = viscous_fluxes(p1, plan.centres, faces, model)
        else:
            phi = np.concatenate([p1[1:3], temperature(p1, gamma)[None], p1[4][None]])
            grads = face_gradients(phi, plan.centres)
            mu_t = []
            for a in range(2):
                fa = face_avg(p1, a)
                T = temperature(fa, gamma)
                mu_t.append(eddy(fa[0], fa[4] * model.mu_inf, model.mu(T) / fa[0]))
            visc = viscous_fluxes(p1, plan.centres, faces, model, mu_t, grads)
            sa = sa_row(p1, [f[0] for f in fluxes], [G[:, 3] for G in grads], faces, plan.volume, model)
        fluxes = [f - v for f, v in zip(fluxes, visc)]
    R = divergence(fluxes)
    return R if sa is None else np.concatenate([R, sa[None]])


def residual(U, model: Model, first_order: bool = False):
    """``where(interior, net flux, U - U0)`` on the canvas (``residual.py:324-327``)."""
    g = model.plan.g
    q = prim(U, model.gamma)
    filled = fill_ghosts(q, model)
    padded = np.pad(filled, ((0, 0), (g, g), (g, g)), mode="edge")
    R = net_flux(padded, model, first_order)
    return np.where(model.plan.interior, R, U - model.U0)


def jvp(U, v, model: Model, first_order: bool = True):
    """Exact ``dR/dU . v`` by the complex step (module docstring)."""
    return np.imag(residual(U.astype(np.complex128) + 1j * STEP * v, model, first_order)) / STEP


# --- wave speeds and norms (residual.py:127-240, atlas.py:163-183) ----------------------


def face_averages(plan, a):
    """Per family, the mean across every canvas face, a block face's partner taken
    from the neighbour map, the canvas edge copied (``atlas.py:163-183``)."""
    lead = a.shape[:-2]
    filled = a.reshape(lead + (-1,))[..., plan.neighbours].reshape(a.shape)
    out = []
    for axis in range(2):
        w = [(0, 0)] * filled.ndim
        w[len(lead) + axis] = (1, 1)
        f = np.pad(filled, w, mode="edge")
        lo, hi = [slice(None)] * f.ndim, [slice(None)] * f.ndim
        lo[len(lead) + axis], hi[len(lead) + axis] = slice(0, -1), slice(1, None)
        out.append(0.5 * (f[tuple(lo)] + f[tuple(hi)]))
    return out


def spectral_radius(q, sx, sy, g):
    vn = q[1] * sx + q[2] * sy
    return np.abs(vn) + sound(q[0], q[3], g) * np.hypot(sx, sy)


def wave_speeds(U, model: Model):
    """``lambda`` per canvas face from face-averaged states, plus the thin-layer
    viscous term (``residual.py:169-192``)."""
    plan, g = model.plan, model.gamma
    q = prim(U, g)
    qf = face_averages(plan, q)
    faces = [plan.faces_i, plan.faces_j]
    lam = [spectral_radius(qf[a], faces[a][0], faces[a][1], g) for a in range(2)]
    if not model.viscous:
        return lam
    vols = face_averages(plan, plan.volume)
    factor = 2.0 * g / PR_LAM
    out = []
    for a in range(2):
        f = qf[a]
        mu = model.mu(temperature(f, g))
        if model.sa:
            mu = mu + eddy(f[0], f[4] * model.mu_inf, mu / f[0])
        s = faces[a]
        out.append(lam[a] + factor * mu * (s[0] * s[0] + s[1] * s[1]) / (f[0] * vols[a]))
    return out


def cell_sum(lam):
    """``sum_faces lambda`` per cell (``residual.py:195-203``)."""
    return ((lam[0][:-1] + lam[0][1:]) + lam[1][:, :-1]) + lam[1][:, 1:]


def norm(R, model: Model):
    """Volume-weighted L2 of the density row over block cells (``residual.py:237-240``)."""
    w = np.where(model.plan.interior, model.plan.volume, 0.0)
    return np.sqrt(np.sum(w * R[0] ** 2) / np.sum(w))
