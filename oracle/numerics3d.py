"""The 3D residual ``R(U)`` and its exact first-order JVP, restated in NumPy (oracle).

TEST INFRASTRUCTURE: the checker of the 3D path, never called by the library.

The reference's residual is written once for 2D and 3D (``src/jaxrans/numerics/
residual.py:54-91, 273-334``); this module restates its 3D form on the canvas of a 3D
plan (``jaxrans_b200.plan3d``), variable-major ``(nvar, NI, NJ, NK)`` with
``q = (rho, u, v, w, p[, nu~])``: the ghost fill by gather stages
(``numerics/boundary.py:54-130, 257-267``), MUSCL on the flow rows
(``reconstruction.py:29-80``), HLLC and Roe with a vector normal (``riemann.py:47-203``),
the 3D diamond face gradients (``gradients.py:26-95``), the viscous flux
(``physics/navier_stokes.py:86-116``), the SA row with the vorticity magnitude
``|curl V|`` (``turbulence.py:38-151``), wave speeds (``residual.py:127-203``).  The
dimension-free parts (limiters, the SA functions, the Sutherland law) are those of
``oracle.numerics``.

Complex-safe throughout, for the complex-step JVP.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .numerics import PR_LAM, PR_TURB, SA, STEP, diffusion, eddy, jabs, jmax, jmin, limit, re, sa_source

D = 3


@dataclass
class Model3:
    """Everything the 3D residual of one case needs besides the state."""

    plan: object
    q_inf: np.ndarray               # (nvar,) primitive freestream
    gamma: float = 1.4
    flux: str = "hllc"
    limiter: str = "minmod"
    kappa: float = 0.0
    mu_inf: float | None = None
    sutherland: float | None = None
    sa: bool = False
    distance: np.ndarray | None = None
    c_cr1: float = 0.0              # QCR2000 on the SA model's stress (0: off)

    @property
    def nvar(self) -> int:
        return 6 if self.sa else 5

    @property
    def viscous(self) -> bool:
        return self.mu_inf is not None

    def mu(self, T):
        s = self.sutherland
        if s is None:
            return self.mu_inf
        return self.mu_inf * T * np.sqrt(T) * (1.0 + s) / (T + s)


def dot(a, b):
    """``sum_k a_k b_k`` in index order (``core/state.py:67-73``)."""
    total = a[0] * b[0]
    for k in range(1, a.shape[0]):
        total = total + a[k] * b[k]
    return total


def magnitude(a):
    return np.sqrt(dot(a, a))


# --- state conversions (core/state.py:88-93) -----------------------------------------


def prim(U, gamma: float):
    rho = U[0]
    vel = U[1:4] / rho
    p = (gamma - 1.0) * (U[4] - 0.5 * rho * dot(vel, vel))
    rows = [rho[None], vel, p[None]]
    if U.shape[0] > 5:
        rows.append((U[5] / rho)[None])
    return np.concatenate(rows)


def conservative(q, gamma: float):
    rho, vel, p = q[0], q[1:4], q[4]
    E = p / (gamma - 1.0) + 0.5 * rho * dot(vel, vel)
    rows = [rho[None], rho * vel, E[None]]
    if q.shape[0] > 5:
        rows.append((rho * q[5])[None])
    return np.concatenate(rows)


def initial_state(model: Model3) -> np.ndarray:
    """The freestream on every canvas cell (``residual.py:250-258``)."""
    q = np.asarray(model.q_inf, dtype=np.float64)
    ones = np.ones(model.plan.shape)
    rho, vel, p = q[0] * ones, q[1:4, None, None, None] * ones, q[4] * ones
    E = p / (model.gamma - 1.0) + 0.5 * rho * dot(vel, vel)
    rows = [rho[None], rho * vel, E[None]]
    if q.shape[0] > 5:
        rows.append(((q[0] * q[5:])[:, None, None, None]) * ones)
    return np.concatenate(rows)


# --- boundary conditions (boundary.py:54-130) ------------------------------------------


def mirror(vel, n):
    return vel - 2.0 * dot(vel, n) * n


def characteristic(edge, n, qf, gamma: float):
    """Riemann-invariant far field against the reference ``qf (nvar, m)``."""
    rho_i, v_i, p_i = edge[0], edge[1:4], edge[4]
    rho_f, v_f, p_f = qf[0], qf[1:4], qf[4]
    a_i = np.sqrt(gamma * p_i / rho_i)
    a_f = np.sqrt(gamma * p_f / rho_f)
    two = 2.0 / (gamma - 1.0)
    vn_i, vn_f = dot(v_i, n), dot(v_f, n)
    rp = vn_i + two * a_i
    rm = vn_f - two * a_f
    vn_b = 0.5 * (rp + rm)
    a_b = 0.25 * (gamma - 1.0) * (rp - rm)
    out = re(vn_b) > 0.0
    s_b = np.where(out, p_i / rho_i ** gamma, p_f / rho_f ** gamma)
    tangential = np.where(out, v_i - vn_i * n, v_f - vn_f * n)
    rho_b = (a_b * a_b / (gamma * s_b)) ** (1.0 / (gamma - 1.0))
    p_b = rho_b * a_b * a_b / gamma
    rows = [rho_b[None], vn_b * n + tangential, p_b[None]]
    if edge.shape[0] > 5:
        rows.append(np.where(out, edge[5:], qf[5:]))
    return np.concatenate(rows)


def _condition(kind: str, q, normal, model: Model3):
    if kind in ("slip_wall", "symmetry"):
        scal = q[5:] if kind == "symmetry" else -q[5:]
        return np.concatenate([q[:1], mirror(q[1:4], normal), q[4:5], scal])
    if kind == "no_slip_wall":
        return np.concatenate([q[:1], -q[1:4], q[4:5], -q[5:]])
    if kind == "far_field":
        nv = q.shape[0]
        qf = np.broadcast_to(model.q_inf[:nv, None], (nv, q.shape[1]))
        return characteristic(q, normal, qf, model.gamma)
    raise ValueError(f"the 3D oracle has no condition {kind!r}")


def fill_ghosts(q, model: Model3):
    """Every ghost of a primitive canvas by the plan's gather stages."""
    flat = q.reshape(q.shape[0], -1)
    for st in model.plan.stages:
        parts = [flat] + [_condition(kind, flat[:, source], normal, model)
                          for kind, source, normal, _ in st.conditions]
        flat = np.concatenate(parts, axis=1)[:, st.index]
    return flat.reshape(q.shape)


# --- reconstruction (reconstruction.py:29-80) ------------------------------------------


def _windows(padded, g: int, shape, axis: int):
    out = []
    for off in range(4):
        idx = [slice(None)] + [slice(g, g + n) for n in shape]
        idx[1 + axis] = slice(g - 2 + off, g - 2 + off + shape[axis] + 1)
        out.append(padded[tuple(idx)])
    return out


def face_states(padded, g, shape, axis, model: Model3, first_order: bool):
    q_mm, q_m, q_p, q_pp = _windows(padded, g, shape, axis)
    if first_order:
        return q_m, q_p
    d_minus, d_mid, d_plus = q_m - q_mm, q_p - q_m, q_pp - q_p
    if model.kappa != 0.0:
        lo, hi = 0.25 * (1.0 - model.kappa), 0.25 * (1.0 + model.kappa)
        return q_m + lo * d_minus + hi * d_mid, q_p - lo * d_plus - hi * d_mid
    return q_m + 0.5 * limit(d_minus, d_mid, model.limiter), q_p - 0.5 * limit(d_mid, d_plus, model.limiter)


# --- Riemann fluxes (riemann.py:47-203, physics/euler.py:43-94) -------------------------


def sound(rho, p, g):
    return np.sqrt(g * p / rho)


def normal_flux(q, n, g):
    rho, vel, p = q[0], q[1:4], q[4]
    vn = dot(vel, n)
    E = p / (g - 1.0) + 0.5 * rho * dot(vel, vel)
    return np.concatenate([(rho * vn)[None], rho * vel * vn + p * n, ((E + p) * vn)[None]])


def roe_average(qL, qR, g):
    rho_l, v_l, p_l = qL[0], qL[1:4], qL[4]
    rho_r, v_r, p_r = qR[0], qR[1:4], qR[4]
    h_l = g / (g - 1.0) * p_l / rho_l + 0.5 * dot(v_l, v_l)
    h_r = g / (g - 1.0) * p_r / rho_r + 0.5 * dot(v_r, v_r)
    w = np.sqrt(rho_r / rho_l)
    den = 1.0 + w
    rho = np.sqrt(rho_l * rho_r)
    vel = (v_l + w * v_r) / den
    H = (h_l + w * h_r) / den
    a2 = (g - 1.0) * (H - 0.5 * dot(vel, vel))
    return rho, vel, H, np.sqrt(jmax(a2, 1e-30))


def _unit(s):
    length = magnitude(s)
    return length, s / np.maximum(re(length), 1e-300)


def roe_flux(qL, qR, s, g):
    length, n = _unit(s)
    rho, vel, H, a = roe_average(qL, qR, g)
    vn = dot(vel, n)
    d_rho, d_p = qR[0] - qL[0], qR[4] - qL[4]
    d_v = qR[1:4] - qL[1:4]
    d_vn = dot(d_v, n)
    d_vt = d_v - d_vn * n
    a2 = a * a
    al_m = (d_p - rho * a * d_vn) / (2.0 * a2)
    al_e = d_rho - d_p / a2
    al_p = (d_p + rho * a * d_vn) / (2.0 * a2)
    lm, l0, lp = jabs(vn - a), jabs(vn), jabs(vn + a)
    kin = 0.5 * dot(vel, vel)
    one = np.ones_like(rho)

    def vec(first, v, last):
        return np.concatenate([first[None], v, last[None]])

    r_m = vec(one, vel - a * n, H - a * vn)
    r_e = vec(one, vel, kin)
    shear = vec(np.zeros_like(rho), rho * d_vt, rho * dot(vel, d_vt))
    r_p = vec(one, vel + a * n, H + a * vn)
    diss = lm * al_m * r_m + l0 * al_e * r_e + l0 * shear + lp * al_p * r_p
    central = 0.5 * (normal_flux(qL, n, g) + normal_flux(qR, n, g))
    return length * (central - 0.5 * diss)


def hllc_flux(qL, qR, s, g):
    length, n = _unit(s)
    rho_l, v_l, p_l = qL[0], qL[1:4], qL[4]
    rho_r, v_r, p_r = qR[0], qR[1:4], qR[4]
    vn_l, vn_r = dot(v_l, n), dot(v_r, n)
    a_l, a_r = sound(rho_l, p_l, g), sound(rho_r, p_r, g)
    _, v_ro, _, a_ro = roe_average(qL, qR, g)
    vn_ro = dot(v_ro, n)
    s_l = jmin(vn_l - a_l, vn_ro - a_ro)
    s_r = jmax(vn_r + a_r, vn_ro + a_ro)
    m_l = rho_l * (s_l - vn_l)
    m_r = rho_r * (s_r - vn_r)
    s_m = (p_r - p_l + m_l * vn_l - m_r * vn_r) / jmin(m_l - m_r, -1e-300)

    def star(rho, vel, p, vn, s_k, f_k, u_k, wide):
        p_star = p + rho * (vn - s_k) * (vn - s_m)
        rho_star = rho * (s_k - vn) / wide
        e_star = ((s_k - vn) * u_k[4] - p * vn + p_star * s_m) / wide
        us = np.concatenate([rho_star[None], rho_star * (vel + (s_m - vn) * n), e_star[None]])
        return f_k + s_k * (us - u_k)

    U_l, U_r = conservative(qL[:5], g), conservative(qR[:5], g)
    f_l, f_r = normal_flux(qL, n, g), normal_flux(qR, n, g)
    st_l = star(rho_l, v_l, p_l, vn_l, s_l, f_l, U_l, jmin(s_l - s_m, -1e-300))
    st_r = star(rho_r, v_r, p_r, vn_r, s_r, f_r, U_r, jmax(s_r - s_m, 1e-300))
    f = np.where(re(s_l) >= 0.0, f_l, np.where(re(s_m) >= 0.0, st_l, np.where(re(s_r) >= 0.0, st_r, f_r)))
    return length * f


# --- gradients and the viscous flux (gradients.py:26-95, navier_stokes.py:86-116) --------


def _node_average(a):
    """Average of the eight cells round each node, axis by axis."""
    for axis in range(a.ndim - 3, a.ndim):
        lo, hi = [slice(None)] * a.ndim, [slice(None)] * a.ndim
        lo[axis], hi[axis] = slice(0, -1), slice(1, None)
        a = 0.5 * (a[tuple(lo)] + a[tuple(hi)])
    return a


def _cross(a, b):
    return np.stack([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def face_gradients(phi, centres):
    """Per family, ``(3, nphi, face)``: the linear field reproducing the differences
    along the centre-to-centre line and the face's two node diagonals (node values and
    positions the means of the eight surrounding cells)."""
    shape = tuple(n - 2 for n in centres.shape[1:])
    xn, pn = _node_average(centres), _node_average(phi)
    out = []
    for a in range(3):
        def cell(off):
            idx = [slice(1, 1 + n) for n in shape]
            idx[a] = slice(off, off + shape[a] + 1)
            return (slice(None),) + tuple(idx)

        def node(shifts):
            idx, others = [], iter(shifts)
            for b in range(3):
                start = 0 if b == a else next(others)
                idx.append(slice(start, start + shape[b] + (b == a)))
            return (slice(None),) + tuple(idx)

        d1 = centres[cell(1)] - centres[cell(0)]
        p1 = phi[cell(1)] - phi[cell(0)]
        (lo2, hi2), (lo3, hi3) = (node((0, 0)), node((1, 1))), (node((1, 0)), node((0, 1)))
        d2, d3 = xn[hi2] - xn[lo2], xn[hi3] - xn[lo3]
        p2, p3 = pn[hi2] - pn[lo2], pn[hi3] - pn[lo3]
        c23, c31, c12 = _cross(d2, d3), _cross(d3, d1), _cross(d1, d2)
        det = d1[0] * c23[0] + d1[1] * c23[1] + d1[2] * c23[2]
        out.append((p1 * c23[:, None] + p2 * c31[:, None] + p3 * c12[:, None]) / det[None, None])
    return out


def _sides(p1, a):
    """Cells before and after every face of family ``a`` of a one-ghost field."""
    lead = p1.ndim - 3
    lo = [slice(None)] * lead + [slice(1, -1)] * 3
    hi = list(lo)
    n = p1.shape[lead + a]
    lo[lead + a], hi[lead + a] = slice(0, n - 1), slice(1, n)
    return p1[tuple(lo)], p1[tuple(hi)]


def face_avg(p1, a):
    lo, hi = _sides(p1, a)
    return 0.5 * (lo + hi)


def temperature(q, g):
    return g * q[4] / q[0]


def qcr_stress(gv, mu_t, c_cr1):
    """QCR2000's addition to the stress (``spalart_allmaras.py:197-216``): ``-c_cr1 (O_ik
    tau_jk + O_jk tau_ik)``, ``O = (grad V - grad V^T) / |grad V|`` (1 in place of the norm
    where grad V is 0), ``tau = mu_t (grad V + grad V^T - 2/3 div V I)``."""
    square = sum(gv[a][b] * gv[a][b] for a in range(3) for b in range(3))
    positive = np.real(square) > 0.0
    norm = np.where(positive, np.sqrt(np.where(positive, square, 1.0)), 1.0)
    div = gv[0][0] + gv[1][1] + gv[2][2]
    rot = [[(gv[a][b] - gv[b][a]) / norm for b in range(3)] for a in range(3)]
    tau = [[mu_t * (gv[a][b] + gv[b][a] - ((2.0 / 3.0) * div if a == b else 0.0)) for b in range(3)]
           for a in range(3)]
    prod = [[rot[i][0] * tau[j][0] + rot[i][1] * tau[j][1] + rot[i][2] * tau[j][2] for j in range(3)]
            for i in range(3)]
    return [[-c_cr1 * (prod[a][b] + prod[b][a]) for b in range(3)] for a in range(3)]


def viscous_flux(vel, gv, gt, s, mu, k, extra=None):
    """``F_v . S`` with ``gv[a][b] = d v_a / d x_b``; ``extra`` added to the stress."""
    div = gv[0][0] + gv[1][1] + gv[2][2]
    ttd = (2.0 / 3.0) * div

    def tau(a, b):
        if a == b:
            t = mu * (2.0 * gv[a][a] - ttd)
        else:
            lo, hi = min(a, b), max(a, b)
            t = mu * (gv[lo][hi] + gv[hi][lo])
        return t if extra is None else t + extra[a][b]

    force = np.stack([dot(np.stack([tau(a, b) for b in range(3)]), s) for a in range(3)])
    energy = dot(vel, force) + k * dot(gt, s)
    return np.concatenate([np.zeros_like(energy)[None], force, energy[None]])


def viscous_fluxes(p1, centres, faces, model: Model3, mu_t=None, grads=None):
    g = model.gamma
    if grads is None:
        phi = np.concatenate([p1[1:4], temperature(p1, g)[None]])
        grads = face_gradients(phi, centres)
    out = []
    for a in range(3):
        lo, hi = _sides(p1, a)
        vel = 0.5 * (lo[1:4] + hi[1:4])
        T = 0.5 * (temperature(lo, g) + temperature(hi, g))
        mu = model.mu(T)
        k = mu / (PR_LAM * (g - 1.0))
        if mu_t is not None:
            mu = mu + mu_t[a]
            k = k + mu_t[a] / (PR_TURB * (g - 1.0))
        G = grads[a]
        gv = [[G[b, c] for b in range(3)] for c in range(3)]       # gv[component][direction]
        extra = qcr_stress(gv, mu_t[a], model.c_cr1) if mu_t is not None and model.c_cr1 else None
        out.append(viscous_flux(vel, gv, G[:, 3], faces[a], mu, k, extra))
    return out


# --- the SA row (turbulence.py:56-151) ----------------------------------------------------


def divergence(fluxes):
    total = None
    for a, f in enumerate(fluxes):
        axis = f.ndim - 3 + a
        lo, hi = [slice(None)] * f.ndim, [slice(None)] * f.ndim
        lo[axis], hi[axis] = slice(0, -1), slice(1, None)
        diff = f[tuple(hi)] - f[tuple(lo)]
        total = diff if total is None else total + diff
    return total


def green_gauss(phi_faces, faces, volume):
    return np.stack([divergence([phi * s[c] for phi, s in zip(phi_faces, faces)]) / volume for c in range(3)])


def vorticity_magnitude(gx):
    """``|curl V|`` from ``gx[b, a] = d v_a / d x_b``, with derivative 0 where it is 0."""
    curl = np.stack([gx[1, 2] - gx[2, 1], gx[2, 0] - gx[0, 2], gx[0, 1] - gx[1, 0]])
    square = dot(curl, curl)
    pos = re(square) > 0.0
    return np.where(pos, np.sqrt(np.where(pos, square, 1.0)), 0.0)


def sa_row(p1, mass, grad_nu, faces, volume, model: Model3):
    g, nu_inf = model.gamma, model.mu_inf
    nu_hat = p1[5]
    fl = []
    for a in range(3):
        lo, hi = _sides(nu_hat, a)
        up = np.where(re(mass[a]) > 0.0, lo, hi)
        fa = face_avg(p1, a)
        mu = model.mu(temperature(fa, g))
        coef = diffusion(fa[0], fa[5] * nu_inf, mu)
        fl.append(mass[a] * up - coef * dot(grad_nu[a], faces[a]))
    cell = p1[:, 1:-1, 1:-1, 1:-1]
    rho = cell[0]
    mu = model.mu(temperature(cell, g))
    omega = vorticity_magnitude(green_gauss([face_avg(p1[1:4], a) for a in range(3)], faces, volume))
    P, Dd = sa_source(cell[5] * nu_inf, mu / rho, omega, model.distance)
    grad = green_gauss([face_avg(nu_hat, a) for a in range(3)], faces, volume)
    src = rho * ((P - Dd) / nu_inf + SA.c_b2 / SA.sigma * nu_inf * dot(grad, grad))
    return divergence(fl) - src * volume


# --- the residual (residual.py:54-91, 273-334) ----------------------------------------------


def net_flux(padded, model: Model3, first_order: bool):
    plan = model.plan
    g, gamma, shape, faces = plan.g, model.gamma, plan.shape, plan.faces
    flow = padded[:5]
    F = hllc_flux if model.flux == "hllc" else roe_flux
    fluxes = [F(*face_states(flow, g, shape, a, model, first_order), faces[a], gamma) for a in range(3)]
    sa = None
    if model.viscous:
        c = g - 1
        p1 = padded[(slice(None),) + (slice(c, -c),) * 3]
        if not model.sa:
            visc = viscous_fluxes(p1, plan.centres, faces, model)
        else:
            phi = np.concatenate([p1[1:4], temperature(p1, gamma)[None], p1[5][None]])
            grads = face_gradients(phi, plan.centres)
            mu_t = []
            for a in range(3):
                fa = face_avg(p1, a)
                mu_t.append(eddy(fa[0], fa[5] * model.mu_inf, model.mu(temperature(fa, gamma)) / fa[0]))
            visc = viscous_fluxes(p1, plan.centres, faces, model, mu_t, grads)
            sa = sa_row(p1, [f[0] for f in fluxes], [G[:, 4] for G in grads], faces, plan.volume, model)
        fluxes = [f - v for f, v in zip(fluxes, visc)]
    R = divergence(fluxes)
    return R if sa is None else np.concatenate([R, sa[None]])


def residual(U, model: Model3, first_order: bool = False):
    """``where(interior, net flux, U - U0)`` on the canvas."""
    g = model.plan.g
    q = prim(U, model.gamma)
    padded = np.pad(fill_ghosts(q, model), ((0, 0),) + ((g, g),) * 3, mode="edge")
    R = net_flux(padded, model, first_order)
    return np.where(model.plan.interior, R, U - initial_state(model))


def jvp(U, v, model: Model3, first_order: bool = True):
    """Exact ``dR/dU . v`` by the complex step."""
    return np.imag(residual(U.astype(np.complex128) + 1j * STEP * v, model, first_order)) / STEP


# --- wave speeds and the norm (residual.py:127-240, atlas.py:163-183) ------------------------


def face_averages(plan, a):
    lead = a.shape[:-3]
    filled = a.reshape(lead + (-1,))[..., plan.neighbours].reshape(a.shape)
    out = []
    for axis in range(3):
        w = [(0, 0)] * filled.ndim
        w[len(lead) + axis] = (1, 1)
        f = np.pad(filled, w, mode="edge")
        lo, hi = [slice(None)] * f.ndim, [slice(None)] * f.ndim
        lo[len(lead) + axis], hi[len(lead) + axis] = slice(0, -1), slice(1, None)
        out.append(0.5 * (f[tuple(lo)] + f[tuple(hi)]))
    return out


def spectral_radius(q, s, g):
    return np.abs(dot(q[1:4], s)) + sound(q[0], q[4], g) * magnitude(s)


def wave_speeds(U, model: Model3):
    plan, g = model.plan, model.gamma
    q = prim(U, g)
    qf = face_averages(plan, q)
    lam = [spectral_radius(qf[a], plan.faces[a], g) for a in range(3)]
    if not model.viscous:
        return lam
    vols = face_averages(plan, plan.volume)
    factor = 2.0 * g / PR_LAM
    out = []
    for a in range(3):
        f = qf[a]
        mu = model.mu(temperature(f, g))
        if model.sa:
            mu = mu + eddy(f[0], f[5] * model.mu_inf, mu / f[0])
        s = plan.faces[a]
        out.append(lam[a] + factor * mu * dot(s, s) / (f[0] * vols[a]))
    return out


def cell_sum(lam):
    total = None
    for a, l in enumerate(lam):
        lo, hi = [slice(None)] * 3, [slice(None)] * 3
        lo[a], hi[a] = slice(0, -1), slice(1, None)
        total = l[tuple(lo)] + l[tuple(hi)] if total is None else total + l[tuple(lo)] + l[tuple(hi)]
    return total


def norm(R, model: Model3):
    w = np.where(model.plan.interior, model.plan.volume, 0.0)
    return np.sqrt(np.sum(w * R[0] ** 2) / np.sum(w))
