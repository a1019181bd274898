"""The 3D line preconditioner restated in NumPy (oracle; TEST INFRASTRUCTURE).

Follows ``src/jaxrans/solvers/preconditioners.py:209-306`` on a 3D plan: the mean-flow
chains carry 5x5 blocks (``diag = sum_f lambda_f (1/CFL + 1/2) I``, ``off = 1/2 A(U_nb,
S_out) - 1/2 lambda_f I``), the SA row its own scalar chains (upwind mass flux, thin
layer diffusion, the destruction derivative, V/dt).  The chains are solved by the
block cyclic reduction of ``oracle.implicit`` (``src/jaxrans/core/linalg.py:159-200``),
which is written for any block size.
"""

from __future__ import annotations

import numpy as np

from . import numerics as nm
from . import numerics3d as n3
from .implicit import cr_factor, cr_solve, thomas_factor, thomas_solve


def _families(fields):
    return np.concatenate([f.reshape(f.shape[:-3] + (-1,)) for f in fields], axis=-1)


def _gather(field, lines):
    cells = np.where(lines.cells >= 0, lines.cells, 0)
    return field.reshape(field.shape[:-3] + (-1,))[..., cells]


def _faces(fields, lines, side):
    idx = lines.up_face if side == "up" else lines.down_face
    return _families(fields)[..., idx]


def normal_flux_jacobian(q, s, g):
    """``A = d(F . S)/dU`` ``(5, 5, ...)`` [row, variable] by the complex step on the flux
    of the conservative state (``physics/euler.py:55-71``)."""
    U = n3.conservative(q[:5], g)
    cols = []
    for k in range(5):
        Uc = U.astype(np.complex128)
        Uc[k] = Uc[k] + 1j * nm.STEP
        cols.append(np.imag(n3.normal_flux(n3.prim(Uc, g), s, g)) / nm.STEP)
    return np.stack(cols, axis=1)


def chain_blocks_flow(U, lam, cfl, model):
    """``(lower, diag, upper)`` ``(L, n_lines, 5, 5)`` of the mean-flow chains."""
    plan, g = model.plan, model.gamma
    lines = plan.lines
    valid = lines.cells >= 0
    q = n3.prim(U[:5], g)
    eye = np.eye(5)
    d = np.where(valid, _gather(n3.cell_sum(lam) * (1.0 / cfl + 0.5), lines), 1.0)
    diag = d.T[:, :, None, None] * eye

    def coupling(side, sign, nb):
        s = _faces(plan.faces, lines, side)
        block = 0.5 * normal_flux_jacobian(nb, sign * s, g) - 0.5 * _faces(lam, lines, side) * eye.reshape(5, 5, 1, 1)
        return np.transpose(np.where(sign != 0, block, 0.0), (3, 2, 0, 1))

    chains = _gather(q, lines)
    above = np.concatenate([chains[:, :, 1:], chains[:, :, -1:]], axis=2)
    upper = coupling("up", lines.up_sign, above)
    below = coupling("down", lines.down_sign, chains)
    lower = np.concatenate([np.zeros_like(below[:1]), below[:-1]], axis=0)
    return lower, diag, upper


def chain_blocks_sa(U, lam, cfl, model):
    """Scalar SA chain blocks ``(L, n_lines, 1, 1)``."""
    plan, g, nu_inf = model.plan, model.gamma, model.mu_inf
    lines = plan.lines
    valid = lines.cells >= 0
    q = n3.prim(U, g)
    qf = n3.face_averages(plan, q)
    vols = n3.face_averages(plan, plan.volume)
    terms = []
    for a in range(3):
        f, s = qf[a], plan.faces[a]
        mu = model.mu(n3.temperature(f, g))
        kap = nm.diffusion(f[0], f[5] * nu_inf, mu)
        terms.append((f[0] * n3.dot(f[1:4], s), kap * n3.dot(s, s) / vols[a]))
    rho = q[0]
    diag = None
    for a, (m_f, d_f) in enumerate(terms):
        lo, hi = [slice(None)] * 3, [slice(None)] * 3
        lo[a], hi[a] = slice(0, -1), slice(1, None)
        out_f = np.maximum(m_f, 0.0) + d_f
        in_f = np.maximum(-m_f, 0.0) + d_f
        diag = out_f[tuple(hi)] + in_f[tuple(lo)] if diag is None else diag + out_f[tuple(hi)] + in_f[tuple(lo)]
    diag = diag / rho
    nu_hat = q[5]
    gx = n3.green_gauss([f[1:4] for f in qf], plan.faces, plan.volume)
    nu = model.mu(n3.temperature(q, g)) / rho
    d = model.distance
    s_t = nm.s_tilde(n3.vorticity_magnitude(gx), nu_hat * nu_inf, nu, d)
    fw = nm.f_w(nm.r_of(nu_hat * nu_inf, s_t, d))
    dest = np.where(nu_hat > 0.0, 2.0 * nm.SA.c_w1 * fw * nu_inf * nu_hat / d ** 2, 0.0)
    diag = diag + dest * plan.volume + n3.cell_sum(lam) / cfl
    d_chain = np.where(valid, _gather(diag, lines), 1.0)
    rho_chain = _gather(rho, lines)
    m, dj = tuple(t[0] for t in terms), tuple(t[1] for t in terms)

    def coupling(side, sign, rho_nb):
        block = -(np.maximum(-sign * _faces(m, lines, side), 0.0) + _faces(dj, lines, side)) / rho_nb
        return np.where(sign != 0, block, 0.0).T[:, :, None, None]

    above = np.concatenate([rho_chain[:, 1:], rho_chain[:, -1:]], axis=1)
    upper = coupling("up", lines.up_sign, above)
    below = coupling("down", lines.down_sign, rho_chain)
    lower = np.concatenate([np.zeros_like(below[:1]), below[:-1]], axis=0)
    return lower, d_chain.T[:, :, None, None], upper


def precondition(U, lam, cfl, model, solver: str = "cr"):
    """``r -> M^-1 r`` of ``line_j`` on a 3D plan: exact solves along the chains, the SA
    row on its own scalar chains."""
    lines = model.plan.lines
    valid = lines.cells >= 0
    found = np.full(model.plan.n_canvas, -1, dtype=np.int64)
    found[lines.cells[valid]] = np.flatnonzero(valid)
    fac = cr_factor if solver == "cr" else thomas_factor
    sol = cr_solve if solver == "cr" else thomas_solve
    parts = [(slice(0, 5), fac(*chain_blocks_flow(U, lam, cfl, model)))]
    if model.sa:
        parts.append((slice(5, 6), fac(*chain_blocks_sa(U, lam, cfl, model))))

    def apply(r):
        out = []
        for rows, factor in parts:
            rr = r[rows]
            rhs = np.where(valid, _gather(rr, lines), 0.0)
            x = np.transpose(sol(factor, np.transpose(rhs, (2, 1, 0))), (2, 1, 0))
            flat = rr.reshape(rr.shape[0], -1)
            vals = x.reshape(x.shape[0], -1)[:, np.where(found >= 0, found, 0)]
            out.append(np.where(found >= 0, vals, flat).reshape(rr.shape))
        return np.concatenate(out)

    return apply


def chain_coupling_sa(U, model):
    """The SA row's coupling to the neighbours' mean flow in the coupled (6x6) line
    blocks: ``(lower, upper)`` ``(L, n_lines, 5)``, half the Jacobian of the SA convective
    flux ``rho nu_hat V.S`` with respect to the neighbour's (rho, rho u, rho v, rho w,
    rho E) at the neighbour's state, ``[-nu_hat vn, nu_hat Sx, nu_hat Sy, nu_hat Sz, 0]``,
    with the link's face vector and sign as the mean-flow blocks use them
    (``chain_blocks_flow``).  The mean-flow rows do not depend on rho nu_hat, so the
    6x6 blocks are block lower triangular.  This build's coupled variant of ``line_j``
    (the 3D form of ``oracle.implicit.chain_coupling_sa``); the reference has only the
    split form (``preconditioners.py:291-306``)."""
    plan, g = model.plan, model.gamma
    lines = plan.lines
    q = n3.prim(U, g)

    def coupling(side, sign, nb):
        s = _faces(plan.faces, lines, side)
        sx, sy, sz = sign * s[0], sign * s[1], sign * s[2]
        nu = nb[5]
        vn = nb[1] * sx + nb[2] * sy + nb[3] * sz
        row = 0.5 * np.stack([-nu * vn, nu * sx, nu * sy, nu * sz, np.zeros_like(vn)])
        return np.transpose(np.where(sign != 0, row, 0.0), (2, 1, 0))

    chains = _gather(q, lines)
    above = np.concatenate([chains[:, :, 1:], chains[:, :, -1:]], axis=2)
    upper = coupling("up", lines.up_sign, above)
    below = coupling("down", lines.down_sign, chains)
    lower = np.concatenate([np.zeros_like(below[:1]), below[:-1]], axis=0)
    return lower, upper


def precondition_coupled(U, lam, cfl, model, solver: str = "cr"):
    """``r -> M^-1 r`` with the coupled 6x6 line blocks: the mean flow solved first, then
    the SA chains with the right-hand side ``r_sa - C z_flow`` (block forward
    substitution of the block lower-triangular blocks)."""
    split = precondition(U, lam, cfl, model, solver)
    lines = model.plan.lines
    valid = lines.cells >= 0
    lower, upper = chain_coupling_sa(U, model)
    fac = cr_factor if solver == "cr" else thomas_factor
    sol = cr_solve if solver == "cr" else thomas_solve
    sa_factor = fac(*chain_blocks_sa(U, lam, cfl, model))

    def apply(r):
        z = split(r)
        zf = np.transpose(np.where(valid, _gather(z[:5], lines), 0.0), (2, 1, 0))   # (L, n_lines, 5)
        below = np.concatenate([np.zeros_like(zf[:1]), zf[:-1]], axis=0)
        above = np.concatenate([zf[1:], np.zeros_like(zf[:1])], axis=0)
        cz = np.sum(lower * below, axis=-1) + np.sum(upper * above, axis=-1)       # (L, n_lines)
        rhs = np.where(valid, _gather(r[5:6], lines), 0.0)[0].T - cz
        x = sol(sa_factor, rhs[:, :, None])[:, :, 0].T                              # (n_lines, L)
        out = z.copy()
        flat = out[5].reshape(-1)
        flat[lines.cells[valid]] = x[valid]
        out[5] = flat.reshape(out[5].shape)
        return out

    return apply


# --- the Newton step (src/jaxrans/solvers/implicit.py:54-168, core/state.py:142-150) ------


def relax(dU, U, g, fraction):
    """One global factor so no cell's density or (linearized) pressure moves by more than
    ``fraction`` of itself, nor ``nu~`` by more than ``fraction`` of ``max(|nu~|, 1)``."""
    if fraction is None:
        return dU, 1.0
    q = n3.prim(U[:5], g)
    rho, vel, p = q[0], q[1:4], q[4]
    d_e = dU[4]
    for k in range(3):
        d_e = d_e - vel[k] * dU[1 + k]
    d_p = (g - 1.0) * (d_e + 0.5 * n3.dot(vel, vel) * dU[0])
    ratios = [np.abs(dU[0]) / rho, np.abs(d_p) / p]
    if U.shape[0] > 5:
        nh = U[5] / rho
        ratios.append(np.abs((dU[5] - nh * dU[0]) / rho) / np.maximum(np.abs(nh), 1.0))
    worst = max(float(np.max(r)) for r in ratios)
    omega = min(1.0, fraction / max(worst, 1e-300))
    return omega * dU, omega


def is_physical(U, g):
    q = n3.prim(U[:5], g)
    return (q[0] > 1e-10) & (q[4] > 1e-10) & np.isfinite(q[0]) & np.isfinite(q[4])


def newton_step(state, model, config, solver: str = "cr"):
    """One pseudo-transient Newton step on a 3D plan (the 2D step of ``oracle.implicit``
    with the 3D residual, JVP, wave speeds and preconditioner)."""
    from .implicit import NewtonState, gmres_right
    U, cfl = state.U, state.cfl
    R = n3.residual(U, model)
    norm = n3.norm(R, model)
    lam = n3.wave_speeds(U, model)
    vdt = n3.cell_sum(lam) / cfl
    prec = precondition(U, lam, cfl, model, solver) if config.preconditioner == "line_j" else (lambda r: r)

    def matvec(d):
        return vdt[None] * d + n3.jvp(U, d, model)

    dU, action = gmres_right(matvec, -R, prec, config.krylov_subspace, config.krylov_restarts, config.krylov_tol)
    dU, omega = relax(dU, U, model.gamma, config.max_relative_update)
    lin = np.linalg.norm(omega * action + R) / max(np.linalg.norm(R), 1e-300)
    cand = U + dU
    physical = bool(np.all(is_physical(cand, model.gamma)) and np.all(np.isfinite(dU)))
    accept = physical and lin < 1.0
    reduction = state.residual_norm / max(norm, 1e-300)
    if accept and lin < config.krylov_success and omega >= 1.0:
        cfl_next = cfl * min(max(reduction, 1.0), config.cfl_growth)
    elif accept:
        cfl_next = cfl
    else:
        cfl_next = cfl / config.cfl_cutback
    return NewtonState(cand if accept else U, min(max(cfl_next, config.cfl_min), config.cfl_max),
                       norm if accept else state.residual_norm), norm
