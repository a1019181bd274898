"""The line preconditioner, GMRES and the Newton step, restated in NumPy (oracle).

Follows ``src/jaxrans/solvers/preconditioners.py:74-306`` (chain blocks),
``src/jaxrans/core/linalg.py:49-200`` (block Thomas and cyclic reduction),
``src/jaxrans/solvers/krylov.py:34-137`` (right-preconditioned GMRES, CGS2,
Givens least squares) and ``src/jaxrans/solvers/implicit.py:54-168`` (the step).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import numerics as nm


# --- chains (preconditioners.py:88-121) --------------------------------------------


def _families(fields):
    return np.concatenate([f.reshape(f.shape[:-2] + (-1,)) for f in fields], axis=-1)


def _gather(field, chains):
    cells = np.where(chains.cells >= 0, chains.cells, 0)
    return field.reshape(field.shape[:-2] + (-1,))[..., cells]


def _faces(fields, chains, side):
    idx = chains.up_face if side == "up" else chains.down_face
    return _families(fields)[..., idx]


def normal_flux_jacobian(q, sx, sy, g):
    """``A = d(F . S)/dU`` ``(4, 4, ...)`` [row, variable] by the complex step on
    the flux of the conservative state (``physics/euler.py:55-71``)."""
    U = nm.conservative(q[:4], g)
    cols = []
    for k in range(4):
        Uc = U.astype(np.complex128)
        Uc[k] = Uc[k] + 1j * nm.STEP
        F = nm.normal_flux(nm.prim(Uc, g), sx, sy, g)
        cols.append(np.imag(F) / nm.STEP)
    return np.stack(cols, axis=1)


def chain_blocks_flow(U, lam, cfl, model):
    """``(lower, diag, upper)`` ``(L, n_lines, 4, 4)`` of the mean-flow chains
    (``preconditioners.py:209-232``)."""
    plan, g = model.plan, model.gamma
    ch = plan.chains
    valid = ch.cells >= 0
    q = nm.prim(U[:4], g)
    eye = np.eye(4)
    d = np.where(valid, _gather(nm.cell_sum(lam) * (1.0 / cfl + 0.5), ch), 1.0)
    diag = d.T[:, :, None, None] * eye
    S = (plan.faces_i, plan.faces_j)

    def coupling(side, sign, nb):
        s = _faces(S, ch, side)
        A = normal_flux_jacobian(nb, sign * s[0], sign * s[1], g)
        block = 0.5 * A - 0.5 * _faces(lam, ch, side) * eye.reshape(4, 4, 1, 1)
        return np.transpose(np.where(sign != 0, block, 0.0), (3, 2, 0, 1))

    chains = _gather(q, ch)
    above = np.concatenate([chains[:, :, 1:], chains[:, :, -1:]], axis=2)
    upper = coupling("up", ch.up_sign, above)
    below = coupling("down", ch.down_sign, chains)
    lower = np.concatenate([np.zeros_like(below[:1]), below[:-1]], axis=0)
    return lower, diag, upper


def chain_blocks_sa(U, lam, cfl, model):
    """Scalar SA chain blocks ``(L, n_lines, 1, 1)`` (``preconditioners.py:235-287``)."""
    plan, g, nu_inf = model.plan, model.gamma, model.mu_inf
    ch = plan.chains
    valid = ch.cells >= 0
    q = nm.prim(U, g)
    qf = nm.face_averages(plan, q)
    vols = nm.face_averages(plan, plan.volume)
    faces = (plan.faces_i, plan.faces_j)
    terms = []
    for a in range(2):
        f, s = qf[a], faces[a]
        mu = model.mu(nm.temperature(f, g))
        kap = nm.diffusion(f[0], f[4] * nu_inf, mu)
        terms.append((f[0] * (f[1] * s[0] + f[2] * s[1]), kap * (s[0] * s[0] + s[1] * s[1]) / vols[a]))
    rho = q[0]
    diag = None
    for a, (m_f, d_f) in enumerate(terms):
        out_f = np.maximum(m_f, 0.0) + d_f
        in_f = np.maximum(-m_f, 0.0) + d_f
        if a == 0:
            out_hi, in_lo = out_f[1:], in_f[:-1]
        else:
            out_hi, in_lo = out_f[:, 1:], in_f[:, :-1]
        diag = out_hi + in_lo if diag is None else diag + out_hi + in_lo
    diag = diag / rho
    nu_hat = q[4]
    gx = nm.green_gauss([f[1:3] for f in qf], faces, plan.volume)
    nu = model.mu(nm.temperature(q, g)) / rho
    d = model.distance
    s_t = nm.s_tilde(nm.vorticity_abs(gx), nu_hat * nu_inf, nu, d)
    fw = nm.f_w(nm.r_of(nu_hat * nu_inf, s_t, d))
    dest = np.where(nu_hat > 0.0, 2.0 * nm.SA.c_w1 * fw * nu_inf * nu_hat / d ** 2, 0.0)
    diag = diag + dest * plan.volume + nm.cell_sum(lam) / cfl
    d_chain = np.where(valid, _gather(diag, ch), 1.0)
    rho_chain = _gather(rho, ch)
    m, dj = tuple(t[0] for t in terms), tuple(t[1] for t in terms)

    def coupling(side, sign, rho_nb):
        block = -(np.maximum(-sign * _faces(m, ch, side), 0.0) + _faces(dj, ch, side)) / rho_nb
        return np.where(sign != 0, block, 0.0).T[:, :, None, None]

    above = np.concatenate([rho_chain[:, 1:], rho_chain[:, -1:]], axis=1)
    upper = coupling("up", ch.up_sign, above)
    below = coupling("down", ch.down_sign, rho_chain)
    lower = np.concatenate([np.zeros_like(below[:1]), below[:-1]], axis=0)
    return lower, d_chain.T[:, :, None, None], upper


# --- block tridiagonal solvers (linalg.py:49-200) -------------------------------------


def invert(A):
    """Unpivoted Gauss-Jordan inverse of every block ``(..., m, m)``."""
    m = A.shape[-1]
    rows = [np.concatenate([A[..., k, :], np.broadcast_to(np.eye(m)[k], A.shape[:-2] + (m,))], axis=-1)
            for k in range(m)]
    for k in range(m):
        rows[k] = rows[k] / rows[k][..., k, None]
        for r in range(m):
            if r != k:
                rows[r] = rows[r] - rows[r][..., k, None] * rows[k]
    return np.stack([row[..., m:] for row in rows], axis=-2)


def _mm(a, b):
    return np.sum(a[..., :, :, None] * b[..., None, :, :], axis=-2)


def _mv(a, x):
    return np.sum(a * x[..., None, :], axis=-1)


def thomas_factor(lower, diag, upper):
    n = diag.shape[0]
    piv, chat = np.empty_like(diag), np.empty_like(diag)
    c_prev = np.zeros_like(diag[0])
    for k in range(n):
        piv[k] = invert(diag[k] - _mm(lower[k], c_prev))
        chat[k] = _mm(piv[k], upper[k])
        c_prev = chat[k]
    return lower, piv, chat


def thomas_solve(factor, rhs):
    lower, piv, chat = factor
    n = rhs.shape[0]
    d = np.empty_like(rhs)
    prev = np.zeros_like(rhs[0])
    for k in range(n):
        d[k] = _mv(piv[k], rhs[k] - _mv(lower[k], prev))
        prev = d[k]
    x = np.empty_like(rhs)
    nxt = np.zeros_like(rhs[0])
    for k in range(n - 1, -1, -1):
        x[k] = d[k] - _mv(chat[k], nxt)
        nxt = x[k]
    return x


def _next(x, n):
    return np.concatenate([x[1:], np.zeros_like(x[:1])])[:n]


def _prev(x, n):
    return np.concatenate([np.zeros_like(x[:1]), x])[:n]


def _first(x, n):
    return np.concatenate([x, np.zeros_like(x[:1])])[:n]


def cr_factor(lower, diag, upper):
    """Block cyclic reduction (``linalg.py:159-182``)."""
    a, d, c = lower, diag, upper
    levels = []
    while d.shape[0] > 1:
        odd = d.shape[0] // 2
        inv, low, upp = invert(d[0::2]), a[0::2], c[0::2]
        alpha, gam = _mm(a[1::2], inv[:odd]), _mm(c[1::2], _next(inv, odd))
        levels.append((inv, low, upp, alpha, gam))
        a, d, c = (-_mm(alpha, low[:odd]),
                   d[1::2] - _mm(alpha, upp[:odd]) - _mm(gam, _next(low, odd)),
                   -_mm(gam, _next(upp, odd)))
    return levels, invert(d)


def cr_solve(factor, rhs):
    levels, last = factor
    b, evens = rhs, []
    for _, _, _, alpha, gam in levels:
        odd = b.shape[0] // 2
        evens.append(b[0::2])
        b = b[1::2] - _mv(alpha, b[0::2][:odd]) - _mv(gam, _next(b[0::2], odd))
    x = _mv(last, b)
    for (inv, low, upp, _, _), be in zip(reversed(levels), reversed(evens)):
        ne, no = be.shape[0], x.shape[0]
        xe = _mv(inv, be - _mv(low, _prev(x, ne)) - _mv(upp, _first(x, ne)))
        pairs = np.stack([xe[:no], x], axis=1).reshape((-1,) + x.shape[1:])
        x = np.concatenate([pairs, xe[no:]])
    return x


def precondition(U, lam, cfl, model, solver: str = "cr"):
    """``r -> M^-1 r`` of ``line_j`` (``preconditioners.py:291-306``): exact
    solves along the chains, the SA row on its own scalar chains."""
    ch = model.plan.chains
    valid = ch.cells >= 0
    found = np.full(model.plan.n_canvas, -1, dtype=np.int64)
    found[ch.cells[valid]] = np.flatnonzero(valid)
    fac = cr_factor if solver == "cr" else thomas_factor
    sol = cr_solve if solver == "cr" else thomas_solve
    parts = [(slice(0, 4), fac(*chain_blocks_flow(U, lam, cfl, model)))]
    if model.sa:
        parts.append((slice(4, 5), fac(*chain_blocks_sa(U, lam, cfl, model))))

    def apply(r):
        out = []
        for rows, factor in parts:
            rr = r[rows]
            rhs = np.where(valid, _gather(rr, ch), 0.0)
            x = np.transpose(sol(factor, np.transpose(rhs, (2, 1, 0))), (2, 1, 0))
            flat = rr.reshape(rr.shape[0], -1)
            vals = x.reshape(x.shape[0], -1)[:, np.where(found >= 0, found, 0)]
            out.append(np.where(found >= 0, vals, flat).reshape(rr.shape))
        return np.concatenate(out)

    return apply


def chain_coupling_sa(U, model):
    """The SA row's coupling to the mean flow in the coupled (5x5) line blocks:
    ``(lower, upper)`` ``(L, n_lines, 4)``, half the Jacobian of the SA convective flux
    ``rho nu_hat V.S`` with respect to the neighbour's (rho, rho u, rho v, rho E) at the
    neighbour's state, ``[-nu_hat vn, nu_hat Sx, nu_hat Sy, 0]``, with the link's face
    vector and sign exactly as the mean-flow blocks use them (``chain_blocks_flow``).
    The mean-flow rows do not depend on rho nu_hat, so the 5x5 blocks are block lower
    triangular.  This coupled form is jaxrans_b200's 5x5 variant of ``line_j``; the
    reference has only the split form (``preconditioners.py:291-306``)."""
    plan, g = model.plan, model.gamma
    ch = plan.chains
    q = nm.prim(U, g)
    S = (plan.faces_i, plan.faces_j)

    def coupling(side, sign, nb):
        s = _faces(S, ch, side)
        sx, sy = sign * s[0], sign * s[1]
        nu = nb[4]
        vn = nb[1] * sx + nb[2] * sy
        row = 0.5 * np.stack([-nu * vn, nu * sx, nu * sy, np.zeros_like(vn)])
        return np.transpose(np.where(sign != 0, row, 0.0), (2, 1, 0))

    chains = _gather(q, ch)
    above = np.concatenate([chains[:, :, 1:], chains[:, :, -1:]], axis=2)
    upper = coupling("up", ch.up_sign, above)
    below = coupling("down", ch.down_sign, chains)
    lower = np.concatenate([np.zeros_like(below[:1]), below[:-1]], axis=0)
    return lower, upper


def precondition_coupled(U, lam, cfl, model):
    """``r -> M^-1 r`` with the coupled 5x5 line blocks: the mean flow solved first, then
    the SA chains with the right-hand side ``r_sa - C z_flow`` (block forward
    substitution of the block lower-triangular blocks)."""
    split = precondition(U, lam, cfl, model)
    ch = model.plan.chains
    valid = ch.cells >= 0
    found = np.full(model.plan.n_canvas, -1, dtype=np.int64)
    found[ch.cells[valid]] = np.flatnonzero(valid)
    lower, upper = chain_coupling_sa(U, model)
    sa_factor = cr_factor(*chain_blocks_sa(U, lam, cfl, model))

    def apply(r):
        z = split(r)
        zf = np.where(valid, _gather(z[:4], ch), 0.0)                       # (4, n_lines, L)
        zf = np.transpose(zf, (2, 1, 0))                                     # (L, n_lines, 4)
        below = np.concatenate([np.zeros_like(zf[:1]), zf[:-1]], axis=0)
        above = np.concatenate([zf[1:], np.zeros_like(zf[:1])], axis=0)
        cz = np.sum(lower * below, axis=-1) + np.sum(upper * above, axis=-1)   # (L, n_lines)
        rhs = np.where(valid, _gather(r[4:5], ch), 0.0)[0].T - cz
        x = cr_solve(sa_factor, rhs[:, :, None])[:, :, 0].T                # (n_lines, L)
        out = z.copy()
        flat = out[4].reshape(-1)
        flat[ch.cells[valid]] = x[valid]
        out[4] = flat.reshape(out[4].shape)
        return out

    return apply


# --- GMRES (krylov.py:34-137) ---------------------------------------------------------


def hessenberg_lstsq(H, beta, rcond):
    m = H.shape[1]
    h = [[H[i, j] for j in range(m)] for i in range(m + 1)]
    g = [beta] + [0.0] * m
    cs, sn = [], []
    for j in range(m):
        for i in range(j):
            a, c = h[i][j], h[i + 1][j]
            h[i][j], h[i + 1][j] = cs[i] * a + sn[i] * c, cs[i] * c - sn[i] * a
        a, c = h[j][j], h[j + 1][j]
        r = np.sqrt(a * a + c * c)
        safe = r if r > 0 else 1.0
        cs.append(a / safe if r > 0 else 1.0)
        sn.append(c / safe if r > 0 else 0.0)
        h[j][j], h[j + 1][j] = r, 0.0
        g[j], g[j + 1] = cs[j] * g[j], -sn[j] * g[j]
    piv = [abs(h[j][j]) for j in range(m)]
    largest = max(piv)
    y = [0.0] * m
    for j in reversed(range(m)):
        rest = g[j]
        for k in range(j + 1, m):
            rest = rest - h[j][k] * y[k]
        y[j] = rest / h[j][j] if piv[j] > rcond * largest else 0.0
    return np.array(y)


def gmres_right(matvec, b, prec, restart, maxiter, tol):
    """Restarted right-preconditioned GMRES with CGS2; returns ``(x, A x)``
    with the action from the Arnoldi relation."""
    bn = np.linalg.norm(b)
    tiny = np.finfo(np.float64).tiny
    rcond = float(np.finfo(np.float64).eps) * (restart + 1)
    x = np.zeros_like(b)
    r = b.copy()
    action = np.zeros_like(b)
    k = 0
    while k < maxiter and np.linalg.norm(r) > tol * bn:
        beta = np.linalg.norm(r)
        V = np.zeros((restart + 1,) + b.shape)
        V[0] = r / max(beta, tiny)
        H = np.zeros((restart + 1, restart))
        for j in range(restart):
            w = matvec(prec(V[j]))
            active = (np.arange(restart + 1) <= j).astype(np.float64)
            h = np.tensordot(V, w, axes=w.ndim) * active
            w = w - np.tensordot(h, V, axes=1)
            h2 = np.tensordot(V, w, axes=w.ndim) * active
            w = w - np.tensordot(h2, V, axes=1)
            h = h + h2
            nrm = np.linalg.norm(w)
            h[j + 1] = nrm
            H[:, j] = h
            V[j + 1] = w / max(nrm, tiny)
        y = hessenberg_lstsq(H, beta, rcond)
        x = x + prec(np.tensordot(y, V[:restart], axes=1))
        action = action + np.tensordot(H @ y, V, axes=1)
        r = b - action
        k += 1
    return x, action


# --- the Newton step (implicit.py:35-168) ----------------------------------------------


@dataclass
class NewtonState:
    U: np.ndarray
    cfl: float
    residual_norm: float


def relax(dU, U, g, fraction):
    if fraction is None:
        return dU, 1.0
    rho = U[0]
    u, v = U[1] / rho, U[2] / rho
    p = (g - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v))
    d_e = dU[3] - u * dU[1] - v * dU[2]
    d_p = (g - 1.0) * (d_e + 0.5 * (u * u + v * v) * dU[0])
    ratios = [np.abs(dU[0]) / rho, np.abs(d_p) / p]
    if U.shape[0] > 4:
        nh = U[4] / rho
        dnh = (dU[4] - nh * dU[0]) / rho
        ratios.append(np.abs(dnh) / np.maximum(np.abs(nh), 1.0))
    worst = max(float(np.max(r)) for r in ratios)
    omega = min(1.0, fraction / max(worst, 1e-300))
    return omega * dU, omega


def is_physical(U, g):
    rho = U[0]
    u, v = U[1] / rho, U[2] / rho
    p = (g - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v))
    return (rho > 1e-10) & (p > 1e-10) & np.isfinite(rho) & np.isfinite(p)


def newton_step(state: NewtonState, model, config, solver: str = "cr"):
    """One pseudo-transient Newton step with the first-order Jacobian (defect
    correction); returns ``(state, |R| before the update)``."""
    U, cfl = state.U, state.cfl
    R = nm.residual(U, model)
    norm = nm.norm(R, model)
    lam = nm.wave_speeds(U, model)
    vdt = nm.cell_sum(lam) / cfl
    prec = precondition(U, lam, cfl, model, solver) if config.preconditioner == "line_j" else (lambda r: r)

    def matvec(d):
        return vdt[None] * d + nm.jvp(U, d, model)

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
