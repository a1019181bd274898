"""Properties the reference's own unit tests pin, checked on the oracle (the checker
the device path is compared with):

* flux consistency, conservation and an exact stationary contact for HLLC and Roe
  (tests/unit/test_riemann.py:35-223 of the reference);
* every limiter of equal differences returns them (tests/unit/test_limiters.py:27-40);
* the diamond face gradient exact for a linear field on a skewed, stretched grid
  (tests/unit/test_viscous.py:58-72);
* cyclic reduction = block Thomas = a dense solve (tests/unit/test_linalg.py:114-128,
  tests/unit/test_preconditioners.py:85-109);
* GMRES solving a small system to its tolerance, the action from the Arnoldi relation
  equal to A x (tests/unit/test_krylov.py:19-93);
* freestream preserved off the wall for every flux x limiter, first order too
  (tests/verification/test_freestream.py:49-113).
"""

from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from goldens import load, oracle_model
from oracle import implicit as im
from oracle import numerics as nm

G = 1.4


def states(rng, n):
    rho = rng.uniform(0.5, 2.0, n)
    u, v = rng.uniform(-0.6, 0.6, n), rng.uniform(-0.6, 0.6, n)
    p = rng.uniform(0.4, 1.5, n)
    return np.stack([rho, u, v, p])


@pytest.mark.parametrize("flux", [nm.hllc_flux, nm.roe_flux])
def test_flux_of_equal_states_is_the_physical_flux(flux):
    rng = np.random.default_rng(1)
    q = states(rng, 200)
    sx, sy = rng.normal(size=200), rng.normal(size=200)
    length = np.hypot(sx, sy)
    exact = length * nm.normal_flux(q, sx / length, sy / length, G)
    assert np.allclose(flux(q, q, sx, sy, G), exact, rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("flux", [nm.hllc_flux, nm.roe_flux])
def test_flux_is_conservative(flux):
    """The flux leaving one cell enters its neighbour: F(L, R, S) = -F(R, L, -S)."""
    rng = np.random.default_rng(2)
    qL, qR = states(rng, 200), states(rng, 200)
    sx, sy = rng.normal(size=200), rng.normal(size=200)
    assert np.allclose(flux(qL, qR, sx, sy, G), -flux(qR, qL, -sx, -sy, G), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("flux", [nm.hllc_flux, nm.roe_flux])
def test_stationary_contact_is_exact(flux):
    """Equal pressure, zero normal velocity, any density and tangential velocity jump:
    no mass or energy crosses, the momentum flux is the pressure."""
    rng = np.random.default_rng(3)
    n = 100
    sx, sy = rng.normal(size=n), rng.normal(size=n)
    length = np.hypot(sx, sy)
    nx, ny = sx / length, sy / length
    tL, tR = rng.uniform(-0.5, 0.5, n), rng.uniform(-0.5, 0.5, n)
    p = rng.uniform(0.5, 1.5, n)
    qL = np.stack([rng.uniform(0.5, 2.0, n), -tL * ny, tL * nx, p])
    qR = np.stack([rng.uniform(0.5, 2.0, n), -tR * ny, tR * nx, p])
    F = flux(qL, qR, sx, sy, G)
    assert np.abs(F[0]).max() < 1e-13 and np.abs(F[3]).max() < 1e-13
    assert np.allclose(F[1], p * sx, atol=1e-13) and np.allclose(F[2], p * sy, atol=1e-13)


@pytest.mark.parametrize("name", ["none", "minmod", "van_albada", "van_albada_smooth"])
def test_limiter_of_equal_differences(name):
    a = np.random.default_rng(4).normal(size=500)
    assert np.allclose(nm.limit(a, a, name), a, rtol=1e-14, atol=0.0)
    assert np.all(nm.limit(a, -a, name) == 0.0) or name in ("none", "van_albada_smooth")


def test_diamond_gradient_is_exact_for_linear_fields():
    """Centres of a skewed, stretched grid (one ghost ring); phi linear in x, y."""
    ni, nj = 9, 7
    s = np.cumsum(np.linspace(1.0, 2.5, nj + 2))
    i, j = np.meshgrid(np.arange(ni + 2, dtype=float), s, indexing="ij")
    x = i + 0.3 * j + 0.05 * i * i
    y = 0.2 * i + j
    centres = np.stack([x, y])
    c = np.array([[0.7, -1.3], [2.0, 0.4], [-0.5, 0.9]])          # (nphi, 2)
    phi = np.stack([1.0 + c[k, 0] * x + c[k, 1] * y for k in range(3)])
    for G_ in nm.face_gradients(phi, centres):
        for k in range(3):
            assert np.allclose(G_[0, k], c[k, 0], rtol=0, atol=1e-11)
            assert np.allclose(G_[1, k], c[k, 1], rtol=0, atol=1e-11)


def _block_system(rng, L, n, m):
    lower = rng.normal(size=(L, n, m, m)) * 0.2
    upper = rng.normal(size=(L, n, m, m)) * 0.2
    lower[0] = 0.0
    upper[-1] = 0.0
    diag = rng.normal(size=(L, n, m, m)) * 0.2 + 3.0 * np.eye(m)
    return lower, diag, upper


@pytest.mark.parametrize("L", [1, 2, 7, 16, 33])
def test_cyclic_reduction_equals_thomas_and_a_dense_solve(L):
    rng = np.random.default_rng(L)
    n, m = 3, 4
    lower, diag, upper = _block_system(rng, L, n, m)
    rhs = rng.normal(size=(L, n, m))
    x_cr = im.cr_solve(im.cr_factor(lower, diag, upper), rhs)
    x_th = im.thomas_solve(im.thomas_factor(lower, diag, upper), rhs)
    assert np.allclose(x_cr, x_th, rtol=1e-12, atol=1e-12)
    for c in range(n):
        A = np.zeros((L * m, L * m))
        for k in range(L):
            A[k * m:(k + 1) * m, k * m:(k + 1) * m] = diag[k, c]
            if k > 0:
                A[k * m:(k + 1) * m, (k - 1) * m:k * m] = lower[k, c]
            if k < L - 1:
                A[k * m:(k + 1) * m, (k + 1) * m:(k + 2) * m] = upper[k, c]
        dense = np.linalg.solve(A, rhs[:, c].reshape(-1)).reshape(L, m)
        assert np.allclose(x_cr[:, c], dense, rtol=1e-12, atol=1e-12)


def test_gmres_solves_to_its_tolerance():
    rng = np.random.default_rng(9)
    n = 40
    A = np.eye(n) * 4.0 + rng.normal(size=(n, n)) * 0.3
    b = rng.normal(size=n)
    x, action = im.gmres_right(lambda d: A @ d, b, lambda r: r, restart=10, maxiter=8, tol=1e-10)
    assert np.linalg.norm(b - A @ x) <= 1e-10 * np.linalg.norm(b) * 10
    assert np.allclose(action, A @ x, rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("flux", ["hllc", "roe"])
@pytest.mark.parametrize("limiter", ["none", "minmod", "van_albada", "van_albada_smooth"])
@pytest.mark.parametrize("first_order", [False, True])
def test_freestream_is_preserved(flux, limiter, first_order):
    """A uniform state leaves no residual away from the wall (the face vectors of every
    cell close; the far field returns the freestream)."""
    z, case, plan = load("c_laminar")
    model = replace(oracle_model(case, plan), flux=flux, limiter=limiter)
    R = nm.residual(model.U0, model, first_order)
    away = plan.interior & (np.hypot(*(plan.centres[:, 1:-1, 1:-1] - 0.5)) > 3.0)
    assert np.abs(R[:, away]).max() < 1e-12
