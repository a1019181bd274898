// The 3D pseudo-transient Newton step: right-preconditioned restarted GMRES with CGS2
// and Givens least squares (src/jaxrans/solvers/krylov.py:34-137), the relaxation, the
// acceptance test and the CFL ramp (src/jaxrans/solvers/implicit.py:54-168), driven on
// the host over vector operations `Ops` supplies.  On the device (capi3d.cu) the
// operations are kernels; a test-only host harness supplies loops, so this logic is
// checked against the reference without a GPU.
#pragma once
#include <cmath>
#include <vector>

namespace jr {

constexpr int MAX_RESTART3 = 64;   // krylov_subspace at most

struct Newton3Config {
  int restart, maxiter, preconditioner;   // preconditioner 0 none, 1 line_j, 2 line_j coupled
  double tol, success, max_relative_update;   // max_relative_update <= 0: none
  double cfl_min, cfl_max, cfl_growth, cfl_cutback;
};

// argmin |beta e1 - H y| by Givens rotations; pivots below rcond * the largest dropped
inline void givens_lstsq(const std::vector<double>& Hc, int m, double beta, double rcond, std::vector<double>& y) {
  // Hc: (m+1) x m, row-major
  std::vector<double> h(Hc), g(m + 1, 0.0), cs(m), sn(m);
  g[0] = beta;
  for (int j = 0; j < m; ++j) {
    for (int i = 0; i < j; ++i) {
      const double a = h[i * m + j], c = h[(i + 1) * m + j];
      h[i * m + j] = cs[i] * a + sn[i] * c;
      h[(i + 1) * m + j] = cs[i] * c - sn[i] * a;
    }
    const double a = h[j * m + j], c = h[(j + 1) * m + j];
    const double r = std::sqrt(a * a + c * c);
    const double safe = r > 0.0 ? r : 1.0;
    cs[j] = r > 0.0 ? a / safe : 1.0;
    sn[j] = r > 0.0 ? c / safe : 0.0;
    h[j * m + j] = r;
    h[(j + 1) * m + j] = 0.0;
    const double gj = g[j];
    g[j] = cs[j] * gj;
    g[j + 1] = -sn[j] * gj;
  }
  double largest = 0.0;
  for (int j = 0; j < m; ++j) largest = std::fmax(largest, std::fabs(h[j * m + j]));
  y.assign(m, 0.0);
  for (int j = m - 1; j >= 0; --j) {
    double rest = g[j];
    for (int k = j + 1; k < m; ++k) rest = rest - h[j * m + k] * y[k];
    y[j] = std::fabs(h[j * m + j]) > rcond * largest ? rest / h[j * m + j] : 0.0;
  }
}

// Ops: vectors by index -- R_, Z_, W_, T_ (GMRES work), RES_, B_, DU_, ACT_ (the step's),
// V(i) the basis -- each of the canvas length N = nvar * cells; the state U is the
// caller's.  Operations: prepare(U, cfl) (V/dt, the line factor), residual, matvec
// (V/dt z + J1 z), precondition, dot, mdot (the dots of V(0..count-1) with a vector, as
// that many dots), maxpy (y += sum of coef_i V(i), as that many axpys in order), nrm2,
// axpy, scale, copy, zero, density_norm, worst_ratio, physical_after, add_to_state.
template <class Ops>
int gmres3(Ops& ops, const double* U, double cfl, const Newton3Config& c, int B, int X, int ACTION) {
  // solves (V/dt + J) X = B; ACTION = the Arnoldi action A X
  const double tiny = 2.2250738585072014e-308;
  const double rcond = 2.220446049250313e-16 * (c.restart + 1);
  const int m = c.restart;
  auto prec = [&](int src, int dst) {
    if (c.preconditioner >= 1) ops.precondition(U, cfl, src, dst);
    else ops.copy(src, dst);
  };
  const double bn = ops.nrm2(B);
  ops.zero(X);
  ops.copy(B, Ops::R_);
  ops.zero(ACTION);
  std::vector<double> H((size_t)(m + 1) * m), h(m + 1), h2(m + 1), neg(m + 1), y, Hy(m + 1);
  for (int k = 0; k < c.maxiter; ++k) {
    const double rn = ops.nrm2(Ops::R_);
    if (!(rn > c.tol * bn)) break;
    const double beta = rn;
    ops.scale(1.0 / std::fmax(beta, tiny), Ops::R_, ops.V(0));
    std::fill(H.begin(), H.end(), 0.0);
    for (int j = 0; j < m; ++j) {
      prec(ops.V(j), Ops::Z_);
      ops.matvec(U, cfl, Ops::Z_, Ops::W_);
      ops.mdot(j + 1, Ops::W_, h.data());
      for (int i = 0; i <= j; ++i) neg[i] = -h[i];
      ops.maxpy(j + 1, neg.data(), Ops::W_);
      ops.mdot(j + 1, Ops::W_, h2.data());
      for (int i = 0; i <= j; ++i) neg[i] = -h2[i];
      ops.maxpy(j + 1, neg.data(), Ops::W_);
      const double nrm = ops.nrm2(Ops::W_);
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = h[i] + h2[i];
      H[(size_t)(j + 1) * m + j] = nrm;
      ops.scale(1.0 / std::fmax(nrm, tiny), Ops::W_, ops.V(j + 1));
    }
    givens_lstsq(H, m, beta, rcond, y);
    ops.zero(Ops::T_);
    ops.maxpy(m, y.data(), Ops::T_);
    prec(Ops::T_, Ops::Z_);
    ops.axpy(1.0, Ops::Z_, X);
    for (int i = 0; i <= m; ++i) {
      double s = 0.0;
      for (int j = 0; j < m; ++j) s = s + H[(size_t)i * m + j] * y[j];
      Hy[i] = s;
    }
    ops.maxpy(m + 1, Hy.data(), ACTION);
    ops.copy(B, Ops::R_);
    ops.axpy(-1.0, ACTION, Ops::R_);
  }
  return 0;
}

// One Newton step on the state (U in place); returns |R| before the update.
template <class Ops>
double newton_step3(Ops& ops, double* U, double& cfl, double& res_prev, const Newton3Config& c) {
  ops.prepare(U, cfl);   // V/dt at (U, cfl), for the matrix-vector products of this step
  ops.residual(U, Ops::RES_);
  const double norm = ops.density_norm(Ops::RES_);
  ops.scale(-1.0, Ops::RES_, Ops::B_);
  gmres3(ops, U, cfl, c, Ops::B_, Ops::DU_, Ops::ACT_);
  double omega = 1.0;
  if (c.max_relative_update > 0.0) {
    const double worst = ops.worst_ratio(U, Ops::DU_);
    omega = std::fmin(1.0, c.max_relative_update / std::fmax(worst, 1e-300));
    ops.scale(omega, Ops::DU_, Ops::DU_);
  }
  ops.scale(omega, Ops::ACT_, Ops::T_);
  ops.axpy(1.0, Ops::RES_, Ops::T_);
  const double lin = ops.nrm2(Ops::T_) / std::fmax(ops.nrm2(Ops::RES_), 1e-300);
  const bool physical = ops.physical_after(U, Ops::DU_);
  const bool accept = physical && lin < 1.0;
  const double reduction = res_prev / std::fmax(norm, 1e-300);
  double next;
  if (accept && lin < c.success && omega >= 1.0) next = cfl * std::fmin(std::fmax(reduction, 1.0), c.cfl_growth);
  else if (accept) next = cfl;
  else next = cfl / c.cfl_cutback;
  if (accept) {
    ops.add_to_state(U, Ops::DU_);
    res_prev = norm;
  }
  cfl = std::fmin(std::fmax(next, c.cfl_min), c.cfl_max);
  return norm;
}

}  // namespace jr
