// The 3D wave speeds and line preconditioner, per-face and per-chain bodies (host and
// device code; linesolve3d.cu launches them, one thread each): the reference's
// face_wave_speeds (src/jaxrans/numerics/residual.py:169-203) and line_j
// (src/jaxrans/solvers/preconditioners.py:209-306) on a 3D plan -- 5x5 mean-flow chain
// blocks, the SA row on its own scalar chains -- solved along each chain by the block
// Thomas algorithm (src/jaxrans/core/linalg.py:80-132).  A first form: one thread walks
// a chain, its blocks assembled as it goes, the eliminated blocks kept in scratch.
#pragma once
#include "residual3d.cuh"

namespace jr {


// primitive state of canvas cell c straight from U (no ghost fill)
__host__ __device__ __forceinline__ void prim_at(const Plan3Dev& p, const double* U, int c, double q[NV3_MAX]) {
  const int n = p.NI * p.NJ * p.NK;
  double u[NV3_MAX];
  for (int v = 0; v < p.nvar; ++v) u[v] = U[(size_t)v * n + c];
  to_prim3(u, q, p.nvar, p.P.gamma);
}

// the two cells either side of face (a, i, j, k), each replaced by its partner across a
// block face (the neighbour map), the canvas edge repeated
__host__ __device__ __forceinline__ void face_cells(const Plan3Dev& p, int a, int i, int j, int k, int& lo, int& hi) {
  int l[3] = {i, j, k}, h[3] = {i, j, k};
  l[a] -= 1;
  lo = p.neighbours[cell_index(p, l[0], l[1], l[2])];
  hi = p.neighbours[cell_index(p, h[0], h[1], h[2])];
}

// face-averaged primitive state and volume (src/jaxrans/mesh/atlas.py:169-183)
__host__ __device__ __forceinline__ void face_average(const Plan3Dev& p, const double* U, int a, int i, int j, int k,
                                                      double qf[NV3_MAX], double& vol) {
  int lo, hi;
  face_cells(p, a, i, j, k, lo, hi);
  double ql[NV3_MAX], qh[NV3_MAX];
  prim_at(p, U, lo, ql);
  prim_at(p, U, hi, qh);
  for (int v = 0; v < p.nvar; ++v) qf[v] = 0.5 * (ql[v] + qh[v]);
  vol = 0.5 * (p.volume[lo] + p.volume[hi]);
}

// lambda = |V.S| + a|S| at the face-averaged state, plus the thin-layer viscous term
__host__ __device__ __forceinline__ double wave_speed(const Plan3Dev& p, const double* U, int a, int i, int j, int k) {
  const Physics3& P = p.P;
  const double g = P.gamma;
  double qf[NV3_MAX], vol, s[3];
  face_average(p, U, a, i, j, k, qf, vol);
  face_vector(p, a, i, j, k, s);
  const double ss = (s[0] * s[0] + s[1] * s[1]) + s[2] * s[2];
  double vn = (qf[1] * s[0] + qf[2] * s[1]) + qf[3] * s[2];
  double lam = (vn >= 0.0 ? vn : -vn) + sqrt(g * qf[4] / qf[0]) * sqrt(ss);
  if (P.mu_inf > 0.0) {
    double mu = viscosity3(P, g * qf[4] / qf[0]);
    if (p.nvar > 5) mu = mu + eddy_viscosity(P.sa, qf[0], qf[5] * P.mu_inf, mu / qf[0]);
    lam = lam + 2.0 * g / PR_LAMINAR * mu * ss / (qf[0] * vol);
  }
  return lam;
}

// sum over the cell's six faces of lambda (the order of cell_wave_speed_sum)
__host__ __device__ __forceinline__ double lambda_sum(const Plan3Dev& p, const double* U, int c) {
  const int i = c / (p.NJ * p.NK), j = (c / p.NK) % p.NJ, k = c % p.NK;
  double total = 0.0;
  for (int a = 0; a < 3; ++a) {
    int h[3] = {i, j, k};
    h[a] += 1;
    const double lo = wave_speed(p, U, a, i, j, k), hi = wave_speed(p, U, a, h[0], h[1], h[2]);
    total = a == 0 ? lo + hi : total + lo + hi;
  }
  return total;
}

// A = d(F . S)/dU (5x5, [row][variable]) by forward-mode tangents of the flux of the
// conservative state (src/jaxrans/physics/euler.py:55-71)
__host__ __device__ __forceinline__ void flux_jacobian3(const double* q, const double* s, double g, double A[5][5]) {
  double U[5];
  U[0] = q[0];
  U[1] = q[0] * q[1];
  U[2] = q[0] * q[2];
  U[3] = q[0] * q[3];
  U[4] = q[4] / (g - 1.0) + 0.5 * q[0] * ((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]);
  for (int col = 0; col < 5; ++col) {
    Dual Ud[5], qd[5], F[5];
    for (int v = 0; v < 5; ++v) Ud[v] = Dual{U[v], v == col ? 1.0 : 0.0};
    to_prim3(Ud, qd, 5, g);
    normal_flux3(qd, s, g, F);
    for (int r = 0; r < 5; ++r) A[r][col] = F[r].d;
  }
}

// unpivoted Gauss-Jordan inverse (src/jaxrans/core/linalg.py:49-77)
template <int M> __host__ __device__ __forceinline__ void invert_n(const double Mx[M][M], double Inv[M][M]) {
  double a[M][2 * M];
  for (int r = 0; r < M; ++r)
    for (int c = 0; c < M; ++c) {
      a[r][c] = Mx[r][c];
      a[r][M + c] = r == c ? 1.0 : 0.0;
    }
  for (int k = 0; k < M; ++k) {
    const double piv = a[k][k];
    for (int c = 0; c < 2 * M; ++c) a[k][c] = a[k][c] / piv;
    for (int r = 0; r < M; ++r) {
      if (r == k) continue;
      const double f = a[r][k];
      for (int c = 0; c < 2 * M; ++c) a[r][c] = a[r][c] - f * a[k][c];
    }
  }
  for (int r = 0; r < M; ++r)
    for (int c = 0; c < M; ++c) Inv[r][c] = a[r][M + c];
}

// the link k -> k+1 of a chain: its face vector (outward from cell k) and lambda there
__host__ __device__ __forceinline__ void link_face(const Plan3Dev& p, const double* U, int flat, double s[3],
                                                   double& lam) {
  int a, i, j, k;
  face_of(p, flat, a, i, j, k);
  face_vector(p, a, i, j, k, s);
  lam = wave_speed(p, U, a, i, j, k);
}

// 1/2 A(q_nb, sign S) - 1/2 lambda I
__host__ __device__ __forceinline__ void coupling5(const double* qnb, const double* s, double sign, double lam,
                                                   double g, double B[5][5]) {
  const double ss[3] = {sign * s[0], sign * s[1], sign * s[2]};
  double A[5][5];
  flux_jacobian3(qnb, ss, g, A);
  for (int r = 0; r < 5; ++r)
    for (int c = 0; c < 5; ++c) B[r][c] = 0.5 * A[r][c] - (r == c ? 0.5 * lam : 0.0);
}

// The line_j factor of one chain (block Thomas, src/jaxrans/core/linalg.py:80-132, and the
// scalar SA chain): for element k of the chain, the block toward k-1 (lower_k), the
// inverse pivot P_k = (D_k - lower_k C_{k-1})^-1 and C_k = P_k upper_k -- 75 entries -- and
// on the SA row the same three scalars.  Entry e of element k of chain ch is stored at
// F[(k * FACTOR3 + e) * n_chains + ch]: neighbouring chains' threads read neighbouring
// words.  The apply is then z_k = P_k (r_k - lower_k d_{k-1}) down the chain and
// x_k = d_k - C_k x_{k+1} back up, the factor computed once per Newton step.
constexpr int F3_LOWER = 0, F3_PIV = 25, F3_CHAT = 50, F3_SA = 75, F3_CPL_LO = 78, F3_CPL_UP = 83;

// the SA row's coupling to a neighbour's mean flow: half the Jacobian of rho nu_hat V.S'
// with respect to its (rho, rho u, rho v, rho w, rho E) at its state qnb, S' = sign S:
// [-nu_hat vn, nu_hat S'x, nu_hat S'y, nu_hat S'z, 0]
__host__ __device__ __forceinline__ void sa_coupling_row(const double* qnb, const double* s, double sign,
                                                         double row[5]) {
  const double sx = sign * s[0], sy = sign * s[1], sz = sign * s[2];
  const double nu = qnb[5];
  const double vn = qnb[1] * sx + qnb[2] * sy + qnb[3] * sz;
  row[0] = 0.5 * (-nu * vn);
  row[1] = 0.5 * (nu * sx);
  row[2] = 0.5 * (nu * sy);
  row[3] = 0.5 * (nu * sz);
  row[4] = 0.5 * 0.0;
}

__host__ __device__ __forceinline__ size_t factor_at(const Plan3Dev& p, int ch, int k, int e) {
  return ((size_t)k * FACTOR3 + e) * p.n_chains + ch;
}

__host__ __device__ __forceinline__ int chain_length(const Plan3Dev& p, int ch) {
  const int* cells = p.ch_cells + (size_t)ch * p.chain_L;
  int len = 0;
  while (len < p.chain_L && cells[len] >= 0) ++len;
  return len;
}

template <class TF>
inline __host__ __device__ void chain_factor_flow(const Plan3Dev& p, const double* U, double cfl, int ch, TF* F) {
  const int L = p.chain_L;
  const double g = p.P.gamma;
  const int* cells = p.ch_cells + (size_t)ch * L;
  const int len = chain_length(p, ch);
  double cprev[5][5] = {};
  double lower[5][5] = {};   // row k's block toward cell k-1
  double cpl_lower[5] = {};  // the coupled form: the SA row k's coupling to cell k-1's mean flow
  for (int k = 0; k < len; ++k) {
    const int c = cells[k];
    const double dg = lambda_sum(p, U, c) * (1.0 / cfl + 0.5);
    double upper[5][5] = {}, lower_next[5][5] = {};
    double cpl_upper[5] = {}, cpl_lower_next[5] = {};
    const int sign = k + 1 < len ? p.ch_sign[(size_t)ch * L + k] : 0;
    if (sign != 0) {
      double s[3], lam, qn[NV3_MAX], qc[NV3_MAX];
      link_face(p, U, p.ch_face[(size_t)ch * L + k], s, lam);
      prim_at(p, U, cells[k + 1], qn);
      prim_at(p, U, c, qc);
      coupling5(qn, s, (double)sign, lam, g, upper);
      coupling5(qc, s, (double)-sign, lam, g, lower_next);
      if (p.line_coupled && p.nvar > 5) {
        sa_coupling_row(qn, s, (double)sign, cpl_upper);
        sa_coupling_row(qc, s, (double)-sign, cpl_lower_next);
      }
    }
    if (p.line_coupled && p.nvar > 5)
      for (int t = 0; t < 5; ++t) {
        F[factor_at(p, ch, k, F3_CPL_LO + t)] = (TF)cpl_lower[t];
        F[factor_at(p, ch, k, F3_CPL_UP + t)] = (TF)cpl_upper[t];
        cpl_lower[t] = cpl_lower_next[t];
      }
    // P = inv(D - lower c_prev); chat = P upper
    double T[5][5], piv[5][5];
    for (int a = 0; a < 5; ++a)
      for (int b = 0; b < 5; ++b) {
        double m = lower[a][0] * cprev[0][b];
        for (int t = 1; t < 5; ++t) m = m + lower[a][t] * cprev[t][b];
        T[a][b] = (a == b ? dg : 0.0) - m;
      }
    invert_n<5>(T, piv);
    for (int a = 0; a < 5; ++a)
      for (int b = 0; b < 5; ++b) {
        double m = piv[a][0] * upper[0][b];
        for (int t = 1; t < 5; ++t) m = m + piv[a][t] * upper[t][b];
        cprev[a][b] = m;
        F[factor_at(p, ch, k, F3_LOWER + a * 5 + b)] = (TF)lower[a][b];
        F[factor_at(p, ch, k, F3_PIV + a * 5 + b)] = (TF)piv[a][b];
        F[factor_at(p, ch, k, F3_CHAT + a * 5 + b)] = (TF)m;
      }
    for (int a = 0; a < 5; ++a)
      for (int b = 0; b < 5; ++b) lower[a][b] = lower_next[a][b];
  }
}

// z = M^-1 r on the mean-flow rows of chain ch from its factor; d_k is kept in z between
// the two sweeps
template <class TF>
inline __host__ __device__ void chain_apply_flow(const Plan3Dev& p, int ch, const TF* F, const double* r, double* z) {
  const int n = p.NI * p.NJ * p.NK;
  const int* cells = p.ch_cells + (size_t)ch * p.chain_L;
  const int len = chain_length(p, ch);
  TF dprev[5] = {};
  for (int k = 0; k < len; ++k) {
    const int c = cells[k];
    TF rhs[5];
    for (int a = 0; a < 5; ++a) {
      TF m = F[factor_at(p, ch, k, F3_LOWER + a * 5)] * dprev[0];
      for (int t = 1; t < 5; ++t) m = m + F[factor_at(p, ch, k, F3_LOWER + a * 5 + t)] * dprev[t];
      rhs[a] = (TF)r[(size_t)a * n + c] - m;
    }
    for (int a = 0; a < 5; ++a) {
      TF m = F[factor_at(p, ch, k, F3_PIV + a * 5)] * rhs[0];
      for (int t = 1; t < 5; ++t) m = m + F[factor_at(p, ch, k, F3_PIV + a * 5 + t)] * rhs[t];
      dprev[a] = m;
      z[(size_t)a * n + c] = (double)m;
    }
  }
  TF nxt[5] = {};
  for (int k = len - 1; k >= 0; --k) {
    const int c = cells[k];
    TF x[5];
    for (int a = 0; a < 5; ++a) {
      TF m = F[factor_at(p, ch, k, F3_CHAT + a * 5)] * nxt[0];
      for (int t = 1; t < 5; ++t) m = m + F[factor_at(p, ch, k, F3_CHAT + a * 5 + t)] * nxt[t];
      x[a] = (TF)z[(size_t)a * n + c] - m;
    }
    for (int a = 0; a < 5; ++a) {
      nxt[a] = x[a];
      z[(size_t)a * n + c] = (double)x[a];
    }
  }
}

// the SA row's face terms at face (a, i, j, k): mass flux rho V.S and diffusion kappa |S|^2 / V
__host__ __device__ __forceinline__ void sa_face_terms(const Plan3Dev& p, const double* U, int a, int i, int j, int k,
                                                       double& m, double& d) {
  const Physics3& P = p.P;
  double qf[NV3_MAX], vol, s[3];
  face_average(p, U, a, i, j, k, qf, vol);
  face_vector(p, a, i, j, k, s);
  const double mu = viscosity3(P, P.gamma * qf[4] / qf[0]);
  const double kap = diffusion_coefficient(P.sa, qf[0], qf[5] * P.mu_inf, mu);
  m = qf[0] * ((qf[1] * s[0] + qf[2] * s[1]) + qf[3] * s[2]);
  d = kap * ((s[0] * s[0] + s[1] * s[1]) + s[2] * s[2]) / vol;
}

// the SA chain diagonal of cell c (src/jaxrans/solvers/preconditioners.py:235-270)
inline __host__ __device__ double sa_diagonal(const Plan3Dev& p, const double* U, double cfl, int c) {
  const Physics3& P = p.P;
  const double g = P.gamma;
  const int i = c / (p.NJ * p.NK), j = (c / p.NK) % p.NJ, k = c % p.NK;
  double diag = 0.0;
  double gv[3][3];   // Green-Gauss of face-averaged velocity: gv[direction][component]
  for (int dir = 0; dir < 3; ++dir)
    for (int m = 0; m < 3; ++m) gv[dir][m] = 0.0;
  double vsum[3][3][3];   // per family: hi*S_hi - lo*S_lo, [family][direction][component]
  for (int a = 0; a < 3; ++a) {
    int h[3] = {i, j, k};
    h[a] += 1;
    double mlo, dlo, mhi, dhi;
    sa_face_terms(p, U, a, i, j, k, mlo, dlo);
    sa_face_terms(p, U, a, h[0], h[1], h[2], mhi, dhi);
    const double out_hi = (mhi > 0.0 ? mhi : 0.0) + dhi;
    const double in_lo = (-mlo > 0.0 ? -mlo : 0.0) + dlo;
    diag = a == 0 ? out_hi + in_lo : diag + out_hi + in_lo;
    double ql[NV3_MAX], qh[NV3_MAX], vl, vh, sl[3], sh[3];
    face_average(p, U, a, i, j, k, ql, vl);
    face_average(p, U, a, h[0], h[1], h[2], qh, vh);
    face_vector(p, a, i, j, k, sl);
    face_vector(p, a, h[0], h[1], h[2], sh);
    for (int dir = 0; dir < 3; ++dir)
      for (int m = 0; m < 3; ++m) vsum[a][dir][m] = qh[1 + m] * sh[dir] - ql[1 + m] * sl[dir];
  }
  const double vol = p.volume[c];
  for (int dir = 0; dir < 3; ++dir)
    for (int m = 0; m < 3; ++m) gv[dir][m] = ((vsum[0][dir][m] + vsum[1][dir][m]) + vsum[2][dir][m]) / vol;
  double q[NV3_MAX];
  prim_at(p, U, c, q);
  diag = diag / q[0];
  const double cx = gv[1][2] - gv[2][1], cy = gv[2][0] - gv[0][2], cz = gv[0][1] - gv[1][0];
  const double sq = (cx * cx + cy * cy) + cz * cz;
  const double omega = sq > 0.0 ? sqrt(sq) : 0.0;
  const double nu = viscosity3(P, g * q[4] / q[0]) / q[0];
  const double dist = p.distance[c];
  const double st = s_tilde(P.sa, omega, q[5] * P.mu_inf, nu, dist);
  const double fw = f_w(P.sa, r_of(P.sa, q[5] * P.mu_inf, st, dist));
  const double dest = q[5] > 0.0 ? 2.0 * P.sa.c_w1 * fw * P.mu_inf * q[5] / (dist * dist) : 0.0;
  return diag + dest * vol + lambda_sum(p, U, c) / cfl;
}

// the SA row's factor of chain ch (scalar Thomas): lower_k, 1 / (d_k - lower_k c_{k-1}), c_k
template <class TF>
inline __host__ __device__ void chain_factor_sa(const Plan3Dev& p, const double* U, double cfl, int ch, TF* F) {
  const int L = p.chain_L;
  const int* cells = p.ch_cells + (size_t)ch * L;
  const int len = chain_length(p, ch);
  double cprev = 0.0, lower = 0.0;
  for (int k = 0; k < len; ++k) {
    const int c = cells[k];
    const double dg = sa_diagonal(p, U, cfl, c);
    double upper = 0.0, lower_next = 0.0;
    const int sign = k + 1 < len ? p.ch_sign[(size_t)ch * L + k] : 0;
    if (sign != 0) {
      int a, i, j, kk;
      face_of(p, p.ch_face[(size_t)ch * L + k], a, i, j, kk);
      double m, d;
      sa_face_terms(p, U, a, i, j, kk, m, d);
      const double rho_up = U[cells[k + 1]], rho_c = U[c];
      const double up_m = -(double)sign * m, down_m = (double)sign * m;
      upper = -((up_m > 0.0 ? up_m : 0.0) + d) / rho_up;
      lower_next = -((down_m > 0.0 ? down_m : 0.0) + d) / rho_c;
    }
    const double piv = 1.0 / (dg - lower * cprev);
    cprev = piv * upper;
    F[factor_at(p, ch, k, F3_SA)] = (TF)lower;
    F[factor_at(p, ch, k, F3_SA + 1)] = (TF)piv;
    F[factor_at(p, ch, k, F3_SA + 2)] = (TF)cprev;
    lower = lower_next;
  }
}

// z = M^-1 r on the SA row of chain ch; in the coupled form after the mean flow's apply,
// the right-hand side less the coupling to the neighbours' z (block forward substitution)
template <class TF>
inline __host__ __device__ void chain_apply_sa(const Plan3Dev& p, int ch, const TF* F, const double* r, double* z) {
  const int n = p.NI * p.NJ * p.NK;
  const int* cells = p.ch_cells + (size_t)ch * p.chain_L;
  const int len = chain_length(p, ch);
  TF dprev = 0;
  for (int k = 0; k < len; ++k) {
    const int c = cells[k];
    TF rhs = (TF)r[(size_t)5 * n + c];
    if (p.line_coupled) {
      TF lo = 0, up = 0;
      if (k > 0) {
        lo = F[factor_at(p, ch, k, F3_CPL_LO)] * (TF)z[cells[k - 1]];
        for (int t = 1; t < 5; ++t) lo = lo + F[factor_at(p, ch, k, F3_CPL_LO + t)] * (TF)z[(size_t)t * n + cells[k - 1]];
      }
      if (k + 1 < len) {
        up = F[factor_at(p, ch, k, F3_CPL_UP)] * (TF)z[cells[k + 1]];
        for (int t = 1; t < 5; ++t) up = up + F[factor_at(p, ch, k, F3_CPL_UP + t)] * (TF)z[(size_t)t * n + cells[k + 1]];
      }
      rhs = rhs - (lo + up);
    }
    dprev = F[factor_at(p, ch, k, F3_SA + 1)] * (rhs - F[factor_at(p, ch, k, F3_SA)] * dprev);
    z[(size_t)5 * n + c] = (double)dprev;
  }
  TF nxt = 0;
  for (int k = len - 1; k >= 0; --k) {
    const int c = cells[k];
    nxt = (TF)z[(size_t)5 * n + c] - F[factor_at(p, ch, k, F3_SA + 2)] * nxt;
    z[(size_t)5 * n + c] = (double)nxt;
  }
}

}  // namespace jr

namespace jr {

// The loads on wall face w (src/jaxrans/post/forces.py:48-68): 7 values -- the gauge
// pressure, the area vector into the fluid (3), the laminar viscous force on the body
// (3) -- from the ghost-filled primitive canvas Q.
inline __host__ __device__ void wall_load(const Plan3Dev& p, const double* Q, int w, double out[7]) {
  const int n = p.NI * p.NJ * p.NK;
  const double g = p.P.gamma;
  const int c = p.w_cell[w], a = p.w_family[w], f = p.w_face[w];
  const int fj = p.NJ + (a == 1), fk = p.NK + (a == 2);
  const int i = f / (fj * fk), j = (f / fk) % fj, k = f % fk;
  double s[3];
  face_vector(p, a, i, j, k, s);
  const double into = p.w_into[w];
  out[0] = Q[(size_t)4 * n + c] - 1.0 / g;
  for (int m = 0; m < 3; ++m) out[1 + m] = into * s[m];
  for (int m = 0; m < 3; ++m) out[4 + m] = 0.0;
  if (p.P.mu_inf > 0.0) {
    double grad[3][5];
    face_gradient<double, 4>(p, Q, a, i, j, k, grad);
    int lo[3] = {i, j, k};
    lo[a] -= 1;
    double ql[NV3_MAX], qh[NV3_MAX];
    load_cell(p, Q, cell_index(p, lo[0], lo[1], lo[2]), ql);
    load_cell(p, Q, cell_index(p, i, j, k), qh);
    const double T = 0.5 * (g * ql[4] / ql[0] + g * qh[4] / qh[0]);
    const double mu = viscosity3(p.P, T);
    const double div = grad[0][0] + grad[1][1] + grad[2][2];
    const double ttd = (2.0 / 3.0) * div;
    for (int comp = 0; comp < 3; ++comp) {
      double tau[3];
      for (int d = 0; d < 3; ++d) {
        if (comp == d) {
          tau[d] = mu * (2.0 * grad[comp][comp] - ttd);
        } else {
          const int lo2 = comp < d ? comp : d, hi2 = comp < d ? d : comp;
          tau[d] = mu * (grad[hi2][lo2] + grad[lo2][hi2]);
        }
      }
      out[4 + comp] = into * ((tau[0] * s[0] + tau[1] * s[1]) + tau[2] * s[2]);
    }
  }
}

}  // namespace jr
