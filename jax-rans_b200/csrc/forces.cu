// Wall loads and force coefficients in FP64 (src/jaxrans/post/forces.py:48-161): gauge
// pressure from the cell on each wall face, the laminar viscous shear of the same
// diamond-gradient viscous flux the residual uses, lift normal and drag along the
// freestream, the pressure moment about the moment centre.  One CTA reduces all wall
// faces in a fixed order.
#include "device.cuh"

namespace jr {

__device__ __forceinline__ double q_at(const Canvas& c, const Physics& P, const double* U, const double* qg, int idx,
                                       int v) {
  const int N = c.ncanvas();
  if (c.interior[idx]) {
    double u[5], q[5];
    for (int k = 0; k < 4; ++k) u[k] = U[k * N + idx];
    to_prim(u, q, 4, P.gamma);
    return q[v];
  }
  return qg[v * N + idx];
}

// laminar F_v . S at the wall face (family a) below canvas cell (i, j) or above it
__device__ void wall_viscous(const Canvas& c, const Physics& P, const double* U, const double* qg, int family, int face,
                             double sx, double sy, double& fx, double& fy) {
  const int NJ = c.NJ;
  int ai, aj, bi, bj;
  if (family == 0) {
    int i = face / NJ, j = face % NJ;
    ai = i - 1; aj = j; bi = i; bj = j;
  } else {
    int i = face / (NJ + 1), j = face % (NJ + 1);
    ai = i; aj = j - 1; bi = i; bj = j;
  }
  const double g = P.gamma;
  auto phi = [&](int i, int j, int k) {
    int idx = i * NJ + j;
    if (k < 2) return q_at(c, P, U, qg, idx, 1 + k);
    return g * q_at(c, P, U, qg, idx, 3) / q_at(c, P, U, qg, idx, 0);
  };
  const int CJ = NJ + 2, CN = (c.NI + 2) * CJ;
  auto cx = [&](int i, int j) { return c.centres[(i + 1) * CJ + j + 1]; };
  auto cy = [&](int i, int j) { return c.centres[CN + (i + 1) * CJ + j + 1]; };
  int n0[4][2], n1[4][2];
  if (family == 0) {
    int n0_[4][2] = {{ai, aj - 1}, {ai + 1, aj - 1}, {ai, aj}, {ai + 1, aj}};
    int n1_[4][2] = {{ai, aj}, {ai + 1, aj}, {ai, aj + 1}, {ai + 1, aj + 1}};
    for (int k = 0; k < 4; ++k) for (int t = 0; t < 2; ++t) { n0[k][t] = n0_[k][t]; n1[k][t] = n1_[k][t]; }
  } else {
    int n0_[4][2] = {{ai - 1, aj}, {ai, aj}, {ai - 1, aj + 1}, {ai, aj + 1}};
    int n1_[4][2] = {{ai, aj}, {ai + 1, aj}, {ai, aj + 1}, {ai + 1, aj + 1}};
    for (int k = 0; k < 4; ++k) for (int t = 0; t < 2; ++t) { n0[k][t] = n0_[k][t]; n1[k][t] = n1_[k][t]; }
  }
  auto corner = [&](int (*n)[2], auto f) { return 0.25 * (((f(n[0][0], n[0][1]) + f(n[1][0], n[1][1])) + f(n[2][0], n[2][1])) + f(n[3][0], n[3][1])); };
  double d1x = cx(bi, bj) - cx(ai, aj), d1y = cy(bi, bj) - cy(ai, aj);
  double d2x = corner(n1, cx) - corner(n0, cx), d2y = corner(n1, cy) - corner(n0, cy);
  double det = d1x * d2y - d2x * d1y;
  double gx[3], gy[3];
  for (int k = 0; k < 3; ++k) {
    auto pk = [&](int i, int j) { return phi(i, j, k); };
    double dpc = phi(bi, bj, k) - phi(ai, aj, k);
    double dpn = corner(n1, pk) - corner(n0, pk);
    gx[k] = (dpc * d2y - dpn * d1y) / det;
    gy[k] = (d1x * dpn - d2x * dpc) / det;
  }
  double Tf = 0.5 * (phi(ai, aj, 2) + phi(bi, bj, 2));
  double mu = viscosity(P, Tf);
  double g00 = gx[0], g01 = gy[0], g10 = gx[1], g11 = gy[1];
  double div = g00 + g11, ttd = (2.0 / 3.0) * div;
  double t00 = mu * (2.0 * g00 - ttd), t11 = mu * (2.0 * g11 - ttd), t01 = mu * (g01 + g10);
  fx = t00 * sx + t01 * sy;
  fy = t01 * sx + t11 * sy;
}

// force_out of each case: cl, cd, cm, cd_friction, fx, fy.  One CTA per case.
__global__ void __launch_bounds__(256) k_forces(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* U = cd.U;
  const double* qg = cd.qg;
  const double length = cd.force_length, cx0 = cd.moment_centre[0], cy0 = cd.moment_centre[1];
  double* out = cd.force_out;
  __shared__ double red[6][32];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const double rho = P.q_inf[0], u = P.q_inf[1], v = P.q_inf[2];
  const double speed = hypot(u, v);
  const double dx = u / speed, dy = v / speed;   // drag direction
  const double lx = -dy, ly = dx;                  // lift direction
  const double q_area = 0.5 * rho * speed * speed * length;
  for (int w = threadIdx.x; w < c.n_walls; w += blockDim.x) {
    int cell = c.w_cell[w], fam = c.w_family[w], f = c.w_face[w];
    double into = c.w_into[w];
    double sx, sy;
    if (fam == 0) {
      sx = c.fi[f];
      sy = c.fi[c.nfi() + f];
    } else {
      sx = c.fj[f];
      sy = c.fj[c.nfj() + f];
    }
    double Sx = into * sx, Sy = into * sy;
    double p = q_at(c, P, U, qg, cell, 3) - 1.0 / P.gamma;
    double px = -p * Sx, py = -p * Sy;
    double shx = 0.0, shy = 0.0;
    if (P.mu_inf > 0.0) {
      double fx, fy;
      wall_viscous(c, P, U, qg, fam, f, sx, sy, fx, fy);
      shx = into * fx;
      shy = into * fy;
    }
    if (cd.wall_out != nullptr) {
      double* o = cd.wall_out + 5 * w;
      o[0] = p;
      o[1] = Sx;
      o[2] = Sy;
      o[3] = shx;
      o[4] = shy;
    }
    double Lx = px + shx, Ly = py + shy;
    double rx = c.w_mid[2 * w] - cx0, ry = c.w_mid[2 * w + 1] - cy0;
    double moment = ry * px - rx * py;
    acc[0] += (lx * Lx + ly * Ly) / q_area;
    acc[1] += (dx * Lx + dy * Ly) / q_area;
    acc[2] += (moment / length) / q_area;
    acc[3] += dx * shx + dy * shy;
    acc[4] += Lx;
    acc[5] += Ly;
  }
  for (int k = 0; k < 6; ++k) {
    double x = acc[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[6];
    for (int k = 0; k < 6; ++k) {
      t[k] = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t[k] += red[k][w];
    }
    out[0] = t[0];
    out[1] = t[1];
    out[2] = t[2];
    out[3] = t[3] / q_area;
    out[4] = t[4];
    out[5] = t[5];
  }
}

void launch_forces(const CaseDev* cases, const BatchDims& d, cudaStream_t st) {
  k_forces<<<dim3(1, d.n_cases), 256, 0, st>>>(cases);
}

// The exit test of every monitored case after a block of block_iters Newton steps whose
// norms sit in rows step0.. of the history, and whose forces k_forces has just written
// (one warp per case).  The decisions are the host driver's, in the same order and with
// the same arithmetic: non-finite (a NaN or Inf norm or force), converged (last <= tol x
// running peak), stalled (every norm of the block equal to the first), settled (CL, CD
// and CM each with a range below forces_tol over the last quarter of the samples, at
// least four there), and max_iters once max_blocks blocks have run.  A case that stops
// with `release` set is disabled in `cases` itself, so the launches already queued skip
// it.
__global__ void __launch_bounds__(32) k_monitor(CaseDev* __restrict__ cases, int n_slots, int step0,
                                                int block_iters) {
  CaseDev& cd = cases[blockIdx.x];
  if (!cd.enabled || cd.mon == nullptr) return;
  Monitor& m = *cd.mon;
  if (m.max_blocks == 0 || m.reason != MON_RUNNING) return;
  const int lane = threadIdx.x;
  const double* hist = cd.history + (size_t)step0 * n_slots + cd.slot;
  const double first = hist[0], last = hist[(size_t)(block_iters - 1) * n_slots];
  bool finite = true, equal = true;
  double top = -INFINITY;
  bool any = false;
  for (int s = lane; s < block_iters; s += 32) {
    const double h = hist[(size_t)s * n_slots];
    const bool ok = isfinite(h);
    finite = finite && ok;
    equal = equal && h == first;
    if (ok) {
      top = fmax(top, h);
      any = true;
    }
  }
  finite = __all_sync(0xffffffffu, finite);
  equal = __all_sync(0xffffffffu, equal);
  any = __any_sync(0xffffffffu, any);
  for (int o = 16; o > 0; o >>= 1) top = fmax(top, __shfl_xor_sync(0xffffffffu, top, o));
  const double cl = cd.force_out[0], cdr = cd.force_out[1], cm = cd.force_out[2];
  const int n = m.blocks + 1;
  if (lane == 0 && m.blocks < MONITOR_BLOCKS) {
    m.coef[m.blocks][0] = cl;
    m.coef[m.blocks][1] = cdr;
    m.coef[m.blocks][2] = cm;
  }
  __syncwarp();
  const double peak = any ? fmax(m.peak, top) : m.peak;
  // the spread of each coefficient over the last quarter of the n samples
  const int start = 3 * n / 4, tail = n - start;
  bool settled = false;
  if (m.forces_tol >= 0.0 && tail >= 4 && n <= MONITOR_BLOCKS) {
    settled = true;
    for (int k = 0; k < 3; ++k) {
      double lo = INFINITY, hi = -INFINITY;
      for (int b = start + lane; b < n; b += 32) {
        lo = fmin(lo, m.coef[b][k]);
        hi = fmax(hi, m.coef[b][k]);
      }
      for (int o = 16; o > 0; o >>= 1) {
        lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      }
      settled = settled && (hi - lo < m.forces_tol);
    }
  }
  if (lane != 0) return;
  m.peak = peak;
  m.blocks = n;
  int reason = MON_RUNNING;
  if (!finite || !isfinite(cl) || !isfinite(cdr) || !isfinite(cm)) reason = MON_NON_FINITE;
  else if (peak > 0.0 && last <= m.tol * peak) reason = MON_CONVERGED;
  else if (block_iters > 1 && equal) reason = MON_STALLED;
  else if (settled) reason = MON_SETTLED;
  else if (n >= m.max_blocks) reason = MON_MAX_ITERS;
  m.reason = reason;
  if (reason != MON_RUNNING && m.release) cd.enabled = 0;
}

// The volume-weighted L2 norm of row `variable` of each case's field R over its block
// cells (src/jaxrans/numerics/residual.py:237-240): sqrt(sum V R^2 / sum V), one CTA per
// case, its threads' partial sums added in a fixed order.
__global__ void __launch_bounds__(256) k_norm(const CaseDev* __restrict__ cases, int variable,
                                              double* __restrict__ out) {
  const CaseDev& cd = cases[blockIdx.x];
  const Canvas& c = cd.c;
  const int N = c.ncanvas();
  const double* __restrict__ R = cd.R + (size_t)variable * N;
  __shared__ double red[8];
  double acc = 0.0;
  for (int k = threadIdx.x; k < N; k += blockDim.x)
    if (c.interior[k]) acc += c.volume[k] * (R[k] * R[k]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    out[blockIdx.x] = sqrt(t / c.volume_sum);
  }
}

void launch_norm(const CaseDev* cases, int n_cases, int variable, double* out, cudaStream_t st) {
  k_norm<<<n_cases, 256, 0, st>>>(cases, variable, out);
}

void launch_monitor(CaseDev* cases, int n_live, int n_slots, int step0, int block_iters, cudaStream_t st) {
  if (n_live > 0) k_monitor<<<n_live, 32, 0, st>>>(cases, n_slots, step0, block_iters);
}

}  // namespace jr
