// Right-preconditioned restarted GMRES (src/jaxrans/solvers/krylov.py:34-137) and the
// pseudo-transient Newton update (src/jaxrans/solvers/implicit.py:54-168), on the device.
//
// Every cycle runs with a fixed launch sequence (so a Newton step can be captured in
// one CUDA graph): the kernels of a cycle read the case's `active` flag and return at
// once when the restart loop has already stopped.  CGS2 is three passes over the basis:
// the dots; the first update fused with the second dots; the second update fused with
// the norm.  Reductions are per-block partial sums finished by the last block in a fixed
// order, so a rerun gives bitwise the same scalars.  TV is the basis type (double;
// float in the mixed form, with FP64 accumulation).
#include "device.cuh"

namespace jr {

constexpr int RED_THREADS = 256;

__device__ __forceinline__ double warp_sum(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

// NaN-propagating max
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

__device__ __forceinline__ double warp_max(double x) {
  for (int o = 16; o > 0; o >>= 1) x = nmax(x, __shfl_down_sync(0xffffffffu, x, o));
  return x;
}

// Block-sums `vals` into partial[block * W + k]; true in thread 0 of the last block to
// finish, whose `vals` then hold the fixed-order totals over blocks.
template <int W, bool MAX = false>
__device__ bool reduce_last(double (&vals)[W], double* partial, unsigned* ticket) {
  __shared__ double sm[RED_THREADS / 32][W];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    double x = MAX ? warp_max(vals[k]) : warp_sum(vals[k]);
    if (lane == 0) sm[warp][k] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      double t = sm[0][k];
      for (int w = 1; w < nw; ++w) t = MAX ? nmax(t, sm[w][k]) : t + sm[w][k];
      partial[blockIdx.x * W + k] = t;
    }
    __threadfence();
    unsigned prev = atomicAdd(ticket, 1u);
    last = prev == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const volatile double* p = partial;
    double t = p[k];
    for (int b = 1; b < (int)gridDim.x; ++b) t = MAX ? nmax(t, p[b * W + k]) : t + p[b * W + k];
    vals[k] = t;
  }
  *ticket = 0u;
  return true;
}

// The range of elements block b owns
__device__ __forceinline__ void chunk(int n, int& lo, int& hi) {
  int per = (n + gridDim.x - 1) / gridDim.x;
  lo = blockIdx.x * per;
  hi = min(n, lo + per);
}

// ---- GMRES ---------------------------------------------------------------------------

// Start of a Newton step: b = -R, x = action = 0, r = b; |b|; the residual norm of the
// density row from the tile partials; the history entry.
__global__ void k_gmres_init(Scalars* sc, const double* R, double* b, double* x, double* action, double* r, int n,
                             const double* tile_partial, int n_tiles, double volume_sum, double* history,
                             double* partial, unsigned* ticket) {
  int lo, hi;
  chunk(n, lo, hi);
  double acc[1] = {0.0};
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double v = -R[i];
    b[i] = v;
    r[i] = v;
    x[i] = 0.0;
    action[i] = 0.0;
    acc[0] += v * v;
  }
  if (reduce_last<1>(acc, partial, ticket)) {
    double s = 0.0;
    for (int t = 0; t < n_tiles; ++t) s += tile_partial[t];
    double nrm = sqrt(s / volume_sum);
    sc->norm = nrm;
    if (history != nullptr) history[sc->hpos] = nrm;
    sc->hpos += 1;
    sc->bnorm = sqrt(acc[0]);
    sc->rnorm = sc->bnorm;
    sc->cycle = 0;
    sc->active = 1;
    sc->status = 0;
  }
}

// Cycle start: the restart test between cycles, beta = |r|
__global__ void k_cycle_start(Scalars* sc, Config cfg) {
  bool go = sc->active != 0 && sc->cycle < cfg.maxiter && sc->rnorm > cfg.krylov_tol * sc->bnorm;
  sc->active = go ? 1 : 0;
  sc->beta = sc->rnorm;
  sc->inv_nrm = 1.0 / fmax(sc->beta, 2.2250738585072014e-308);
  for (int k = 0; k < (cfg.restart + 1) * cfg.restart; ++k) sc->H[k] = 0.0;
}

// Block partial dots of w with V_0..V_{nk-1}, finished by the last block into hout.
template <class TV>
__device__ void dots_tail(const TV* V, size_t ldv, int nk, const double* w, int lo, int hi, double* partial,
                          unsigned* ticket, double* hout) {
  __shared__ double sm[RED_THREADS / 32][MAX_KRYLOV + 1];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int k = 0; k < nk; ++k) {
    const TV* vk = V + k * ldv;
    double s = 0.0;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) s += double(vk[i]) * w[i];
    s = warp_sum(s);
    if (lane == 0) sm[warp][k] = s;
  }
  __syncthreads();
  if (threadIdx.x < nk) {
    double t = 0.0;
    for (int ww = 0; ww < nw; ++ww) t += sm[ww][threadIdx.x];
    partial[blockIdx.x * (MAX_KRYLOV + 1) + threadIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < nk) {
    const volatile double* p = partial;
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t += p[b * (MAX_KRYLOV + 1) + threadIdx.x];
    hout[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
}

// h1[k] = V_k . w for k <= j
template <class TV>
__global__ void __launch_bounds__(RED_THREADS) k_dots(const Scalars* sc, const TV* V, size_t ldv, int nk,
                                                      const double* w, int n, double* partial, unsigned* ticket,
                                                      double* hout) {
  if (sc->active == 0) return;
  int lo, hi;
  chunk(n, lo, hi);
  dots_tail(V, ldv, nk, w, lo, hi, partial, ticket, hout);
}

// w -= sum_k h1_k V_k; h2 = V^T w  (the first CGS2 update fused with the second dots)
template <class TV>
__global__ void __launch_bounds__(RED_THREADS) k_update_dots(const Scalars* sc, const TV* V, size_t ldv, int nk,
                                                             double* w, int n, const double* hin, double* partial,
                                                             unsigned* ticket, double* hout) {
  if (sc->active == 0) return;
  __shared__ double h[MAX_KRYLOV + 1];
  if (threadIdx.x < nk) h[threadIdx.x] = hin[threadIdx.x];
  __syncthreads();
  int lo, hi;
  chunk(n, lo, hi);
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nk; ++k) s += h[k] * double(V[k * ldv + i]);
    w[i] = w[i] - s;
  }
  dots_tail(V, ldv, nk, w, lo, hi, partial, ticket, hout);
}

// w -= sum_k h2_k V_k; |w|; column j of H; 1/|w| for the next vector
template <class TV>
__global__ void __launch_bounds__(RED_THREADS) k_update_norm(Scalars* sc, const TV* V, size_t ldv, int nk, double* w,
                                                             int n, int j, int m, double* partial, unsigned* ticket) {
  if (sc->active == 0) return;
  __shared__ double h[MAX_KRYLOV + 1];
  if (threadIdx.x < nk) h[threadIdx.x] = sc->h2[threadIdx.x];
  __syncthreads();
  int lo, hi;
  chunk(n, lo, hi);
  double acc[1] = {0.0};
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nk; ++k) s += h[k] * double(V[k * ldv + i]);
    double wi = w[i] - s;
    w[i] = wi;
    acc[0] += wi * wi;
  }
  if (reduce_last<1>(acc, partial, ticket)) {
    double nrm = sqrt(acc[0]);
    for (int k = 0; k < nk; ++k) sc->H[k + (m + 1) * j] = sc->h1[k] + sc->h2[k];
    sc->H[j + 1 + (m + 1) * j] = nrm;
    sc->nrm = nrm;
    sc->inv_nrm = 1.0 / fmax(nrm, 2.2250738585072014e-308);
    if (nrm == 0.0) sc->status |= ST_GMRES_BREAKDOWN;
  }
}

// argmin |beta e1 - H y| by Givens rotations, pivots below rcond * the largest dropped
// (krylov.py:100-137); hy = H y
__global__ void k_lstsq(Scalars* sc, int m) {
  if (sc->active == 0) return;
  const double rcond = 2.220446049250313e-16 * (m + 1);
  double h[MAX_KRYLOV + 1][MAX_KRYLOV];  // local copy (m small)
  double g[MAX_KRYLOV + 1], cs[MAX_KRYLOV], sn[MAX_KRYLOV];
  for (int i = 0; i <= m; ++i)
    for (int j = 0; j < m; ++j) h[i][j] = sc->H[i + (m + 1) * j];
  g[0] = sc->beta;
  for (int i = 1; i <= m; ++i) g[i] = 0.0;
  for (int j = 0; j < m; ++j) {
    for (int i = 0; i < j; ++i) {
      double a = h[i][j], c = h[i + 1][j];
      h[i][j] = cs[i] * a + sn[i] * c;
      h[i + 1][j] = cs[i] * c - sn[i] * a;
    }
    double a = h[j][j], c = h[j + 1][j];
    double r = sqrt(a * a + c * c);
    double safe = r > 0.0 ? r : 1.0;
    cs[j] = r > 0.0 ? a / safe : 1.0;
    sn[j] = r > 0.0 ? c / safe : 0.0;
    h[j][j] = r;
    h[j + 1][j] = 0.0;
    double gj = g[j];
    g[j] = cs[j] * gj;
    g[j + 1] = -sn[j] * gj;
  }
  double largest = fabs(h[0][0]);
  for (int j = 1; j < m; ++j) largest = fmax(largest, fabs(h[j][j]));
  double y[MAX_KRYLOV];
  for (int j = m - 1; j >= 0; --j) {
    double rest = g[j];
    for (int k = j + 1; k < m; ++k) rest = rest - h[j][k] * y[k];
    bool keep = fabs(h[j][j]) > rcond * largest;
    y[j] = keep ? rest / h[j][j] : 0.0;
  }
  for (int j = 0; j < m; ++j) sc->y[j] = y[j];
  for (int i = 0; i <= m; ++i) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += sc->H[i + (m + 1) * j] * y[j];
    sc->hy[i] = s;
  }
}

// tmp = V_{0..m-1} y; action += V_{0..m} (H y), V_m = w / |w|
template <class TV>
__global__ void k_combine(const Scalars* sc, const TV* V, size_t ldv, int m, const double* w, double* tmp,
                          double* action, int n) {
  if (sc->active == 0) return;
  const double inv = sc->inv_nrm;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0, a = 0.0;
    for (int k = 0; k < m; ++k) {
      double v = double(V[k * ldv + i]);
      s += sc->y[k] * v;
      a += sc->hy[k] * v;
    }
    a += sc->hy[m] * double(TV(w[i] * inv));
    tmp[i] = s;
    action[i] += a;
  }
}

// x += z; r = b - action; |r|; the cycle count
__global__ void __launch_bounds__(RED_THREADS) k_cycle_end(Scalars* sc, double* x, const double* z, const double* b,
                                                           const double* action, double* r, int n, double* partial,
                                                           unsigned* ticket) {
  if (sc->active == 0) return;
  int lo, hi;
  chunk(n, lo, hi);
  double acc[1] = {0.0};
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    x[i] += z[i];
    double ri = b[i] - action[i];
    r[i] = ri;
    acc[0] += ri * ri;
  }
  if (reduce_last<1>(acc, partial, ticket)) {
    sc->rnorm = sqrt(acc[0]);
    sc->cycle += 1;
  }
}

// ---- the Newton update -------------------------------------------------------------

// omega = min(1, fraction / max relative change of rho, p, nu_hat)  (implicit.py:54-81)
__global__ void __launch_bounds__(RED_THREADS) k_relax(Scalars* sc, Canvas c, Physics P, Config cfg, const double* U,
                                                       const double* dU, double* partial, unsigned* ticket) {
  const int N = c.ncanvas(), nv = c.nvar;
  const double g = P.gamma;
  double worst[1] = {0.0};
  if (cfg.max_relative_update > 0.0) {
    int lo, hi;
    chunk(N, lo, hi);
    for (int idx = lo + threadIdx.x; idx < hi; idx += blockDim.x) {
      double rho = U[idx], u = U[N + idx] / rho, v = U[2 * N + idx] / rho;
      double p = (g - 1.0) * (U[3 * N + idx] - 0.5 * rho * (u * u + v * v));
      double de = dU[3 * N + idx] - u * dU[N + idx] - v * dU[2 * N + idx];
      double dp = (g - 1.0) * (de + 0.5 * (u * u + v * v) * dU[idx]);
      double w = nmax(fabs(dU[idx]) / rho, fabs(dp) / p);
      if (nv > 4) {
        double nh = U[4 * N + idx] / rho;
        double dnh = (dU[4 * N + idx] - nh * dU[idx]) / rho;
        w = nmax(w, fabs(dnh) / fmax(fabs(nh), 1.0));
      }
      worst[0] = nmax(worst[0], w);
    }
  }
  if (reduce_last<1, true>(worst, partial, ticket)) {
    sc->worst = worst[0];
    if (cfg.max_relative_update > 0.0) {
      double q = cfg.max_relative_update / (worst[0] != worst[0] ? NAN : fmax(worst[0], 1e-300));
      sc->omega = q != q ? NAN : fmin(1.0, q);
    } else {
      sc->omega = 1.0;
    }
  }
}

// the linear reduction, physicality of the candidate, accept, the SER CFL ramp
__global__ void __launch_bounds__(RED_THREADS) k_accept(Scalars* sc, Canvas c, Physics P, Config cfg, const double* U,
                                                        const double* dU, const double* action, const double* R,
                                                        double* partial, unsigned* ticket) {
  const int N = c.ncanvas(), nv = c.nvar, n = nv * N;
  const double g = P.gamma, om = sc->omega;
  int lo, hi;
  chunk(n, lo, hi);
  double acc[3] = {0.0, 0.0, 0.0};  // |omega action + R|^2, |R|^2, bad cells
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double t = om * action[i] + R[i];
    acc[0] += t * t;
    acc[1] += R[i] * R[i];
    if (!isfinite(om * dU[i])) acc[2] += 1.0;
    if (i < N) {
      double rho = U[i] + om * dU[i];
      double mx = U[N + i] + om * dU[N + i], my = U[2 * N + i] + om * dU[2 * N + i];
      double E = U[3 * N + i] + om * dU[3 * N + i];
      double u = mx / rho, v = my / rho;
      double p = (g - 1.0) * (E - 0.5 * rho * (u * u + v * v));
      bool ok = rho > 1e-10 && p > 1e-10 && isfinite(rho) && isfinite(p);
      if (!ok) acc[2] += 1.0;
    }
  }
  if (reduce_last<3>(acc, partial, ticket)) {
    double lin = sqrt(acc[0]) / fmax(sqrt(acc[1]), 1e-300);
    bool physical = acc[2] == 0.0;
    bool accept = physical && lin < 1.0;
    double reduction = sc->res_prev / fmax(sc->norm, 1e-300);
    double cfl = sc->cfl, next;
    if (accept && lin < cfg.krylov_success && om >= 1.0)
      next = cfl * fmin(fmax(reduction, 1.0), cfg.cfl_growth);
    else if (accept)
      next = cfl;
    else
      next = cfl / cfg.cfl_cutback;
    sc->lin_red = lin;
    sc->accept = accept ? 1 : 0;
    sc->cfl = fmin(fmax(next, cfg.cfl_min), cfg.cfl_max);
    if (accept) sc->res_prev = sc->norm;
    sc->steps += 1;
    if (!accept) {
      sc->rejected += 1;
      sc->status |= ST_REJECTED;
    }
    if (!physical) sc->status |= ST_NONFINITE;
  }
}

__global__ void k_update(const Scalars* sc, double* U, const double* dU, int n) {
  if (sc->accept == 0) return;
  const double om = sc->omega;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) U[i] = U[i] + om * dU[i];
}

// ---- launch wrappers ------------------------------------------------------------------

int reduce_blocks(int n) { return max(1, min(2 * 148, (n + 1023) / 1024)); }

void launch_gmres_init(Scalars* sc, const double* R, double* b, double* x, double* action, double* r, int n,
                       const double* tile_partial, int n_tiles, double volume_sum, double* history, Reduce red,
                       cudaStream_t st) {
  k_gmres_init<<<reduce_blocks(n), RED_THREADS, 0, st>>>(sc, R, b, x, action, r, n, tile_partial, n_tiles,
                                                         volume_sum, history, red.partial, red.ticket);
}

void launch_cycle_start(Scalars* sc, Config cfg, cudaStream_t st) { k_cycle_start<<<1, 1, 0, st>>>(sc, cfg); }

template <class TV>
static void arnoldi_t(Scalars* sc, const TV* V, size_t ldv, int j, int m, double* w, int n, Reduce red,
                      cudaStream_t st) {
  int blocks = reduce_blocks(n);
  k_dots<TV><<<blocks, RED_THREADS, 0, st>>>(sc, V, ldv, j + 1, w, n, red.partial, red.ticket, sc->h1);
  k_update_dots<TV><<<blocks, RED_THREADS, 0, st>>>(sc, V, ldv, j + 1, w, n, sc->h1, red.partial, red.ticket,
                                                    sc->h2);
  k_update_norm<TV><<<blocks, RED_THREADS, 0, st>>>(sc, V, ldv, j + 1, w, n, j, m, red.partial, red.ticket);
}

void launch_arnoldi_orth(Scalars* sc, const void* V, bool fp32, size_t ldv, int j, int m, double* w, int n,
                         Reduce red, cudaStream_t st) {
  if (fp32) arnoldi_t<float>(sc, (const float*)V, ldv, j, m, w, n, red, st);
  else arnoldi_t<double>(sc, (const double*)V, ldv, j, m, w, n, red, st);
}

void launch_lstsq(Scalars* sc, int m, cudaStream_t st) { k_lstsq<<<1, 1, 0, st>>>(sc, m); }

void launch_combine(const Scalars* sc, const void* V, bool fp32, size_t ldv, int m, const double* w, double* tmp,
                    double* action, int n, cudaStream_t st) {
  int blocks = min((n + 255) / 256, 148 * 4);
  if (fp32) k_combine<float><<<blocks, 256, 0, st>>>(sc, (const float*)V, ldv, m, w, tmp, action, n);
  else k_combine<double><<<blocks, 256, 0, st>>>(sc, (const double*)V, ldv, m, w, tmp, action, n);
}

void launch_cycle_end(Scalars* sc, double* x, const double* z, const double* b, const double* action, double* r,
                      int n, Reduce red, cudaStream_t st) {
  k_cycle_end<<<reduce_blocks(n), RED_THREADS, 0, st>>>(sc, x, z, b, action, r, n, red.partial, red.ticket);
}

void launch_newton_update(Scalars* sc, const Canvas& c, const Physics& P, Config cfg, double* U, const double* dU,
                          const double* action, const double* R, Reduce red, cudaStream_t st) {
  int N = c.NI * c.NJ, n = c.nvar * N;
  k_relax<<<reduce_blocks(N), RED_THREADS, 0, st>>>(sc, c, P, cfg, U, dU, red.partial, red.ticket);
  k_accept<<<reduce_blocks(n), RED_THREADS, 0, st>>>(sc, c, P, cfg, U, dU, action, R, red.partial, red.ticket);
  k_update<<<min((n + 255) / 256, 148 * 4), 256, 0, st>>>(sc, U, dU, n);
}

}  // namespace jr
