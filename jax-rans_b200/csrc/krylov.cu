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

// In the last block of a reduction: out[k] = the sum (or NaN-propagating max) over the
// nb rows of partial[b * stride + k], k < W, by all the block's threads in a fixed order
// -- thread (k, r) takes the rows b = r, r + R, ... (R = blockDim.x / W groups), with its
// loads issued eight at a time, then thread k adds the R group totals in order.  Loads go
// to L2 (ld.global.cg), where the other blocks' partials are.
template <bool MAX>
__device__ void reduce_rows(const double* partial, int stride, int W, int nb, double* out) {
  __shared__ double group[RED_THREADS];
  const int R = max(1, (int)blockDim.x / W);
  const int t = threadIdx.x, k = t % W, r = t / W;
  if (r < R) {
    double acc = MAX ? -INFINITY : 0.0;
    // rows r, r + R, ... in order, eight loads in flight at a time (the last eight
    // predicated, so the tail costs one round trip, not one per row)
    for (int b = r; b < nb; b += 8 * R) {
      double x[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) x[u] = b + u * R < nb ? __ldcg(partial + (size_t)(b + u * R) * stride + k) : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (b + u * R < nb) acc = MAX ? nmax(acc, x[u]) : acc + x[u];
    }
    group[t] = acc;
  }
  __syncthreads();
  if (t < W) {
    double v = group[t];
    for (int g = 1; g < R; ++g) v = MAX ? nmax(v, group[g * W + t]) : v + group[g * W + t];
    out[t] = v;
  }
  __syncthreads();
}

// Block-sums `vals` into partial[block * W + k]; true in thread 0 of the last block to
// finish, whose `vals` then hold the fixed-order totals over blocks.
template <int W, bool MAX = false>
__device__ bool reduce_last(double (&vals)[W], double* partial, unsigned* ticket, int nb) {
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
    last = prev == (unsigned)nb - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  __shared__ double total[W];
  reduce_rows<MAX>(partial, W, W, nb, total);
  if (threadIdx.x != 0) return false;
#pragma unroll
  for (int k = 0; k < W; ++k) vals[k] = total[k];
  *ticket = 0u;
  return true;
}

// The NK accumulators of every lane summed over the warp by a butterfly that halves the
// values a lane holds at each of the five exchanges: at the end lane l holds the sums of
// accumulators l*(NK/32) .. l*(NK/32) + NK/32 - 1 (NK >= 32), or of l / (32/NK) in
// acc[0] (NK < 32).  The additions follow a fixed tree, so a rerun is bitwise the same.
template <int NK>
__device__ __forceinline__ void warp_transpose_sum(double (&acc)[NK], int lane) {
  int held = NK;
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    if (held >= 2) {
      const int half = held / 2;
      const bool upper = (lane & o) != 0;
#pragma unroll
      for (int k = 0; k < NK / 2; ++k) {
        if (k < half) {
          const double send = upper ? acc[k] : acc[k + half];
          const double keep = upper ? acc[k + half] : acc[k];
          acc[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
      held = half;
    } else {
      acc[0] += __shfl_xor_sync(0xffffffffu, acc[0], o);
    }
  }
}

// The range of elements block b of nb owns
__device__ __forceinline__ void chunk(int n, int nb, int& lo, int& hi) {
  int per = (n + nb - 1) / nb;
  lo = blockIdx.x * per;
  hi = min(n, lo + per);
}

// ---- GMRES ---------------------------------------------------------------------------
// Every kernel takes the batch's case table and reads its case from blockIdx.y.  The
// per-case block count of a reduction depends on that case's size alone, so a case's
// scalars are bitwise the same alone and in a batch; the blocks past it return at once.

// blocks of a chunked per-case reduction over n elements (<= the grid's x)
__device__ __forceinline__ bool chunk_owner(int n, int& nb, int& lo, int& hi) {
  nb = chunk_blocks(n);
  if ((int)blockIdx.x >= nb) return false;
  chunk(n, nb, lo, hi);
  return true;
}

// Start of a Newton step: b = -R, x = action = 0, r = b; |b|; the residual norm of the
// density row from the tile partials; the history entry.
__global__ void __launch_bounds__(RED_THREADS) k_gmres_init(const CaseDev* __restrict__ cases, int n_cases_hist) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  const int n = cd.n_vec;
  int nb, lo, hi;
  if (!chunk_owner(n, nb, lo, hi)) return;
  const double* __restrict__ R = cd.R;
  double *b = cd.b, *r = cd.r, *x = cd.x, *action = cd.action;
  double acc[1] = {0.0};
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double v = -R[i];
    b[i] = v;
    r[i] = v;
    x[i] = 0.0;
    action[i] = 0.0;
    acc[0] += v * v;
  }
  if (reduce_last<1>(acc, cd.partial, cd.ticket, nb)) {
    Scalars* sc = cd.sc;
    double s = 0.0;
    for (int t = 0; t < cd.n_tiles; ++t) s += cd.tile_partial[t];
    double nrm = sqrt(s / cd.c.volume_sum);
    sc->norm = nrm;
    // history: [step][case] over the cases of the batch
    if (cd.history != nullptr) cd.history[(size_t)sc->hpos * n_cases_hist + cd.slot] = nrm;
    sc->hpos += 1;
    sc->bnorm = sqrt(acc[0]);
    sc->rnorm = sc->bnorm;
    sc->cycle = 0;
    sc->active = 1;
    sc->status &= ST_STAGE_FAILED;
  }
}

// Cycle start: the restart test between cycles, beta = |r|; H = 0
__global__ void k_cycle_start(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  Scalars* sc = cd.sc;
  const Config& cfg = cd.cfg;
  for (int k = threadIdx.x; k < (cfg.restart + 1) * cfg.restart; k += blockDim.x) sc->H[k] = 0.0;
  if (threadIdx.x != 0) return;
  bool go = sc->active != 0 && sc->cycle < cfg.maxiter && sc->rnorm > cfg.krylov_tol * sc->bnorm;
  sc->active = go ? 1 : 0;
  sc->beta = sc->rnorm;
  sc->inv_nrm = 1.0 / fmax(sc->beta, 2.2250738585072014e-308);
}

// The gate of a Krylov cycle in the step graph: the cycle's body (an IF node) runs only
// when some case of the launch is still active; `cycles` counts the bodies run.
__global__ void k_cycle_gate(const CaseDev* __restrict__ cases, int n_cases, cudaGraphConditionalHandle gate,
                             unsigned long long* cycles) {
  int any = 0;
  for (int k = threadIdx.x; k < n_cases; k += blockDim.x) any |= cases[k].enabled && cases[k].sc->active != 0;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    cudaGraphSetConditional(gate, any ? 1u : 0u);
    if (any) *cycles += 1ull;
  }
}

// The three passes of CGS2 over the basis, one kernel: MODE 0 h = V^T w; MODE 1
// w -= V hin, then h = V^T w; MODE 2 w -= V hin, then |w| and column j of H.  A block
// owns a chunk of cgs_chunk(n) elements.  The update runs thread per element (for an FP64
// basis the nk loads of an element issued together, up to 32 in flight, before they are
// added in order); the dot products run warp per basis vector against the block's w held
// in shared memory, each lane with 32 loads in flight (16 for an FP32 basis).  With one
// or two blocks per SM the passes are bound by the bytes in flight, hence the batches;
// the order of every sum is that of one load at a time.  In MODE 1 the second read of
// the chunk's basis rows is served by L2.
template <class TV, int NK, int MODE>
__global__ void __launch_bounds__(RED_THREADS) k_mdot(const CaseDev* __restrict__ cases, int nk, int j) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  Scalars* sc = cd.sc;
  if (sc->active == 0) return;
  const int n = cd.n_vec, m = cd.m;
  const int nb = cgs_blocks(n), C = cgs_chunk(n);
  if ((int)blockIdx.x >= nb) return;
  const TV* __restrict__ V = (const TV*)cd.V;
  const size_t ldv = (size_t)n;
  double* __restrict__ w = cd.w;
  double* __restrict__ partial = cd.partial;
  unsigned* ticket = cd.ticket;
  const double* hin = MODE == 1 ? sc->h1 : sc->h2;
  double* hout = MODE == 0 ? sc->h1 : sc->h2;
  __shared__ double ws[MODE == 2 ? 1 : CGS_MAX_CHUNK];
  __shared__ double h[MODE == 0 ? 1 : NK];
  __shared__ double sm[RED_THREADS / 32];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  if constexpr (MODE != 0) {
    if ((int)threadIdx.x < NK) h[threadIdx.x] = (int)threadIdx.x < nk ? hin[threadIdx.x] : 0.0;
    __syncthreads();
  }
  const int i0 = blockIdx.x * C;
  const int cn = min(C, n - i0);
  // 1. the update (MODE 1, 2), or the copy of w (MODE 0), element by element
  double acc = 0.0;
  for (int e = threadIdx.x; e < cn; e += blockDim.x) {
    const int i = i0 + e;
    double wi = w[i];
    if constexpr (MODE != 0) {
      // an FP64 basis: the element's nk entries loaded together, then added in order (an
      // FP32 basis keeps one load per entry: measured faster there)
      constexpr int KB = sizeof(TV) == 4 ? 1 : (NK < 32 ? NK : 32);
      double s = 0.0;
#pragma unroll
      for (int k0 = 0; k0 < NK; k0 += KB) {
        double vk[KB];
#pragma unroll
        for (int u = 0; u < KB; ++u) vk[u] = k0 + u < nk ? double(V[(size_t)(k0 + u) * ldv + i]) : 0.0;
#pragma unroll
        for (int u = 0; u < KB; ++u)
          if (k0 + u < nk) s += h[k0 + u] * vk[u];
      }
      wi = wi - s;
      w[i] = wi;
    }
    if constexpr (MODE == 2) acc += wi * wi;
    else ws[e] = wi;
  }
  const int width = MODE == 2 ? 1 : nk;
  if constexpr (MODE == 2) {
    double x = warp_sum(acc);
    if (lane == 0) sm[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = sm[0];
      for (int ww = 1; ww < nw; ++ww) t += sm[ww];
      partial[blockIdx.x * (MAX_KRYLOV + 1)] = t;
    }
  } else {
    __syncthreads();
    // 2. the dot products, warp per basis vector
    for (int k = warp; k < nk; k += nw) {
      const TV* __restrict__ vk = V + k * ldv + i0;
      double a = 0.0;
      int e = lane;
      if constexpr (sizeof(TV) == 8) {   // an FP64 basis: 32 loads in flight per lane
        for (; e + 32 * 31 < cn; e += 32 * 32) {
          double x[32];
#pragma unroll
          for (int u = 0; u < 32; ++u) x[u] = double(vk[e + 32 * u]);
#pragma unroll
          for (int u = 0; u < 32; ++u) a += x[u] * ws[e + 32 * u];
        }
      }
      for (; e + 32 * 15 < cn; e += 32 * 16) {
        double x[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) x[u] = double(vk[e + 32 * u]);
#pragma unroll
        for (int u = 0; u < 16; ++u) a += x[u] * ws[e + 32 * u];
      }
      for (; e < cn; e += 32) a += double(vk[e]) * ws[e];
      a = warp_sum(a);
      if (lane == 0) partial[blockIdx.x * (MAX_KRYLOV + 1) + k] = a;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == (unsigned)nb - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double total[MAX_KRYLOV + 1];
  reduce_rows<false>(partial, MAX_KRYLOV + 1, width, nb, total);
  if ((int)threadIdx.x < width) {
    const double t = total[threadIdx.x];
    if constexpr (MODE == 2) {
      double nrm = sqrt(t);
      for (int k = 0; k < nk; ++k) sc->H[k + (m + 1) * j] = sc->h1[k] + sc->h2[k];
      sc->H[j + 1 + (m + 1) * j] = nrm;
      sc->nrm = nrm;
      sc->inv_nrm = 1.0 / fmax(nrm, 2.2250738585072014e-308);
      if (nrm == 0.0) sc->status |= ST_GMRES_BREAKDOWN;
    } else {
      hout[threadIdx.x] = t;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
}

// argmin |beta e1 - H y| by Givens rotations, pivots below rcond * the largest dropped
// (krylov.py:100-137); hy = H y.  One CTA per case: rotation j, once formed, is applied
// to rows j, j+1 of every later column at once -- each entry sees the same rotations in
// the same order as column-by-column elimination.
__global__ void __launch_bounds__(64) k_lstsq(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  Scalars* sc = cd.sc;
  if (sc->active == 0) return;
  const int m = cd.m;
  __shared__ double h[MAX_KRYLOV + 1][MAX_KRYLOV + 1];
  __shared__ double g[MAX_KRYLOV + 1], cs[MAX_KRYLOV], sn[MAX_KRYLOV], y[MAX_KRYLOV];
  __shared__ double largest;
  const int t = threadIdx.x;
  for (int e = t; e < (m + 1) * m; e += blockDim.x) {
    int i = e % (m + 1), jj = e / (m + 1);
    h[i][jj] = sc->H[e];
  }
  if (t <= m) g[t] = t == 0 ? sc->beta : 0.0;
  __syncthreads();
  for (int j = 0; j < m; ++j) {
    if (t == 0) {
      double a = h[j][j], c = h[j + 1][j];
      double r = sqrt(a * a + c * c);
      double safe = r > 0.0 ? r : 1.0;
      double cj = r > 0.0 ? a / safe : 1.0, sj = r > 0.0 ? c / safe : 0.0;
      cs[j] = cj;
      sn[j] = sj;
      h[j][j] = r;
      h[j + 1][j] = 0.0;
      double gj = g[j];
      g[j] = cj * gj;
      g[j + 1] = -sj * gj;
    }
    __syncthreads();
    for (int col = j + 1 + t; col < m; col += blockDim.x) {
      double a = h[j][col], c = h[j + 1][col];
      h[j][col] = cs[j] * a + sn[j] * c;
      h[j + 1][col] = cs[j] * c - sn[j] * a;
    }
    __syncthreads();
  }
  if (t == 0) {
    double l = fabs(h[0][0]);
    for (int jj = 1; jj < m; ++jj) l = fmax(l, fabs(h[jj][jj]));
    largest = l;
  }
  __syncthreads();
  const double rcond = 2.220446049250313e-16 * (m + 1);
  for (int j = m - 1; j >= 0; --j) {
    if (t < 32) {
      double s = 0.0;
      for (int k = j + 1 + t; k < m; k += 32) s += h[j][k] * y[k];
      s = warp_sum(s);
      if (t == 0) {
        double rest = g[j] - s;
        bool keep = fabs(h[j][j]) > rcond * largest;
        y[j] = keep ? rest / h[j][j] : 0.0;
      }
    }
    __syncthreads();
  }
  if (t < m) sc->y[t] = y[t];
  if (t <= m) {
    double s = 0.0;
    for (int jj = 0; jj < m; ++jj) s += sc->H[t + (m + 1) * jj] * y[jj];
    sc->hy[t] = s;
  }
}

// tmp = V_{0..m-1} y; action += V_{0..m} (H y), V_m = w / |w|
template <class TV>
__global__ void k_combine(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  const Scalars* sc = cd.sc;
  if (sc->active == 0) return;
  const int m = cd.m, n = cd.n_vec;
  const TV* __restrict__ V = (const TV*)cd.V;
  const size_t ldv = (size_t)n;
  const double* __restrict__ w = cd.w;
  double* __restrict__ tmp = cd.tmp;
  double* __restrict__ action = cd.action;
  __shared__ double y[MAX_KRYLOV], hy[MAX_KRYLOV + 1];
  if ((int)threadIdx.x < m) y[threadIdx.x] = sc->y[threadIdx.x];
  if ((int)threadIdx.x <= m) hy[threadIdx.x] = sc->hy[threadIdx.x];
  __syncthreads();
  const double inv = sc->inv_nrm;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0.0, a = 0.0;
    for (int k = 0; k < m; ++k) {
      double v = double(V[k * ldv + i]);
      s += y[k] * v;
      a += hy[k] * v;
    }
    a += hy[m] * double(TV(w[i] * inv));
    tmp[i] = s;
    action[i] += a;
  }
}

// x += z; r = b - action; |r|; the cycle count
__global__ void __launch_bounds__(RED_THREADS) k_cycle_end(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  Scalars* sc = cd.sc;
  if (sc->active == 0) return;
  int nb, lo, hi;
  if (!chunk_owner(cd.n_vec, nb, lo, hi)) return;
  double *x = cd.x, *r = cd.r;
  const double *z = cd.z, *b = cd.b, *action = cd.action;
  double acc[1] = {0.0};
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    x[i] += z[i];
    double ri = b[i] - action[i];
    r[i] = ri;
    acc[0] += ri * ri;
  }
  if (reduce_last<1>(acc, cd.partial, cd.ticket, nb)) {
    sc->rnorm = sqrt(acc[0]);
    sc->cycle += 1;
  }
}

// ---- the Newton update -------------------------------------------------------------

// omega = min(1, fraction / max relative change of rho, p, nu_hat)  (implicit.py:54-81)
__global__ void __launch_bounds__(RED_THREADS) k_relax(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  const Canvas& c = cd.c;
  const Config& cfg = cd.cfg;
  const int N = c.ncanvas(), nv = c.nvar;
  int nb, lo, hi;
  if (!chunk_owner(N, nb, lo, hi)) return;
  const double g = cd.P.gamma;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ dU = cd.x;
  double worst[1] = {0.0};
  if (cfg.max_relative_update > 0.0) {
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
  if (reduce_last<1, true>(worst, cd.partial, cd.ticket, nb)) {
    Scalars* sc = cd.sc;
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
__global__ void __launch_bounds__(RED_THREADS) k_accept(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  const Canvas& c = cd.c;
  const Config& cfg = cd.cfg;
  Scalars* sc = cd.sc;
  const int N = c.ncanvas(), nv = c.nvar, n = nv * N;
  int nb, lo, hi;
  if (!chunk_owner(n, nb, lo, hi)) return;
  const double g = cd.P.gamma, om = sc->omega;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ dU = cd.x;
  const double* __restrict__ action = cd.action;
  const double* __restrict__ R = cd.R;
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
  if (reduce_last<3>(acc, cd.partial, cd.ticket, nb)) {
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

__global__ void k_update(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled) return;
  const Scalars* sc = cd.sc;
  if (sc->accept == 0) return;
  const double om = sc->omega;
  double* __restrict__ U = cd.U;
  const double* __restrict__ dU = cd.x;
  const int n = cd.n_vec;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) U[i] = U[i] + om * dU[i];
}

// z = scale * src, optionally V_j = z rounded to the basis type: the Arnoldi step
// without a preconditioner (scale_on: by 1/|w| of the case)
template <class TV>
__global__ void k_scale_copy(const CaseDev* __restrict__ cases, int src_id, int scale_on, int vout_j, int out_id,
                             int check_active) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled || (check_active && cd.sc->active == 0)) return;
  const int n = cd.n_vec;
  const double* __restrict__ src = buf(cd, src_id);
  double* __restrict__ z = buf(cd, out_id);
  TV* vout = vout_j >= 0 ? (TV*)cd.V + (size_t)vout_j * n : nullptr;
  const double s = scale_on ? cd.sc->inv_nrm : 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x = s * src[i];
    if (vout != nullptr) {
      TV xv = TV(x);
      vout[i] = xv;
      x = double(xv);
    }
    z[i] = x;
  }
}

// ---- launch wrappers ------------------------------------------------------------------

// blocks of the basis passes of a case of n elements (and the largest block count any
// reduction uses: the size of a case's partial array)
int reduce_blocks(int n) { return max(max(2 * 148, chunk_blocks(n)), cgs_blocks(n)); }

static dim3 chunk_grid(const BatchDims& d) { return dim3(chunk_blocks(d.n_vec), d.n_cases); }
static dim3 stride_grid(const BatchDims& d) { return dim3(min((d.n_vec + 255) / 256, 148 * 4), d.n_cases); }

void launch_gmres_init(const CaseDev* cases, const BatchDims& d, cudaStream_t st) {
  k_gmres_init<<<chunk_grid(d), RED_THREADS, 0, st>>>(cases, d.n_slots);
}

void launch_cycle_start(const CaseDev* cases, const BatchDims& d, cudaStream_t st) {
  k_cycle_start<<<dim3(1, d.n_cases), 128, 0, st>>>(cases);
}

void launch_cycle_gate(const CaseDev* cases, const BatchDims& d, cudaGraphConditionalHandle gate,
                       unsigned long long* cycles, cudaStream_t st) {
  k_cycle_gate<<<1, 256, 0, st>>>(cases, d.n_cases, gate, cycles);
}

template <class TV, int NK>
static void arnoldi_nk(const CaseDev* cases, const BatchDims& d, int j, cudaStream_t st) {
  dim3 grid(d.cgs_blocks, d.n_cases);
  k_mdot<TV, NK, 0><<<grid, RED_THREADS, 0, st>>>(cases, j + 1, j);
  k_mdot<TV, NK, 1><<<grid, RED_THREADS, 0, st>>>(cases, j + 1, j);
  k_mdot<TV, NK, 2><<<grid, RED_THREADS, 0, st>>>(cases, j + 1, j);
}

template <class TV>
static void arnoldi_t(const CaseDev* cases, const BatchDims& d, int j, cudaStream_t st) {
  const int nk = j + 1;
  if (nk <= 8) arnoldi_nk<TV, 8>(cases, d, j, st);
  else if (nk <= 16) arnoldi_nk<TV, 16>(cases, d, j, st);
  else if (nk <= 32) arnoldi_nk<TV, 32>(cases, d, j, st);
  else arnoldi_nk<TV, 64>(cases, d, j, st);
}

// orthogonalise w against V_0..V_j (CGS2) and append column j of H
void launch_arnoldi_orth(const CaseDev* cases, const BatchDims& d, bool fp32, int j, cudaStream_t st) {
  if (fp32) arnoldi_t<float>(cases, d, j, st);
  else arnoldi_t<double>(cases, d, j, st);
}

void launch_lstsq(const CaseDev* cases, const BatchDims& d, cudaStream_t st) {
  k_lstsq<<<dim3(1, d.n_cases), 64, 0, st>>>(cases);
}

void launch_combine(const CaseDev* cases, const BatchDims& d, bool fp32, cudaStream_t st) {
  if (fp32) k_combine<float><<<stride_grid(d), 256, 0, st>>>(cases);
  else k_combine<double><<<stride_grid(d), 256, 0, st>>>(cases);
}

void launch_cycle_end(const CaseDev* cases, const BatchDims& d, cudaStream_t st) {
  k_cycle_end<<<chunk_grid(d), RED_THREADS, 0, st>>>(cases);
}

void launch_scale_copy(const CaseDev* cases, const BatchDims& d, bool fp32, int src_id, int scale_on, int vout_j,
                       int out_id, int check_active, cudaStream_t st) {
  if (fp32 && vout_j >= 0)
    k_scale_copy<float><<<stride_grid(d), 256, 0, st>>>(cases, src_id, scale_on, vout_j, out_id, check_active);
  else
    k_scale_copy<double><<<stride_grid(d), 256, 0, st>>>(cases, src_id, scale_on, vout_j, out_id, check_active);
}

void launch_newton_update(const CaseDev* cases, const BatchDims& d, cudaStream_t st) {
  k_relax<<<dim3(chunk_blocks(d.cells), d.n_cases), RED_THREADS, 0, st>>>(cases);
  k_accept<<<chunk_grid(d), RED_THREADS, 0, st>>>(cases);
  k_update<<<stride_grid(d), 256, 0, st>>>(cases);
}

}  // namespace jr
