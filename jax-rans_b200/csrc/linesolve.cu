// The line-implicit preconditioner `line_j` (src/jaxrans/solvers/preconditioners.py:209-306):
// block-tridiagonal systems along the line chains (cells linked along j, continued
// through the C-grid wake cut), with the first-order Rusanov approximate Jacobian
//   diag  = sum_f lambda_f (1/CFL + 1/2) I
//   off   = 1/2 A(U_nb, S_out) - 1/2 lambda_f I
// for the mean flow (4x4 blocks), and scalar chains for the SA row.
//
// Each chain is factored and solved by block cyclic reduction, the reference's own
// algorithm (src/jaxrans/core/linalg.py:159-200): ceil(log2 L) levels, each eliminating
// the even rows of a block-tridiagonal system and leaving one on the odd rows.  One CTA
// owns one chain and its threads own rows, so a solve is 2 log2(L) short barriers
// instead of 2L dependent steps.  A chain's factor lives in global memory (L2 resident
// at these sizes), level after level: for the even rows the inverse of the diagonal and
// the off-diagonal blocks, for the odd rows the multipliers alpha and gamma; entries are
// stored [entry][row] so a level's loads are coalesced.  TF is the factor's type
// (double; float in the mixed form).
#include "device.cuh"

namespace jr {

constexpr int LS_THREADS = 128;

// A = d(F.S)/dU (4x4, [row][col]) by forward-mode tangents of the flux of the
// conservative state (physics/euler.py:55-71)
__device__ __forceinline__ void flux_jacobian(const double* q, double sx, double sy, double g, double A[4][4]) {
  double U[4];
  U[0] = q[0];
  U[1] = q[0] * q[1];
  U[2] = q[0] * q[2];
  U[3] = q[3] / (g - 1.0) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    Dual Ud[4], qd[4], F[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) Ud[v] = Dual{U[v], v == k ? 1.0 : 0.0};
    to_prim(Ud, qd, 4, g);
    normal_flux(qd, sx, sy, g, F);
#pragma unroll
    for (int r = 0; r < 4; ++r) A[r][k] = F[r].d;
  }
}

// unpivoted Gauss-Jordan inverse (core/linalg.py:49-77)
template <class S> __device__ __forceinline__ void invert4(const S M[4][4], S Inv[4][4]) {
  S a[4][8];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      a[r][c] = M[r][c];
      a[r][4 + c] = r == c ? S(1) : S(0);
    }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    S p = a[k][k];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[k][c] = a[k][c] / p;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (r == k) continue;
      S f = a[r][k];
#pragma unroll
      for (int c = 0; c < 8; ++c) a[r][c] = a[r][c] - f * a[k][c];
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) Inv[r][c] = a[r][4 + c];
}

template <class S> __device__ __forceinline__ void mm4(const S A[4][4], const S B[4][4], S C[4][4]) {
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      S s = A[r][0] * B[0][c];
#pragma unroll
      for (int t = 1; t < 4; ++t) s = s + A[r][t] * B[t][c];
      C[r][c] = s;
    }
}

template <class S> __device__ __forceinline__ void mv4(const S A[4][4], const S* x, S* y) {
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    S s = A[r][0] * x[0];
#pragma unroll
    for (int t = 1; t < 4; ++t) s = s + A[r][t] * x[t];
    y[r] = s;
  }
}

// block (16 entries) of row r in an [entry][row] array of `rows` rows
template <class S> __device__ __forceinline__ void load4(const S* base, int rows, int r, S B[4][4]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) B[e >> 2][e & 3] = base[(size_t)e * rows + r];
}
template <class S> __device__ __forceinline__ void store4(S* base, int rows, int r, const S B[4][4]) {
#pragma unroll
  for (int e = 0; e < 16; ++e) base[(size_t)e * rows + r] = B[e >> 2][e & 3];
}

__device__ __forceinline__ void face_vector(const Canvas& cv, int f, double& sx, double& sy) {
  const int nfi = cv.nfi();
  if (f < nfi) {
    sx = cv.fi[f];
    sy = cv.fi[nfi + f];
  } else {
    f -= nfi;
    sx = cv.fj[f];
    sy = cv.fj[cv.nfj() + f];
  }
}

__device__ __forceinline__ void prim_at(const Canvas& cv, const Physics& P, const double* U, int idx, double* q) {
  const int N = cv.ncanvas();
  double u[5];
  for (int v = 0; v < cv.nvar; ++v) u[v] = U[v * N + idx];
  to_prim(u, q, cv.nvar, P.gamma);
}

// 1/2 A(q_nb, sign S) - 1/2 lambda I, or zero where the link does not exist
__device__ __forceinline__ void coupling(const Canvas& cv, const Physics& P, const double* U, const double* lam,
                                         int sign, int face, int nb, double B[4][4]) {
  if (sign == 0) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) B[r][c] = 0.0;
    return;
  }
  double sx, sy, q[5];
  face_vector(cv, face, sx, sy);
  prim_at(cv, P, U, nb, q);
  double A[4][4];
  flux_jacobian(q, sign * sx, sign * sy, P.gamma, A);
  double l = lam[face];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) B[r][c] = 0.5 * A[r][c] - (r == c ? 0.5 * l : 0.0);
}

// Sizes of the cyclic-reduction levels of a chain of length L: level l has n_l rows,
// ne = ceil(n/2) even and no = n/2 odd; n_{l+1} = no.  The flow factor of level l is
// 3*16*ne + 2*16*no entries (inverse, lower, upper of the evens; alpha, gamma of the
// odds); after the last level one inverse (16).  The SA factor is the same in scalars.
__device__ __forceinline__ int level_rows(int L, int level) {
  int n = L;
  for (int k = 0; k < level; ++k) n >>= 1;
  return n;
}

// ------------------------------------------------------------------------------------
// Factor: assemble the chain blocks (rows in parallel), then reduce level by level.
// scratch holds the level's reduced system (a, d, c: 3 x 16 x rows) and the next one's.
// ------------------------------------------------------------------------------------
template <class TF, bool SA>
__global__ void __launch_bounds__(LS_MAX_THREADS) k_cr_factor(const CaseDev* __restrict__ cases) {
  __shared__ CaseDev scase;
  if (idle_block(cases[blockIdx.y], (int)blockIdx.x >= cases[blockIdx.y].c.n_chains, 0)) return;
  const CaseDev& cd = stage_case(cases, blockIdx.y, &scase);
  if (!cd.enabled || (int)blockIdx.x >= cd.c.n_chains) return;
  const Canvas& cv = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ lam = cd.lam;
  const double* __restrict__ mflux = cd.mflux;
  const double* __restrict__ dflux = cd.dflux;
  const double* __restrict__ dflow = cd.dflow;
  const double* __restrict__ dsa = cd.dsa;
  TF* __restrict__ fflow = (TF*)cd.fflow;
  TF* __restrict__ fsa = (TF*)cd.fsa;
  TF* __restrict__ scratch = (TF*)cd.scratch;
  const int c = blockIdx.x, n = cv.n_chains;
  const int L = cv.ch_len[c];
  TF* F = fflow + (size_t)cv.ch_fbase[c] * 80;   // flow factor: <= 80 entries per row
  TF* Fs = fsa + (size_t)cv.ch_fbase[c] * 5;     // SA factor: <= 5 scalars per row
  TF* s0 = scratch + (size_t)cv.ch_fbase[c] * 104;   // two level systems: 3*16*L + 3*16*L/2 (+ SA)
  TF* A0 = s0;                 // a, d, c of the current level: 3 x 16 x L
  TF* A1 = s0 + (size_t)48 * L;   // the next level's: 3 x 16 x L/2
  TF* S0 = A1 + (size_t)48 * ((L + 1) / 2);   // SA scalars, current: 3 x L
  TF* S1 = S0 + (size_t)3 * L;                // SA, next: 3 x L/2
  // 1. the blocks of every row
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int cell = cv.ch_cells[k * n + c];
    double Lb[4][4], Ub[4][4];
    coupling(cv, P, U, lam, k > 0 ? cv.ch_down_sign[(k - 1) * n + c] : 0,
             k > 0 ? cv.ch_down_face[(k - 1) * n + c] : 0, k > 0 ? cv.ch_cells[(k - 1) * n + c] : 0, Lb);
    coupling(cv, P, U, lam, k + 1 < L ? cv.ch_up_sign[k * n + c] : 0, k + 1 < L ? cv.ch_up_face[k * n + c] : 0,
             k + 1 < L ? cv.ch_cells[(k + 1) * n + c] : 0, Ub);
    const double d = dflow[cell];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      A0[(size_t)e * L + k] = TF(Lb[e >> 2][e & 3]);
      A0[(size_t)(16 + e) * L + k] = TF((e >> 2) == (e & 3) ? d : 0.0);
      A0[(size_t)(32 + e) * L + k] = TF(Ub[e >> 2][e & 3]);
    }
    if constexpr (SA) {
      double ls = 0.0, us = 0.0;
      if (k > 0) {
        int sg = cv.ch_down_sign[(k - 1) * n + c], f = cv.ch_down_face[(k - 1) * n + c];
        if (sg != 0) ls = -(fmax(-sg * mflux[f], 0.0) + dflux[f]) / U[cv.ch_cells[(k - 1) * n + c]];
      }
      if (k + 1 < L) {
        int sg = cv.ch_up_sign[k * n + c], f = cv.ch_up_face[k * n + c];
        if (sg != 0) us = -(fmax(-sg * mflux[f], 0.0) + dflux[f]) / U[cv.ch_cells[(k + 1) * n + c]];
      }
      S0[k] = TF(ls);
      S0[L + k] = TF(dsa[cell]);
      S0[2 * L + k] = TF(us);
    }
  }
  __syncthreads();
  // 2. the levels
  int rows = L;
  size_t off = 0, offs = 0;
  TF *cur = A0, *nxt = A1, *scur = S0, *snxt = S1;
  while (rows > 1) {
    const int ne = (rows + 1) / 2, no = rows / 2;
    TF* inv = F + off;                    // [16][ne]
    TF* low = inv + (size_t)16 * ne;      // [16][ne]
    TF* upp = low + (size_t)16 * ne;      // [16][ne]
    TF* alp = upp + (size_t)16 * ne;      // [16][no]
    TF* gam = alp + (size_t)16 * no;      // [16][no]
    for (int e = threadIdx.x; e < ne; e += blockDim.x) {
      TF D[4][4], I[4][4], B[4][4];
      load4(cur + (size_t)16 * rows, rows, 2 * e, D);
      invert4(D, I);
      store4(inv, ne, e, I);
      load4(cur, rows, 2 * e, B);
      store4(low, ne, e, B);
      load4(cur + (size_t)32 * rows, rows, 2 * e, B);
      store4(upp, ne, e, B);
      if constexpr (SA) {
        TF* sf = Fs + offs;
        sf[e] = TF(1) / scur[rows + 2 * e];            // inverse
        sf[ne + e] = scur[2 * e];                      // lower
        sf[2 * ne + e] = scur[2 * rows + 2 * e];       // upper
      }
    }
    __syncthreads();
    for (int o = threadIdx.x; o < no; o += blockDim.x) {
      TF Ao[4][4], Co[4][4], I0[4][4], al[4][4], ga[4][4], T[4][4], X[4][4];
      load4(cur, rows, 2 * o + 1, Ao);
      load4(inv, ne, o, I0);
      mm4(Ao, I0, al);
      load4(cur + (size_t)32 * rows, rows, 2 * o + 1, Co);
      const bool has_next = o + 1 < ne;
      if (has_next) {
        TF I1[4][4];
        load4(inv, ne, o + 1, I1);
        mm4(Co, I1, ga);
      } else {
#pragma unroll
        for (int e = 0; e < 16; ++e) ga[e >> 2][e & 3] = TF(0);
      }
      store4(alp, no, o, al);
      store4(gam, no, o, ga);
      // the odd row's new lower, diagonal and upper blocks
      TF lw[4][4], up[4][4], Dn[4][4];
      load4(low, ne, o, lw);
      mm4(al, lw, T);
#pragma unroll
      for (int e = 0; e < 16; ++e) X[e >> 2][e & 3] = -T[e >> 2][e & 3];
      store4(nxt, no, o, X);
      load4(cur + (size_t)16 * rows, rows, 2 * o + 1, Dn);
      load4(upp, ne, o, up);
      mm4(al, up, T);
#pragma unroll
      for (int e = 0; e < 16; ++e) Dn[e >> 2][e & 3] = Dn[e >> 2][e & 3] - T[e >> 2][e & 3];
      if (has_next) {
        load4(low, ne, o + 1, lw);
        mm4(ga, lw, T);
#pragma unroll
        for (int e = 0; e < 16; ++e) Dn[e >> 2][e & 3] = Dn[e >> 2][e & 3] - T[e >> 2][e & 3];
        load4(upp, ne, o + 1, up);
        mm4(ga, up, T);
#pragma unroll
        for (int e = 0; e < 16; ++e) X[e >> 2][e & 3] = -T[e >> 2][e & 3];
      } else {
#pragma unroll
        for (int e = 0; e < 16; ++e) X[e >> 2][e & 3] = TF(0);
      }
      store4(nxt + (size_t)16 * no, no, o, Dn);
      store4(nxt + (size_t)32 * no, no, o, X);
      if constexpr (SA) {
        TF* sf = Fs + offs;
        TF* sal = sf + 3 * ne;
        TF* sga = sal + no;
        TF a_ = scur[2 * o + 1] * sf[o];
        TF g_ = has_next ? scur[2 * rows + 2 * o + 1] * sf[o + 1] : TF(0);
        sal[o] = a_;
        sga[o] = g_;
        snxt[o] = -(a_ * sf[ne + o]);
        TF dn = scur[rows + 2 * o + 1] - a_ * sf[2 * ne + o];
        if (has_next) dn = dn - g_ * sf[ne + o + 1];
        snxt[no + o] = dn;
        snxt[2 * no + o] = has_next ? -(g_ * sf[2 * ne + o + 1]) : TF(0);
      }
    }
    __syncthreads();
    off += (size_t)48 * ne + (size_t)32 * no;
    offs += (size_t)3 * ne + (size_t)2 * no;
    TF* t = cur;
    cur = nxt;
    nxt = t;
    TF* ts = scur;
    scur = snxt;
    snxt = ts;
    rows = no;
  }
  if (threadIdx.x == 0) {
    TF D[4][4], I[4][4];
    load4(cur + 16, 1, 0, D);   // rows == 1: the diagonal block at entries 16..31
    invert4(D, I);
    store4(F + off, 1, 0, I);
    if constexpr (SA) Fs[offs] = TF(1) / scur[1];
  }
}

// ------------------------------------------------------------------------------------
// Apply: z = M^-1 (scale * r) on one chain per CTA.  With `vout`, the scaled input is
// also written there (the normalised Arnoldi vector).  The right-hand side of every
// level is kept in shared memory for the back substitution.
// ------------------------------------------------------------------------------------
// off-chain blocks of a case: enough to cover its cells on no chain, at most 64
__host__ __device__ __forceinline__ int offchain_blocks(int n_offchain) {
  int b = (n_offchain + LS_THREADS - 1) / LS_THREADS;
  return b < 1 ? 1 : (b > 64 ? 64 : b);
}

// ------------------------------------------------------------------------------------
// Staging a chain's factor.  A solve reads every entry of its chain's factor once, level
// by level, and each level waits on its loads before the next barrier: at one chain per
// CTA the solve is a chain of L2 round trips.  The staged form instead copies the chain's
// flow factor (contiguous, 16-byte aligned, a multiple of 64 bytes) into shared memory
// with one bulk asynchronous copy issued at the start, completed on an mbarrier while
// the threads gather the right-hand side, and its SA scalars with plain loads; the
// levels then read shared memory.  It costs the factor's size in shared memory per CTA
// (fewer CTAs per SM), so the plan's autotuner times both forms.
// ------------------------------------------------------------------------------------
// entries of a chain's flow factor: every level's even-row blocks (inverse, lower, upper)
// and odd-row multipliers (alpha, gamma), then the last row's inverse
__host__ __device__ __forceinline__ int cr_chain_entries(int L) {
  int e = 16, rows = L;
  while (rows > 1) {
    const int ne = (rows + 1) / 2, no = rows / 2;
    e += 48 * ne + 32 * no;
    rows = no;
  }
  return e;
}

// entries of a chain's SA factor (three scalars per even row, two per odd row, the last)
__host__ __device__ __forceinline__ int cr_chain_sa_entries(int L) {
  int e = 1, rows = L;
  while (rows > 1) {
    const int ne = (rows + 1) / 2, no = rows / 2;
    e += 3 * ne + 2 * no;
    rows = no;
  }
  return e;
}

constexpr int STAGE_WAIT_TRIES = 1 << 20;      // x a suspend hint of 1 us: about a second
constexpr unsigned STAGE_WAIT_HINT_NS = 1000;
// dynamic shared memory of the staged solve at most: the opt-in limit of one CTA (227 KB,
// static and dynamic together) less room for the kernel's static shared memory
constexpr size_t SMEM_PER_BLOCK_MAX = 232448 - 2048;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// One thread: arm the barrier for `bytes` and start the bulk copy src (global) -> dst
// (this CTA's shared memory).  Both addresses 16-byte aligned, bytes a multiple of 16
// and below 2^20 (the barrier's transaction count).
__device__ __forceinline__ void stage_issue(unsigned long long* bar, void* dst, const void* src, unsigned bytes) {
  const unsigned b = smem_u32(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}

// Wait for the barrier's first phase, a bounded number of tries; false if it gave up.
__device__ __forceinline__ bool stage_wait(unsigned long long* bar, int tries = STAGE_WAIT_TRIES) {
  const unsigned b = smem_u32(bar);
  for (int i = 0; i < tries; ++i) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(b), "r"(0u), "r"(STAGE_WAIT_HINT_NS)
        : "memory");
    if (done) return true;
  }
  return false;
}

// The bounded wait's own check: a barrier armed for 16 bytes that no copy delivers, so the
// wait runs out after `tries` tries and the block reports it -- the path a staged solve
// takes if its copy does not land.  Nothing is in flight when the block exits.
__device__ int g_wait_check;

__global__ void k_wait_limit_check(int tries) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    const unsigned b = smem_u32(&bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(16u) : "memory");
  }
  __syncthreads();
  const bool ok = stage_wait(&bar, tries);
  const bool gave_up = __syncthreads_or(!ok);
  if (threadIdx.x == 0) g_wait_check = gave_up ? (int)ST_STAGE_FAILED : 0;
}

// status <- the check's status word (ST_STAGE_FAILED when the wait ran out, as it must)
int wait_limit_check(int tries, int* status, cudaStream_t st) {
  const int zero = -1;
  cudaMemcpyToSymbolAsync(g_wait_check, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st);
  k_wait_limit_check<<<1, 64, 0, st>>>(tries);
  cudaMemcpyFromSymbolAsync(status, g_wait_check, sizeof(int), 0, cudaMemcpyDeviceToHost, st);
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : 1;
}

// Shared memory of the line solve: [flow factor | SA factor] when staged, then the
// level-concatenated right-hand sides (at most 2 L rows of 5).  Stage s >= 1 reserves
// the largest footprint of any chain of up to max_L >> (s - 1) cells: a chain stages
// its levels from the first whose remaining rows fit (the longest chain from level s-1)
// and reads the levels above from global memory, while the copy is in flight.
struct ApplyLayout {
  int ent_f, ent_s;       // staged entries (0 unstaged)
  size_t off_s, off_b;    // byte offsets of the SA factor and of the right-hand sides
  size_t bytes;           // dynamic shared memory of a CTA
};

static ApplyLayout apply_layout(int max_L, bool fp32, int stage) {
  const size_t tb = fp32 ? 4 : 8;
  ApplyLayout a{0, 0, 0, 0, 0};
  if (stage > 0) {
    const int Lb = (max_L >> (stage - 1)) > 1 ? (max_L >> (stage - 1)) : 1;
    for (int l = 1; l <= Lb; ++l) {
      a.ent_f = cr_chain_entries(l) > a.ent_f ? cr_chain_entries(l) : a.ent_f;
      a.ent_s = cr_chain_sa_entries(l) > a.ent_s ? cr_chain_sa_entries(l) : a.ent_s;
    }
    a.off_s = ((size_t)a.ent_f * tb + 127) / 128 * 128;
    a.off_b = a.off_s + ((size_t)a.ent_s * tb + 15) / 16 * 16;
  }
  a.bytes = a.off_b + (size_t)2 * max_L * 5 * tb + 64;
  return a;
}

// whether the line solve's stage form fits one CTA's shared memory for chains up to max_L
bool apply_stage_fits(int max_L, bool fp32, int stage) {
  return stage == 0 || (stage >= 1 && stage <= APPLY_STAGES && apply_layout(max_L, fp32, stage).bytes <= SMEM_PER_BLOCK_MAX);
}

// One level of the reduction: the odd rows' right-hand sides of the next level,
// bn[o] = b[2o+1] - alpha_o b[2o] - gamma_o b[2o+2] (4x4 blocks; scalars for SA).
template <class TF, bool SA>
__device__ __forceinline__ void cr_reduce_level(const TF* alp, const TF* gam, const TF* sal, const TF* sga, const TF* b,
                                                TF* bn, int rows) {
  const int no = rows / 2;
  for (int o = threadIdx.x; o < no; o += blockDim.x) {
    TF al[4][4], ga[4][4], t[4], u[4];
    load4(alp, no, o, al);
    load4(gam, no, o, ga);
    TF be[4], bo[4], bx[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      be[v] = b[(2 * o) * 5 + v];
      bo[v] = b[(2 * o + 1) * 5 + v];
      bx[v] = 2 * o + 2 < rows ? b[(2 * o + 2) * 5 + v] : TF(0);
    }
    mv4(al, be, t);
    mv4(ga, bx, u);
#pragma unroll
    for (int v = 0; v < 4; ++v) bn[o * 5 + v] = bo[v] - t[v] - u[v];
    if constexpr (SA) {
      TF bx4 = 2 * o + 2 < rows ? b[(2 * o + 2) * 5 + 4] : TF(0);
      bn[o * 5 + 4] = b[(2 * o + 1) * 5 + 4] - sal[o] * b[(2 * o) * 5 + 4] - sga[o] * bx4;
    }
  }
}

// One level of the back substitution: the even rows' solution from the odd rows' x,
// x_e = D_e^-1 (b[2e] - lower_e x[e-1] - upper_e x[e]), kept in registers (xe, xs: up
// to 4 rows per thread) until every thread has read b.
template <class TF, bool SA>
__device__ __forceinline__ void cr_back_level(const TF* inv, const TF* si, const TF* b, const TF* x, int rows, TF* xe,
                                              TF* xs) {
  const int ne = (rows + 1) / 2, no = rows / 2;
  const TF* low = inv + (size_t)16 * ne;
  const TF* upp = low + (size_t)16 * ne;
  int cnt = 0;
  for (int e = threadIdx.x; e < ne; e += blockDim.x, ++cnt) {
    TF I[4][4], lw[4][4], up[4][4], t[4], u[4], w[4], res[4];
    load4(inv, ne, e, I);
    load4(low, ne, e, lw);
    load4(upp, ne, e, up);
    TF xp[4], xn[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      xp[v] = e >= 1 ? x[(e - 1) * 5 + v] : TF(0);
      xn[v] = e < no ? x[e * 5 + v] : TF(0);
    }
    mv4(lw, xp, t);
    mv4(up, xn, u);
#pragma unroll
    for (int v = 0; v < 4; ++v) w[v] = b[(2 * e) * 5 + v] - t[v] - u[v];
    mv4(I, w, res);
#pragma unroll
    for (int v = 0; v < 4; ++v) xe[cnt * 4 + v] = res[v];
    if constexpr (SA) {
      TF xps = e >= 1 ? x[(e - 1) * 5 + 4] : TF(0);
      TF xns = e < no ? x[e * 5 + 4] : TF(0);
      xs[cnt] = si[e] * (b[(2 * e) * 5 + 4] - si[ne + e] * xps - si[2 * ne + e] * xns);
    }
  }
}

// src_id: the right-hand side buffer; scale_on: multiply it by the case's 1/|w|;
// vout_j >= 0: also write the scaled input to basis vector j; out_id: the result.
// STAGE: the chain's factor from its first level whose remaining rows fit ent_f flow
// entries (and ent_s SA entries) is copied into shared memory (byte offsets 0 and off_s)
// at the start; the right-hand sides at off_b.
template <class TF, class TV, bool SA, bool STAGE>
__global__ void __launch_bounds__(LS_MAX_THREADS) k_cr_apply(const CaseDev* __restrict__ cases, int src_id, int scale_on,
                                                         int vout_j, int out_id, int check_active, int ent_f,
                                                         int ent_s, int off_s, int off_b) {
  __shared__ CaseDev scase;
  {
    const Canvas& g = cases[blockIdx.y].c;
    if (idle_block(cases[blockIdx.y], (int)blockIdx.x >= g.n_chains + offchain_blocks(g.n_offchain), check_active))
      return;
  }
  const CaseDev& cd = stage_case(cases, blockIdx.y, &scase);
  if (!cd.enabled || (check_active && cd.sc->active == 0)) return;
  const Canvas& cv = cd.c;
  const TF* __restrict__ fflow = (const TF*)cd.fflow;
  const TF* __restrict__ fsa = (const TF*)cd.fsa;
  const double* __restrict__ r = buf(cd, src_id);
  double* __restrict__ z = buf(cd, out_id);
  TV* __restrict__ vout = vout_j >= 0 ? (TV*)cd.V + (size_t)vout_j * cd.n_vec : nullptr;
  const int N = cv.ncanvas(), nv = cv.nvar, n = cv.n_chains;
  const double scale = scale_on ? cd.sc->inv_nrm : 1.0;
  if ((int)blockIdx.x >= n + offchain_blocks(cv.n_offchain)) return;
  if ((int)blockIdx.x >= n) {
    // the cells on no chain: z = scale * r
    const int stride = offchain_blocks(cv.n_offchain) * blockDim.x;
    for (int e = (blockIdx.x - n) * blockDim.x + threadIdx.x; e < cv.n_offchain; e += stride) {
      int idx = cv.offchain[e];
      for (int v = 0; v < nv; ++v) {
        double b = scale * r[v * N + idx];
        if (vout != nullptr) {
          TV bv = TV(b);
          vout[v * N + idx] = bv;
          b = double(bv);
        }
        z[v * N + idx] = b;
      }
    }
    return;
  }
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long stage_bar;
  const int c = blockIdx.x;
  const int L = cv.ch_len[c];
  TF* bs = reinterpret_cast<TF*>(smem_raw + off_b);   // [level-concatenated rows][5]
  const TF* Fg = fflow + (size_t)cv.ch_fbase[c] * 80;
  const TF* Fsg = fsa + (size_t)cv.ch_fbase[c] * 5;
  TF* const sf = reinterpret_cast<TF*>(smem_raw);
  TF* const ss = reinterpret_cast<TF*>(smem_raw + off_s);
  // levels [0, k0) read the factor from global memory, the rest (from entry off0, SA
  // entry offs0) from the staged copy
  int k0 = 1 << 30;
  size_t off0 = 0, offs0 = 0;
  if constexpr (STAGE) {
    int rows0 = L;
    k0 = 0;
    while (cr_chain_entries(rows0) > ent_f || (SA && cr_chain_sa_entries(rows0) > ent_s)) {
      const int ne = (rows0 + 1) / 2, no = rows0 / 2;
      off0 += (size_t)48 * ne + (size_t)32 * no;
      offs0 += (size_t)3 * ne + (size_t)2 * no;
      rows0 = no;
      ++k0;
    }
    const int ef = cr_chain_entries(rows0), es = cr_chain_sa_entries(rows0);
    const bool aligned = ((smem_u32(sf) | (unsigned)reinterpret_cast<uintptr_t>(Fg + off0)) & 15u) == 0;
    if (ef > ent_f || !aligned) {   // not reached: ent_f >= 16 (one row) and 64-byte levels
      if (threadIdx.x == 0) atomicOr(&cd.sc->status, (int)ST_STAGE_FAILED);
      return;
    }
    if (threadIdx.x == 0) stage_issue(&stage_bar, sf, Fg + off0, (unsigned)(ef * sizeof(TF)));
    if constexpr (SA)
      for (int k = threadIdx.x; k < es; k += blockDim.x) ss[k] = Fsg[offs0 + k];
  }
  // gather the right-hand side
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int cell = cv.ch_cells[k * n + c];
    for (int v = 0; v < nv; ++v) {
      double b = scale * r[v * N + cell];
      if (vout != nullptr) {
        TV bv = TV(b);
        vout[v * N + cell] = bv;
        b = double(bv);
      }
      bs[k * 5 + v] = TF(b);
    }
  }
  __syncthreads();
  // before the first staged level: wait for the copy (uniform in the CTA)
  auto staged_ready = [&]() {
    const bool ok = stage_wait(&stage_bar);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) atomicOr(&cd.sc->status, (int)ST_STAGE_FAILED);
      stage_wait(&stage_bar);   // a copy still in flight lands in this CTA's shared memory
      return false;
    }
    return true;
  };
  // reduce: b_odd <- b_odd - alpha b_even - gamma b_next_even, level by level
  int rows = L, lev = 0;
  size_t off = 0, offs = 0, boff = 0;
  while (rows > 1) {
    const int ne = (rows + 1) / 2, no = rows / 2;
    TF* b = bs + boff * 5;
    TF* bn = bs + (boff + rows) * 5;
    if (!STAGE || lev < k0) {
      const TF* alp = Fg + off + (size_t)48 * ne;
      const TF* sal = Fsg + offs + 3 * ne;
      cr_reduce_level<TF, SA>(alp, alp + (size_t)16 * no, sal, sal + no, b, bn, rows);
    } else {
      if (lev == k0 && !staged_ready()) return;
      const TF* alp = sf + (off - off0) + (size_t)48 * ne;
      const TF* sal = ss + (offs - offs0) + 3 * ne;
      cr_reduce_level<TF, SA>(alp, alp + (size_t)16 * no, sal, sal + no, b, bn, rows);
    }
    __syncthreads();
    off += (size_t)48 * ne + (size_t)32 * no;
    offs += (size_t)3 * ne + (size_t)2 * no;
    boff += rows;
    rows = no;
    ++lev;
  }
  if (STAGE && lev == k0 && !staged_ready()) return;   // only the last row staged
  // the last row, then substitute back level by level; x of a level overwrites its b
  if (threadIdx.x == 0) {
    TF* b = bs + boff * 5;
    TF I[4][4], x[4];
    if constexpr (STAGE) load4(sf + (off - off0), 1, 0, I);
    else load4(Fg + off, 1, 0, I);
    mv4(I, b, x);
#pragma unroll
    for (int v = 0; v < 4; ++v) b[v] = x[v];
    if constexpr (SA) b[4] = (STAGE ? ss[offs - offs0] : Fsg[offs]) * b[4];
  }
  __syncthreads();
  // walk the levels back: recompute their offsets from the top
  const int depth = lev;
  for (lev = depth - 1; lev >= 0; --lev) {
    int rws = L;
    size_t of = 0, ofs = 0, bo_ = 0;
    for (int k = 0; k < lev; ++k) {
      int ne_ = (rws + 1) / 2, no_ = rws / 2;
      of += (size_t)48 * ne_ + (size_t)32 * no_;
      ofs += (size_t)3 * ne_ + (size_t)2 * no_;
      bo_ += rws;
      rws = no_;
    }
    const int ne = (rws + 1) / 2, no = rws / 2;
    TF* b = bs + bo_ * 5;           // this level's right-hand side; becomes its solution
    const TF* x = bs + (bo_ + rws) * 5;   // the next level's solution (the odd rows)
    // evens from the odd solution; the odds copied into place after a barrier
    TF xe[4 * 4];   // up to 4 even rows per thread kept in registers when rows <= 4*threads
    TF xs[4];
    if (!STAGE || lev < k0) cr_back_level<TF, SA>(Fg + of, Fsg + ofs, b, x, rws, xe, xs);
    else cr_back_level<TF, SA>(sf + (of - off0), ss + (ofs - offs0), b, x, rws, xe, xs);
    __syncthreads();
    int cnt = 0;
    for (int e = threadIdx.x; e < ne; e += blockDim.x, ++cnt) {
#pragma unroll
      for (int v = 0; v < 4; ++v) b[(2 * e) * 5 + v] = xe[cnt * 4 + v];
      if constexpr (SA) b[(2 * e) * 5 + 4] = xs[cnt];
    }
    for (int o = threadIdx.x; o < no; o += blockDim.x)
      for (int v = 0; v < 5; ++v) b[(2 * o + 1) * 5 + v] = x[o * 5 + v];
    __syncthreads();
  }
  // scatter
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int cell = cv.ch_cells[k * n + c];
    for (int v = 0; v < nv; ++v) z[v * N + cell] = double(bs[k * 5 + v]);
  }
}

// ------------------------------------------------------------------------------------
// The coupled (5x5) form of the line blocks: the SA row also depends on the neighbours'
// mean flow, through half the Jacobian of its convective flux rho nu_hat V.S,
// [-nu_hat vn, nu_hat Sx, nu_hat Sy, 0] at the neighbour's state (the mean-flow rows do
// not depend on rho nu_hat).  The blocks are block lower triangular, so the solve is the
// split solve followed by one more SA chain solve: z_sa -= M_sa^-1 (C z_flow), C the
// coupling along the chain.  This kernel does that second step, one CTA per chain, with
// the SA factor of the split form and the same cyclic-reduction formulas.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double sa_coupling_dot(const Canvas& cv, const Physics& P, const double* U,
                                                  const double* z, int sign, int face, int nb) {
  if (sign == 0) return 0.0;
  double sx, sy, q[5];
  face_vector(cv, face, sx, sy);
  sx *= sign;
  sy *= sign;
  prim_at(cv, P, U, nb, q);
  const int N = cv.ncanvas();
  const double nu = q[4], vn = q[1] * sx + q[2] * sy;
  return 0.5 * ((-nu * vn) * z[nb] + (nu * sx) * z[N + nb] + (nu * sy) * z[2 * N + nb]);
}

template <class TF>
__global__ void __launch_bounds__(LS_MAX_THREADS) k_cr_sa_couple(const CaseDev* __restrict__ cases, int out_id,
                                                                 int check_active) {
  __shared__ CaseDev scase;
  if (idle_block(cases[blockIdx.y], (int)blockIdx.x >= cases[blockIdx.y].c.n_chains, check_active)) return;
  const CaseDev& cd = stage_case(cases, blockIdx.y, &scase);
  const Canvas& cv = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  double* __restrict__ z = buf(cd, out_id);
  const TF* __restrict__ fsa = (const TF*)cd.fsa;
  const int N = cv.ncanvas(), n = cv.n_chains, c = blockIdx.x;
  const int L = cv.ch_len[c];
  const TF* Fs = fsa + (size_t)cv.ch_fbase[c] * 5;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  TF* bs = reinterpret_cast<TF*>(smem_raw);   // level-concatenated rows, one scalar each
  // 1. the right-hand side C z_flow along the chain
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    double t = 0.0;
    if (k > 0)
      t += sa_coupling_dot(cv, P, U, z, cv.ch_down_sign[(k - 1) * n + c], cv.ch_down_face[(k - 1) * n + c],
                           cv.ch_cells[(k - 1) * n + c]);
    if (k + 1 < L)
      t += sa_coupling_dot(cv, P, U, z, cv.ch_up_sign[k * n + c], cv.ch_up_face[k * n + c],
                           cv.ch_cells[(k + 1) * n + c]);
    bs[k] = TF(t);
  }
  __syncthreads();
  // 2. the SA chain solve (the split apply's scalar formulas)
  int rows = L;
  size_t offs = 0, boff = 0;
  while (rows > 1) {
    const int ne = (rows + 1) / 2, no = rows / 2;
    const TF* sal = Fs + offs + 3 * ne;
    const TF* sga = sal + no;
    TF* b = bs + boff;
    TF* bn = bs + boff + rows;
    for (int o = threadIdx.x; o < no; o += blockDim.x) {
      TF bx = 2 * o + 2 < rows ? b[2 * o + 2] : TF(0);
      bn[o] = b[2 * o + 1] - sal[o] * b[2 * o] - sga[o] * bx;
    }
    __syncthreads();
    offs += (size_t)3 * ne + (size_t)2 * no;
    boff += rows;
    rows = no;
  }
  if (threadIdx.x == 0) bs[boff] = Fs[offs] * bs[boff];
  __syncthreads();
  int depth = 0;
  for (int m = L; m > 1; m >>= 1) ++depth;
  for (int lev = depth - 1; lev >= 0; --lev) {
    int rws = L;
    size_t ofs = 0, bo_ = 0;
    for (int k = 0; k < lev; ++k) {
      int ne_ = (rws + 1) / 2, no_ = rws / 2;
      ofs += (size_t)3 * ne_ + (size_t)2 * no_;
      bo_ += rws;
      rws = no_;
    }
    const int ne = (rws + 1) / 2, no = rws / 2;
    const TF* si = Fs + ofs;
    TF* b = bs + bo_;
    const TF* x = bs + bo_ + rws;   // the next level's solution (the odd rows)
    TF xe[4];
    int cnt = 0;
    for (int e = threadIdx.x; e < ne; e += blockDim.x, ++cnt) {
      TF xps = e >= 1 ? x[e - 1] : TF(0);
      TF xns = e < no ? x[e] : TF(0);
      xe[cnt] = si[e] * (b[2 * e] - si[ne + e] * xps - si[2 * ne + e] * xns);
    }
    __syncthreads();
    cnt = 0;
    for (int e = threadIdx.x; e < ne; e += blockDim.x, ++cnt) b[2 * e] = xe[cnt];
    for (int o = threadIdx.x; o < no; o += blockDim.x) b[2 * o + 1] = x[o];
    __syncthreads();
  }
  // 3. z_sa -= the solution
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int cell = cv.ch_cells[k * n + c];
    z[4 * N + cell] -= double(bs[k]);
  }
}

size_t cr_couple_smem(int max_L, bool fp32) { return (size_t)2 * max_L * (fp32 ? 4 : 8) + 64; }

// z_sa -= M_sa^-1 (C z_flow) on every chain: the coupled form's second SA solve
void launch_chain_couple(const CaseDev* cases, const BatchDims& d, bool fp32, int out_id, int check_active,
                         cudaStream_t st) {
  dim3 grid(d.chain_blocks, d.n_cases);
  const int th = d.ls_apply_threads > 0 ? d.ls_apply_threads : LS_THREADS;
  const size_t smem = cr_couple_smem(d.max_L, fp32);
  if (fp32) k_cr_sa_couple<float><<<grid, th, smem, st>>>(cases, out_id, check_active);
  else k_cr_sa_couple<double><<<grid, th, smem, st>>>(cases, out_id, check_active);
}


void launch_chain_factor(const CaseDev* cases, const BatchDims& d, bool sa, bool fp32, cudaStream_t st) {
  dim3 grid(d.chain_blocks, d.n_cases);
  const int th = d.ls_factor_threads > 0 ? d.ls_factor_threads : LS_THREADS;
  if (fp32) {
    if (sa) k_cr_factor<float, true><<<grid, th, 0, st>>>(cases);
    else k_cr_factor<float, false><<<grid, th, 0, st>>>(cases);
  } else {
    if (sa) k_cr_factor<double, true><<<grid, th, 0, st>>>(cases);
    else k_cr_factor<double, false><<<grid, th, 0, st>>>(cases);
  }
}

template <class TF, class TV>
static void apply_t(const CaseDev* cases, const BatchDims& d, bool sa, int src_id, int scale_on, int vout_j, int out_id,
                    int check_active, cudaStream_t st) {
  dim3 grid(d.chain_blocks, d.n_cases);
  const bool fp32 = sizeof(TF) == 4;
  const int stage = apply_stage_fits(d.max_L, fp32, d.ls_apply_stage) ? d.ls_apply_stage : 0;
  const ApplyLayout a = apply_layout(d.max_L, fp32, stage);
  const int th = d.ls_apply_threads > 0 ? d.ls_apply_threads : LS_THREADS;
  const int os = (int)a.off_s, ob = (int)a.off_b;
  if (stage > 0) {
    if (sa)
      k_cr_apply<TF, TV, true, true><<<grid, th, a.bytes, st>>>(cases, src_id, scale_on, vout_j, out_id, check_active,
                                                                a.ent_f, a.ent_s, os, ob);
    else
      k_cr_apply<TF, TV, false, true><<<grid, th, a.bytes, st>>>(cases, src_id, scale_on, vout_j, out_id, check_active,
                                                                 a.ent_f, a.ent_s, os, ob);
  } else {
    if (sa)
      k_cr_apply<TF, TV, true, false><<<grid, th, a.bytes, st>>>(cases, src_id, scale_on, vout_j, out_id, check_active,
                                                                 0, 0, 0, 0);
    else
      k_cr_apply<TF, TV, false, false><<<grid, th, a.bytes, st>>>(cases, src_id, scale_on, vout_j, out_id,
                                                                  check_active, 0, 0, 0, 0);
  }
}

// z = M^-1 (scale * src) for every case; vout_j >= 0 writes the scaled input to basis
// vector j (FP32 when the basis is)
void launch_chain_apply(const CaseDev* cases, const BatchDims& d, bool sa, bool fp32, int src_id, int scale_on,
                        int vout_j, int out_id, int check_active, cudaStream_t st) {
  if (fp32) apply_t<float, float>(cases, d, sa, src_id, scale_on, vout_j, out_id, check_active, st);
  else apply_t<double, double>(cases, d, sa, src_id, scale_on, vout_j, out_id, check_active, st);
}

int chain_grid_blocks(int n_chains, int n_offchain) { return n_chains + offchain_blocks(n_offchain); }

// A thread of the solve keeps up to four even rows of a level in registers, so a block
// must have at least a quarter as many threads as the longest chain has even rows.
bool apply_threads_valid(int threads, int max_L) { return 4 * threads >= (max_L + 1) / 2 && threads <= LS_MAX_THREADS; }

void configure_line_kernels(int max_L) {
  cudaFuncSetAttribute(k_cr_sa_couple<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)cr_couple_smem(max_L, false));
  cudaFuncSetAttribute(k_cr_sa_couple<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)cr_couple_smem(max_L, true));
  const int s8 = (int)apply_layout(max_L, false, 0).bytes, s4 = (int)apply_layout(max_L, true, 0).bytes;
  const int most = (int)SMEM_PER_BLOCK_MAX;
  cudaFuncSetAttribute(k_cr_apply<double, double, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s8);
  cudaFuncSetAttribute(k_cr_apply<double, double, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s8);
  cudaFuncSetAttribute(k_cr_apply<float, float, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s4);
  cudaFuncSetAttribute(k_cr_apply<float, float, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s4);
  cudaFuncSetAttribute(k_cr_apply<double, double, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
  cudaFuncSetAttribute(k_cr_apply<double, double, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
  cudaFuncSetAttribute(k_cr_apply<float, float, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
  cudaFuncSetAttribute(k_cr_apply<float, float, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
}

}  // namespace jr
