// The line-implicit preconditioner `line_j` (src/jaxrans/solvers/preconditioners.py:209-306):
// block-tridiagonal systems along the line chains (cells linked along j, continued
// through the C-grid wake cut), with the first-order Rusanov approximate Jacobian
//   diag  = sum_f lambda_f (1/CFL + 1/2) I
//   off   = 1/2 A(U_nb, S_out) - 1/2 lambda_f I
// for the mean flow, and scalar chains for the SA row.  Each chain is factored and
// solved exactly; one thread owns one chain and runs the block Thomas recurrence (the
// reference's cyclic reduction gives the same solve to round-off).  Factor rows are
// stored row-major across chains, [(k * E + e) * n_chains + c], so a warp's loads of one
// row are coalesced.  TF is the factor's type (double; float in the mixed form).
#include "device.cuh"

namespace jr {

constexpr int FLOW_E = 48;   // lower, pivot inverse, c_hat: 3 x 16
constexpr int SA_E = 3;      // the scalar chain's lower, pivot inverse, c_hat

// A = d(F.S)/dU (4x4, [row][col]): columns by forward-mode tangents of the flux of the
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

template <class TF, bool SA>
__global__ void k_chain_factor(Canvas cv, Physics P, const double* __restrict__ U, const double* __restrict__ lam,
                               const double* __restrict__ mflux, const double* __restrict__ dflux,
                               const double* __restrict__ dflow, const double* __restrict__ dsa,
                               TF* __restrict__ fflow, TF* __restrict__ fsa) {
  const int n = cv.n_chains;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const int len = cv.ch_len[c];
  const int N = cv.ncanvas();
  TF Cp[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) Cp[r][q] = TF(0);
  TF cps = TF(0);
  for (int k = 0; k < len; ++k) {
    const int cell = cv.ch_cells[k * n + c];
    double Lb[4][4], Ub[4][4];
    if (k > 0) {
      coupling(cv, P, U, lam, cv.ch_down_sign[(k - 1) * n + c], cv.ch_down_face[(k - 1) * n + c],
               cv.ch_cells[(k - 1) * n + c], Lb);
    } else {
      coupling(cv, P, U, lam, 0, 0, 0, Lb);
    }
    if (k + 1 < len) {
      coupling(cv, P, U, lam, cv.ch_up_sign[k * n + c], cv.ch_up_face[k * n + c], cv.ch_cells[(k + 1) * n + c],
               Ub);
    } else {
      coupling(cv, P, U, lam, 0, 0, 0, Ub);
    }
    const double d = dflow[cell];
    TF M[4][4], Pv[4][4], Cn[4][4], Lt[4][4], Ut[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        Lt[r][q] = TF(Lb[r][q]);
        Ut[r][q] = TF(Ub[r][q]);
      }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        TF s = TF(0);
#pragma unroll
        for (int t = 0; t < 4; ++t) s = s + Lt[r][t] * Cp[t][q];
        M[r][q] = (r == q ? TF(d) : TF(0)) - s;
      }
    invert4(M, Pv);
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        TF s = TF(0);
#pragma unroll
        for (int t = 0; t < 4; ++t) s = s + Pv[r][t] * Ut[t][q];
        Cn[r][q] = s;
      }
    TF* row = fflow + (size_t)k * FLOW_E * n + c;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      row[(size_t)e * n] = Lt[e / 4][e % 4];
      row[(size_t)(16 + e) * n] = Pv[e / 4][e % 4];
      row[(size_t)(32 + e) * n] = Cn[e / 4][e % 4];
      Cp[e / 4][e % 4] = Cn[e / 4][e % 4];
    }
    if constexpr (SA) {
      double ls = 0.0, us = 0.0;
      if (k > 0) {
        int sg = cv.ch_down_sign[(k - 1) * n + c], f = cv.ch_down_face[(k - 1) * n + c];
        if (sg != 0) ls = -(fmax(-sg * mflux[f], 0.0) + dflux[f]) / U[cv.ch_cells[(k - 1) * n + c]];
      }
      if (k + 1 < len) {
        int sg = cv.ch_up_sign[k * n + c], f = cv.ch_up_face[k * n + c];
        if (sg != 0) us = -(fmax(-sg * mflux[f], 0.0) + dflux[f]) / U[cv.ch_cells[(k + 1) * n + c]];
      }
      TF ps = TF(1) / (TF(dsa[cell]) - TF(ls) * cps);
      TF cs = ps * TF(us);
      TF* srow = fsa + (size_t)k * SA_E * n + c;
      srow[0] = TF(ls);
      srow[(size_t)n] = ps;
      srow[(size_t)2 * n] = cs;
      cps = cs;
    }
    (void)N;
  }
}

// z = M^-1 (scale * r); with `vout`, also vout = scale * r (the normalised Arnoldi vector).
// Threads past the chains copy the cells on no chain (z = scale * r there).
template <class TF, class TV, bool SA>
__global__ void k_chain_apply(Canvas cv, const TF* __restrict__ fflow, const TF* __restrict__ fsa,
                              const double* __restrict__ r, const double* __restrict__ scale_ptr,
                              const int* __restrict__ skip, TV* __restrict__ vout, double* __restrict__ z) {
  if (skip != nullptr && *skip == 0) return;
  const int n = cv.n_chains;
  const int N = cv.ncanvas();
  const int nv = cv.nvar;
  const double scale = scale_ptr != nullptr ? *scale_ptr : 1.0;
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) {
    t -= n;
    const int stride = gridDim.x * blockDim.x - n;
    for (int e = t; e < cv.n_offchain; e += stride) {
      int idx = cv.offchain[e];
      for (int v = 0; v < nv; ++v) {
        double b = scale * r[v * N + idx];
        if (vout != nullptr) vout[v * N + idx] = TV(b);
        z[v * N + idx] = vout != nullptr ? double(TV(b)) : b;
      }
    }
    return;
  }
  const int c = t;
  const int len = cv.ch_len[c];
  TF d[4] = {TF(0), TF(0), TF(0), TF(0)};
  TF ds = TF(0);
  for (int k = 0; k < len; ++k) {
    const int cell = cv.ch_cells[k * n + c];
    TF b[5];
    for (int v = 0; v < nv; ++v) {
      double x = scale * r[v * N + cell];
      if (vout != nullptr) {
        TV xv = TV(x);
        vout[v * N + cell] = xv;
        x = double(xv);
      }
      b[v] = TF(x);
    }
    const TF* row = fflow + (size_t)k * FLOW_E * n + c;
    TF t4[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      TF s = TF(0);
#pragma unroll
      for (int j = 0; j < 4; ++j) s = s + row[(size_t)(i * 4 + j) * n] * d[j];
      t4[i] = b[i] - s;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      TF s = TF(0);
#pragma unroll
      for (int j = 0; j < 4; ++j) s = s + row[(size_t)(16 + i * 4 + j) * n] * t4[j];
      d[i] = s;
    }
    for (int v = 0; v < 4; ++v) z[v * N + cell] = double(d[v]);
    if constexpr (SA) {
      const TF* srow = fsa + (size_t)k * SA_E * n + c;
      ds = srow[(size_t)n] * (b[4] - srow[0] * ds);
      z[4 * N + cell] = double(ds);
    }
  }
  TF x[4] = {TF(0), TF(0), TF(0), TF(0)};
  TF xs = TF(0);
  for (int k = len - 1; k >= 0; --k) {
    const int cell = cv.ch_cells[k * n + c];
    const TF* row = fflow + (size_t)k * FLOW_E * n + c;
    TF nx[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      TF s = TF(0);
#pragma unroll
      for (int j = 0; j < 4; ++j) s = s + row[(size_t)(32 + i * 4 + j) * n] * x[j];
      nx[i] = TF(z[i * N + cell]) - s;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      x[i] = nx[i];
      z[i * N + cell] = double(nx[i]);
    }
    if constexpr (SA) {
      const TF* srow = fsa + (size_t)k * SA_E * n + c;
      xs = TF(z[4 * N + cell]) - srow[(size_t)2 * n] * xs;
      z[4 * N + cell] = double(xs);
    }
  }
}

template <class TF>
void launch_chain_factor_t(const Canvas& c, const Physics& P, bool sa, const double* U, const double* lam,
                           const double* mflux, const double* dflux, const double* dflow, const double* dsa,
                           void* fflow, void* fsa, cudaStream_t st) {
  int blocks = (c.n_chains + 63) / 64;
  if (sa)
    k_chain_factor<TF, true><<<blocks, 64, 0, st>>>(c, P, U, lam, mflux, dflux, dflow, dsa, (TF*)fflow, (TF*)fsa);
  else
    k_chain_factor<TF, false><<<blocks, 64, 0, st>>>(c, P, U, lam, mflux, dflux, dflow, dsa, (TF*)fflow, (TF*)fsa);
}

void launch_chain_factor(const Canvas& c, const Physics& P, bool sa, bool fp32, const double* U, const double* lam,
                         const double* mflux, const double* dflux, const double* dflow, const double* dsa,
                         void* fflow, void* fsa, cudaStream_t st) {
  if (fp32) launch_chain_factor_t<float>(c, P, sa, U, lam, mflux, dflux, dflow, dsa, fflow, fsa, st);
  else launch_chain_factor_t<double>(c, P, sa, U, lam, mflux, dflux, dflow, dsa, fflow, fsa, st);
}

template <class TF, class TV>
static void apply_t(const Canvas& c, bool sa, const void* fflow, const void* fsa, const double* r, const double* scale,
                    const int* skip, TV* vout, double* z, cudaStream_t st) {
  int threads = c.n_chains + 1024;
  int blocks = (threads + 63) / 64;
  if (sa)
    k_chain_apply<TF, TV, true><<<blocks, 64, 0, st>>>(c, (const TF*)fflow, (const TF*)fsa, r, scale, skip, vout, z);
  else
    k_chain_apply<TF, TV, false><<<blocks, 64, 0, st>>>(c, (const TF*)fflow, (const TF*)fsa, r, scale, skip, vout, z);
}

void launch_chain_apply(const Canvas& c, bool sa, bool fp32, const void* fflow, const void* fsa, const double* r,
                        const double* scale, const int* skip, void* vout, bool vout_fp32, double* z, cudaStream_t st) {
  if (fp32) {
    if (vout_fp32) apply_t<float, float>(c, sa, fflow, fsa, r, scale, skip, (float*)vout, z, st);
    else apply_t<float, double>(c, sa, fflow, fsa, r, scale, skip, (double*)vout, z, st);
  } else {
    if (vout_fp32) apply_t<double, float>(c, sa, fflow, fsa, r, scale, skip, (float*)vout, z, st);
    else apply_t<double, double>(c, sa, fflow, fsa, r, scale, skip, (double*)vout, z, st);
  }
}

}  // namespace jr
