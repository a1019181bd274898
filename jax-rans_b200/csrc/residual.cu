// The residual R(U) of one canvas and the exact first-order J.v, in one tile kernel.
//
// Follows src/jaxrans/numerics/residual.py:54-334 (block_residual, the ghost fill, the
// edge pad that interior cells never reach), with the SA row of turbulence.py:112-151
// and the viscous flux of residual.py:94-124.  Each CTA owns a 15 x 16 tile of canvas
// cells: it stages the primitive state of the tile plus a 2-cell halo in shared memory
// (prim(U) computed on the fly for block cells, ghost cells read from the ghost-filled
// buffer), computes every face flux of the tile once into shared memory, then sums the
// faces of each cell -- a per-cell reduction with no atomics.  The same source gives
// R(U) (T = double) and dR1/dU . v (T = Dual, first-order faces).
#include "device.cuh"

namespace jr {

__device__ __forceinline__ bool interior_at(const Canvas& c, int i, int j) {
  return i >= 0 && i < c.NI && j >= 0 && j < c.NJ && c.interior[i * c.NJ + j];
}

// primitive state of canvas cell `idx`: prim(U) on block cells, the ghost buffer elsewhere
template <class T>
__device__ __forceinline__ void load_prim(const Canvas& c, const Physics& P, int idx, const double* U,
                                          const double* V, const double* qg, const double* dqg, T* q) {
  const int N = c.ncanvas();
  if (c.interior[idx]) {
    T u[5];
    for (int v = 0; v < c.nvar; ++v) {
      double x = U[v * N + idx];
      if constexpr (sizeof(T) == sizeof(Dual)) {
        u[v] = T{x, V[v * N + idx]};
      } else {
        u[v] = x;
      }
    }
    to_prim(u, q, c.nvar, P.gamma);
  } else {
    for (int v = 0; v < c.nvar; ++v) {
      double x = qg[v * N + idx];
      if constexpr (sizeof(T) == sizeof(Dual)) {
        q[v] = T{x, dqg[v * N + idx]};
      } else {
        q[v] = x;
      }
    }
  }
}

// the same with the case's variable count NV (== c.nvar) fixed at compile time, so the
// cell's values stay in registers
template <int NV, class T>
__device__ __forceinline__ void load_prim_n(const Canvas& c, const Physics& P, int idx, const double* U,
                                            const double* V, const double* qg, const double* dqg, T* q) {
  const int N = c.ncanvas();
  if (c.interior[idx]) {
    T u[5];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double x = U[v * N + idx];
      if constexpr (sizeof(T) == sizeof(Dual)) {
        u[v] = T{x, V[v * N + idx]};
      } else {
        u[v] = x;
      }
    }
    to_prim(u, q, NV, P.gamma);
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double x = qg[v * N + idx];
      if constexpr (sizeof(T) == sizeof(Dual)) {
        q[v] = T{x, dqg[v * N + idx]};
      } else {
        q[v] = x;
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// Ghost fill (src/jaxrans/numerics/boundary.py:257-267 and the stages of
// src/jaxrans/mesh/atlas.py:331-367): one CTA per case; stage 1 (j sides), then
// stage 2 (i sides and corners, which read stage-1 ghosts).  T = Dual fills the
// tangent of the ghosts (dqg) for a J.v; the base ghosts are left as they are.
// ------------------------------------------------------------------------------------

template <class T>
__device__ void point_vortex_state(const Physics& P, double dx, double dy, T circ, T* out) {
  const double g = P.gamma;
  double rho_f = P.q_inf[0], u_f = P.q_inf[1], v_f = P.q_inf[2], p_f = P.q_inf[3];
  double a2 = g * p_f / rho_f;
  double speed2 = u_f * u_f + v_f * v_f;
  double mach2 = speed2 / a2;
  double alpha = atan2(v_f, u_f);
  double r = hypot(dx, dy);
  double theta = atan2(dy, dx);
  double st = sin(theta - alpha);
  T strength = circ * sqrt(1.0 - mach2) / (2.0 * 3.141592653589793 * r * (1.0 - mach2 * (st * st)));
  T u = u_f + strength * sin(theta);
  T v = v_f - strength * cos(theta);
  T ratio = 1.0 + 0.5 * (g - 1.0) * (speed2 - u * u - v * v) / a2;
  out[0] = rho_f * dpow(ratio, 1.0 / (g - 1.0));
  out[1] = u;
  out[2] = v;
  out[3] = p_f * dpow(ratio, g / (g - 1.0));
  out[4] = cst<T>(P.q_inf[4]);
}

template <class T>
__device__ void condition(const Physics& P, int kind, const T* q, const double* geom, T circ, T* out) {
  const int nv = P.nvar;
  const double nx = geom[0], ny = geom[1];
  const double g = P.gamma;
  switch (kind) {
    case G_SLIP:
    case G_SYMMETRY: {
      T vn = q[1] * nx + q[2] * ny;
      out[0] = q[0];
      out[1] = q[1] - 2.0 * vn * nx;
      out[2] = q[2] - 2.0 * vn * ny;
      out[3] = q[3];
      if (nv > 4) out[4] = kind == G_SLIP ? -q[4] : q[4];
      return;
    }
    case G_NOSLIP:
      out[0] = q[0];
      out[1] = -q[1];
      out[2] = -q[2];
      out[3] = q[3];
      if (nv > 4) out[4] = -q[4];
      return;
    case G_FARFIELD: {
      T ref[5];
      if (P.far_field == 1) {
        point_vortex_state(P, geom[2] - P.quarter_chord[0], geom[3] - P.quarter_chord[1], circ, ref);
      } else {
        for (int v = 0; v < 5; ++v) ref[v] = cst<T>(P.q_inf[v]);
      }
      characteristic(q, nx, ny, ref, nv, g, out);
      return;
    }
    case G_INFLOW: {
      double g1 = g - 1.0;
      double t_f = g * P.q_inf[3] / P.q_inf[0];
      double speed_f = hypot(P.q_inf[1], P.q_inf[2]);
      double t_total = t_f + 0.5 * g1 * speed_f * speed_f;
      double p_total = P.q_inf[3] * pow(t_total / t_f, g / g1);
      T pb = q[3];
      T mach2 = dmax(2.0 / g1 * (dpow(p_total / pb, g1 / g) - 1.0), 0.0);
      T tb = t_total / (1.0 + 0.5 * g1 * mach2);
      T speed = dsqrt(mach2 * tb);
      out[0] = g * pb / tb;
      out[1] = speed * P.q_inf[1] / speed_f;
      out[2] = speed * P.q_inf[2] / speed_f;
      out[3] = pb;
      if (nv > 4) out[4] = cst<T>(P.q_inf[4]);
      return;
    }
    case G_OUTFLOW:
      for (int v = 0; v < nv; ++v) out[v] = q[v];
      out[3] = cst<T>(P.q_inf[3]);
      return;
    default:
      for (int v = 0; v < nv; ++v) out[v] = q[v];
  }
}

// the value a ghost record gives, from its source state
template <class T>
__device__ __forceinline__ void eval_record(const Canvas& c, const Physics& P, int s, int r, const T* q, T circ,
                                            T* out) {
  const int kind = c.g_kind[s][r];
  if (kind == G_COPY) {
    for (int v = 0; v < c.nvar; ++v) out[v] = q[v];
  } else {
    condition<T>(P, kind, q, c.g_geom[s] + 4 * r, circ, out);
  }
}

// Both stages in one launch: a stage-2 record whose source is a stage-1 ghost (a
// corner) evaluates that stage-1 record itself rather than reading it, so no record
// waits on another and every CTA works independently.
template <class T>
__global__ void __launch_bounds__(GHOST_THREADS) k_ghosts(const CaseDev* __restrict__ cases, int tangent_id,
                                                          int check_active) {
  __shared__ CaseDev scase;
  {
    const Canvas& g = cases[blockIdx.y].c;
    if (idle_block(cases[blockIdx.y], (int)(blockIdx.x * blockDim.x) >= g.n_ghost[0] + g.n_ghost[1], check_active))
      return;
  }
  const CaseDev& cd = stage_case(cases, blockIdx.y, &scase);
  if (!cd.enabled || (check_active && cd.sc->active == 0)) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* U = cd.U;
  const double* V = tangent_id >= 0 ? buf(cd, tangent_id) : nullptr;
  double* qg = cd.qg;
  double* dqg = cd.dqg;
  const int N = c.ncanvas();
  if ((int)blockIdx.x * (int)blockDim.x >= c.n_ghost[0] + c.n_ghost[1]) return;
  __shared__ double red_v[GHOST_THREADS / 32][2], red_d[GHOST_THREADS / 32][2];
  __shared__ T circ_s;
  T circ = cst<T>(0.0);
  if (P.far_field == 1) {
    // Kutta-Joukowski circulation of the wall pressure lift (boundary.py:227-240)
    T fx = cst<T>(0.0), fy = cst<T>(0.0);
    for (int w = threadIdx.x; w < c.n_walls; w += blockDim.x) {
      int cell = c.w_cell[w];
      T q[5];
      load_prim<T>(c, P, cell, U, V, qg, dqg, q);
      T p = q[3] - P.q_inf[3];
      int f = c.w_face[w];
      double sx, sy;
      if (c.w_family[w] == 0) {
        sx = c.fi[f];
        sy = c.fi[c.nfi() + f];
      } else {
        sx = c.fj[f];
        sy = c.fj[c.nfj() + f];
      }
      double into = c.w_into[w];
      fx = fx + p * (into * sx);
      fy = fy + p * (into * sy);
    }
    // block reduction in a fixed order
    double vals[4] = {val(fx), val(fy), 0.0, 0.0};
    if constexpr (sizeof(T) == sizeof(Dual)) {
      vals[2] = fx.d;
      vals[3] = fy.d;
    }
    for (int o = 16; o > 0; o >>= 1)
      for (int k = 0; k < 4; ++k) vals[k] += __shfl_down_sync(0xffffffffu, vals[k], o);
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      red_v[warp][0] = vals[0];
      red_v[warp][1] = vals[1];
      red_d[warp][0] = vals[2];
      red_d[warp][1] = vals[3];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double s[4] = {0, 0, 0, 0};
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
        s[0] += red_v[k][0];
        s[1] += red_v[k][1];
        s[2] += red_d[k][0];
        s[3] += red_d[k][1];
      }
      T Fx, Fy;
      if constexpr (sizeof(T) == sizeof(Dual)) {
        Fx = T{-s[0], -s[2]};
        Fy = T{-s[1], -s[3]};
      } else {
        Fx = -s[0];
        Fy = -s[1];
      }
      double u_f = P.q_inf[1], v_f = P.q_inf[2];
      double speed = hypot(u_f, v_f);
      circ_s = (Fy * u_f - Fx * v_f) / speed / (P.q_inf[0] * speed);
    }
    __syncthreads();
    circ = circ_s;
  }
  const int n0 = c.n_ghost[0], total = n0 + c.n_ghost[1];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int s = t < n0 ? 0 : 1, r = t < n0 ? t : t - n0;
    T q[5], out[5];
    const int r1 = s == 1 ? c.g_src_rec[r] : -1;
    if (r1 >= 0) {
      T q1[5];
      load_prim<T>(c, P, c.g_source[0][r1], U, V, qg, dqg, q1);
      eval_record<T>(c, P, 0, r1, q1, circ, q);
    } else {
      load_prim<T>(c, P, c.g_source[s][r], U, V, qg, dqg, q);
    }
    eval_record<T>(c, P, s, r, q, circ, out);
    const int ghost = c.g_ghost[s][r];
    for (int v = 0; v < c.nvar; ++v) {
      if constexpr (sizeof(T) == sizeof(Dual)) {
        dqg[v * N + ghost] = out[v].d;
      } else {
        qg[v * N + ghost] = out[v];
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// The tile kernel
// ------------------------------------------------------------------------------------

constexpr int HI = TILE_I + 4, HJ = TILE_J + 4;
constexpr double PR_LAM = 0.72, PR_TURB = 0.9;

template <class T, int NV> struct TileSmem {
  T q[NV][HI][HJ];
  double cx[TILE_I + 2][TILE_J + 2], cy[TILE_I + 2][TILE_J + 2];
  double Fi[NV][TILE_I + 1][TILE_J];
  double Fj[NV][TILE_I][TILE_J + 1];
  double red[TILE_THREADS / 32];
};

// The viscous face terms in two parts.  face_intermediates gathers, from the cells
// either side of a face and the four other cells of its two nodes, what the viscous flux
// depends on: the diamond gradients of u, v, T (and nu_hat), the two-cell means of u,
// v and T (and rho, p, nu_hat).  Each is linear in the cells' values of (u, v, T, ...),
// so the same function maps tangents of those values to tangents of the intermediates.
// viscous_tail is the nonlinear rest (viscosity, eddy viscosity, QCR, stresses, heat
// flux, SA diffusion).  x: [0..3] du/dx, du/dy, dv/dx, dv/dy; [4, 5] dT/dx, dT/dy;
// [6, 7] face u, v; [8] face T; SA: [9, 10] dnu_hat/dx, dnu_hat/dy; [11..13] face rho,
// p, nu_hat.  (residual.py:94-124, gradients.py:59-95, turbulence.py:78-90,129-135)
template <int VISC> struct ViscShape {
  static constexpr int NX = VISC == 2 ? 14 : 9;   // intermediates
  static constexpr int NR = VISC == 2 ? 4 : 3;    // tail outputs: fx, fy, energy[, SA diffusion]
  // the intermediates each output depends on (bit k: x[k]): fx and fy on the velocity
  // gradients, the laminar face T and (SA) the face rho, p, nu_hat through the eddy
  // viscosity; the energy on all of those and the T gradient and face velocity; the SA
  // diffusion on the nu_hat gradient and the face rho, p, nu_hat
  __host__ __device__ static constexpr unsigned depends(int r) {
    return VISC == 2 ? (r < 2 ? 0x390Fu : (r == 2 ? 0x39FFu : 0x3E00u)) : (r < 2 ? 0x10Fu : 0x1FFu);
  }
  // the place of d out[r] / d x[k] among the stored derivatives (those a dependence allows)
  __host__ __device__ static constexpr int slot(int r, int k) {
    int n = 0;
    for (int q = 0; q < r; ++q)
      for (int b = 0; b < NX; ++b) n += (depends(q) >> b) & 1u;
    for (int b = 0; b < k; ++b) n += (depends(r) >> b) & 1u;
    return n;
  }
  static constexpr int NSTORED = slot(NR - 1, NX);
};

// q(v, i, j): primitive row v of staged cell (i, j); phi(i, j, k): (u, v, T, nu_hat)[k];
// cx(i, j), cy(i, j): the cell's centre.  The face lies between A = (ai, aj) and the next
// cell along `axis`.
template <class T, int VISC, class Q, class PHI, class CX, class CY>
__device__ __forceinline__ void face_intermediates(Q q, PHI phi, CX cxv, CY cyv, int axis, int ai, int aj, T* x) {
  const int di = axis == 0 ? 1 : 0, dj = axis == 0 ? 0 : 1;
  const int bi = ai + di, bj = aj + dj;
  // the face's two nodes, each the mean of its four cells
  int n0i[4], n0j[4], n1i[4], n1j[4];
  if (axis == 0) {
    // i-face between (ai, aj) and (ai+1, aj): nodes at (i, j) and (i, j+1)
    n0i[0] = ai; n0j[0] = aj - 1; n0i[1] = ai + 1; n0j[1] = aj - 1;
    n0i[2] = ai; n0j[2] = aj;     n0i[3] = ai + 1; n0j[3] = aj;
    n1i[0] = ai; n1j[0] = aj;     n1i[1] = ai + 1; n1j[1] = aj;
    n1i[2] = ai; n1j[2] = aj + 1; n1i[3] = ai + 1; n1j[3] = aj + 1;
  } else {
    // j-face between (ai, aj) and (ai, aj+1): nodes at (i, j) and (i+1, j)
    n0i[0] = ai - 1; n0j[0] = aj; n0i[1] = ai;     n0j[1] = aj;
    n0i[2] = ai - 1; n0j[2] = aj + 1; n0i[3] = ai; n0j[3] = aj + 1;
    n1i[0] = ai;     n1j[0] = aj; n1i[1] = ai + 1; n1j[1] = aj;
    n1i[2] = ai;     n1j[2] = aj + 1; n1i[3] = ai + 1; n1j[3] = aj + 1;
  }
  double d1x = cxv(bi, bj) - cxv(ai, aj), d1y = cyv(bi, bj) - cyv(ai, aj);
  double xn0 = 0.25 * (((cxv(n0i[0], n0j[0]) + cxv(n0i[1], n0j[1])) + cxv(n0i[2], n0j[2])) + cxv(n0i[3], n0j[3]));
  double yn0 = 0.25 * (((cyv(n0i[0], n0j[0]) + cyv(n0i[1], n0j[1])) + cyv(n0i[2], n0j[2])) + cyv(n0i[3], n0j[3]));
  double xn1 = 0.25 * (((cxv(n1i[0], n1j[0]) + cxv(n1i[1], n1j[1])) + cxv(n1i[2], n1j[2])) + cxv(n1i[3], n1j[3]));
  double yn1 = 0.25 * (((cyv(n1i[0], n1j[0]) + cyv(n1i[1], n1j[1])) + cyv(n1i[2], n1j[2])) + cyv(n1i[3], n1j[3]));
  double d2x = xn1 - xn0, d2y = yn1 - yn0;
  double det = d1x * d2y - d2x * d1y;
  constexpr int NPHI = VISC == 2 ? 4 : 3;
  T gx[NPHI], gy[NPHI];
#pragma unroll
  for (int k = 0; k < NPHI; ++k) {
    T dpc = phi(bi, bj, k) - phi(ai, aj, k);
    T p0 = 0.25 * (((phi(n0i[0], n0j[0], k) + phi(n0i[1], n0j[1], k)) + phi(n0i[2], n0j[2], k)) + phi(n0i[3], n0j[3], k));
    T p1 = 0.25 * (((phi(n1i[0], n1j[0], k) + phi(n1i[1], n1j[1], k)) + phi(n1i[2], n1j[2], k)) + phi(n1i[3], n1j[3], k));
    T dpn = p1 - p0;
    gx[k] = (dpc * d2y - dpn * d1y) / det;
    gy[k] = (d1x * dpn - d2x * dpc) / det;
  }
  x[0] = gx[0];
  x[1] = gy[0];
  x[2] = gx[1];
  x[3] = gy[1];
  x[4] = gx[2];
  x[5] = gy[2];
  x[6] = 0.5 * (q(1, ai, aj) + q(1, bi, bj));
  x[7] = 0.5 * (q(2, ai, aj) + q(2, bi, bj));
  x[8] = 0.5 * (phi(ai, aj, 2) + phi(bi, bj, 2));
  if constexpr (VISC == 2) {
    x[9] = gx[3];
    x[10] = gy[3];
    x[11] = 0.5 * (q(0, ai, aj) + q(0, bi, bj));
    x[12] = 0.5 * (q(3, ai, aj) + q(3, bi, bj));
    x[13] = 0.5 * (q(4, ai, aj) + q(4, bi, bj));
  }
}

// out: fx, fy, energy (the viscous parts of rows 1-3, subtracted) and, SA, the
// diffusion of nu_hat through the face (subtracted from row 4)
template <class T, int VISC>
__device__ __forceinline__ void viscous_tail(const Physics& P, const T* x, double sx, double sy, T* out) {
  const double g = P.gamma;
  T mu = viscosity(P, x[8]);
  T k = mu / (PR_LAM * (g - 1.0));
  T g00 = x[0], g01 = x[1], g10 = x[2], g11 = x[3];
  T mut = cst<T>(0.0);
  T ex00 = cst<T>(0.0), ex01 = cst<T>(0.0), ex10 = cst<T>(0.0), ex11 = cst<T>(0.0);
  bool extra = false;
  T rho_f, nuh_f, Tface;
  if constexpr (VISC == 2) {
    rho_f = x[11];
    T p_f = x[12];
    nuh_f = x[13];
    Tface = g * p_f / rho_f;
    T mu_face = viscosity(P, Tface);
    mut = eddy_viscosity(P.sa, rho_f, nuh_f * P.mu_inf, mu_face / rho_f);
    mu = mu + mut;
    k = k + mut / (PR_TURB * (g - 1.0));
    if (P.c_cr1 != 0.0) {
      extra = true;
      T square = ((g00 * g00 + g01 * g01) + g10 * g10) + g11 * g11;
      bool pos = val(square) > 0.0;
      T nrm = pos ? dsqrt(square) : cst<T>(1.0);
      T r01 = (g01 - g10) / nrm, r10 = (g10 - g01) / nrm;
      T r00 = (g00 - g00) / nrm, r11 = (g11 - g11) / nrm;
      T div = g00 + g11;
      T t00 = mut * (g00 + g00 - (2.0 / 3.0) * div * 1.0);
      T t01 = mut * (g01 + g10 - (2.0 / 3.0) * div * 0.0);
      T t10 = mut * (g10 + g01 - (2.0 / 3.0) * div * 0.0);
      T t11 = mut * (g11 + g11 - (2.0 / 3.0) * div * 1.0);
      T p00 = r00 * t00 + r01 * t01, p01 = r00 * t10 + r01 * t11;
      T p10 = r10 * t00 + r11 * t01, p11 = r10 * t10 + r11 * t11;
      ex00 = -P.c_cr1 * (p00 + p00);
      ex01 = -P.c_cr1 * (p01 + p10);
      ex10 = -P.c_cr1 * (p10 + p01);
      ex11 = -P.c_cr1 * (p11 + p11);
    }
  }
  T div = g00 + g11;
  T ttd = (2.0 / 3.0) * div;
  T t00 = mu * (2.0 * g00 - ttd), t11 = mu * (2.0 * g11 - ttd), t01 = mu * (g01 + g10);
  T t10 = t01;
  if (extra) {
    t00 = t00 + ex00;
    t01 = t01 + ex01;
    t10 = t10 + ex10;
    t11 = t11 + ex11;
  }
  T fx = t00 * sx + t01 * sy;
  T fy = t10 * sx + t11 * sy;
  out[0] = fx;
  out[1] = fy;
  out[2] = (x[6] * fx + x[7] * fy) + k * (x[4] * sx + x[5] * sy);
  if constexpr (VISC == 2) {
    T mu_face = viscosity(P, Tface);
    T coef = diffusion_coefficient(P.sa, rho_f, nuh_f * P.mu_inf, mu_face);
    out[3] = coef * (x[9] * sx + x[10] * sy);
  }
}

// The SA source of one cell times nothing (the caller multiplies by the volume):
// y = (rho, p, nu_hat, dv/dx, du/dy, dnu_hat/dx, dnu_hat/dy), the gradients by
// Green-Gauss over face-averaged values (turbulence.py:93-103,138-151).
template <class T>
__device__ __forceinline__ T sa_cell_source(const Physics& P, const T* y, double d) {
  T omega = dabs(y[3] - y[4]);
  T rho = y[0];
  T mu = viscosity(P, P.gamma * y[1] / rho);
  T Pr, D;
  sa_source(P.sa, y[2] * P.mu_inf, mu / rho, omega, d, Pr, D);
  return rho * ((Pr - D) / P.mu_inf + P.sa.c_b2 / P.sa.sigma * P.mu_inf * (y[5] * y[5] + y[6] * y[6]));
}

// Flux through one face of the tile: inviscid (MUSCL or first-order faces), minus the
// viscous flux, plus the SA convection-diffusion flux.  The face lies between the tile
// cells A (lower) and B (upper) along `axis`; (ai, aj) is A's position in the staged
// tile (halo included).  Returns the total flux in F[0..nvar).
template <class T, int NV, bool SECOND, int VISC>
__device__ __forceinline__ void face_flux(const Physics& P, TileSmem<T, NV>& s, int axis, int ai, int aj,
                                          double sx, double sy, T* F) {
  const double g = P.gamma;
  const int di = axis == 0 ? 1 : 0, dj = axis == 0 ? 0 : 1;
  T qL[4], qR[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    T qm = s.q[v][ai][aj], qp = s.q[v][ai + di][aj + dj];
    if constexpr (SECOND) {
      T qmm = s.q[v][ai - di][aj - dj], qpp = s.q[v][ai + 2 * di][aj + 2 * dj];
      T dm = qm - qmm, d0 = qp - qm, dp = qpp - qp;
      if (P.limiter == 4) {
        double lo = 0.25 * (1.0 - P.kappa), hi = 0.25 * (1.0 + P.kappa);
        qL[v] = qm + lo * dm + hi * d0;
        qR[v] = qp - lo * dp - hi * d0;
      } else {
        qL[v] = qm + 0.5 * limit(dm, d0, P.limiter);
        qR[v] = qp - 0.5 * limit(d0, dp, P.limiter);
      }
    } else {
      qL[v] = qm;
      qR[v] = qp;
    }
  }
  T Finv[4];
  riemann(P.flux, qL, qR, sx, sy, g, Finv);
#pragma unroll
  for (int v = 0; v < 4; ++v) F[v] = Finv[v];
  if constexpr (VISC > 0) {
    auto q = [&](int v, int i, int j) -> T { return s.q[v][i][j]; };
    auto phi = [&](int i, int j, int k) -> T {
      if (k < 2) return s.q[1 + k][i][j];
      if (k == 2) return g * s.q[3][i][j] / s.q[0][i][j];
      return s.q[4][i][j];
    };
    // centres: staged with a 1-cell halo, offset 1 from the q tile's 2-cell halo
    auto cxv = [&](int i, int j) { return s.cx[i - 1][j - 1]; };
    auto cyv = [&](int i, int j) { return s.cy[i - 1][j - 1]; };
    T x[ViscShape<VISC>::NX], out[ViscShape<VISC>::NR];
    face_intermediates<T, VISC>(q, phi, cxv, cyv, axis, ai, aj, x);
    viscous_tail<T, VISC>(P, x, sx, sy, out);
    F[1] = F[1] - out[0];
    F[2] = F[2] - out[1];
    F[3] = F[3] - out[2];
    if constexpr (VISC == 2) {
      // SA face flux: upwind nu_hat on the inviscid mass flux, diffusion through the
      // face gradient (turbulence.py:129-135)
      T mass = Finv[0];
      T up = val(mass) > 0.0 ? s.q[4][ai][aj] : s.q[4][ai + di][aj + dj];
      F[4] = mass * up - out[3];
    }
  }
}

template <class T> __device__ __forceinline__ double tangent_or_value(const T& x);
template <> __device__ __forceinline__ double tangent_or_value<double>(const double& x) { return x; }
template <> __device__ __forceinline__ double tangent_or_value<Dual>(const Dual& x) { return x.d; }

// out = R(U) (second or first order); partial[block] = sum vol R0^2.  T is the staged
// scalar (double).
template <class T, int NV, bool SECOND, int VISC>
__global__ void __launch_bounds__(TILE_THREADS, TILE_MIN_BLOCKS)
    k_residual(const CaseDev* __restrict__ cases, int out_id, int with_partial, int check_active) {
  __shared__ CaseDev scase;
  if (idle_block(cases[blockIdx.z],
                 (int)blockIdx.x >= cases[blockIdx.z].tiles_x || (int)blockIdx.y >= cases[blockIdx.z].tiles_y,
                 check_active))
    return;
  const CaseDev& cd = stage_case(cases, blockIdx.z, &scase);
  if (!cd.enabled || (check_active && cd.sc->active == 0)) return;
  if ((int)blockIdx.x >= cd.tiles_x || (int)blockIdx.y >= cd.tiles_y) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ qg = cd.qg;
  double* __restrict__ out = buf(cd, out_id);
  double* __restrict__ partial = with_partial ? cd.tile_partial : nullptr;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem<T, NV>& s = *reinterpret_cast<TileSmem<T, NV>*>(smem_raw);
  const int NI = c.NI, NJ = c.NJ, N = c.ncanvas();
  const int i0 = blockIdx.y * TILE_I, j0 = blockIdx.x * TILE_J;
  const int tid = threadIdx.x;
  // 1. stage the primitive state of the tile and its halo
  for (int e = tid; e < HI * HJ; e += TILE_THREADS) {
    int li = e / HJ, lj = e % HJ;
    int i = i0 - 2 + li, j = j0 - 2 + lj;
    T q[5];
    if (i >= 0 && i < NI && j >= 0 && j < NJ) {
      load_prim_n<NV, T>(c, P, i * NJ + j, U, nullptr, qg, nullptr, q);
    } else {
      for (int v = 0; v < NV; ++v) q[v] = cst<T>(1.0);
    }
    for (int v = 0; v < NV; ++v) s.q[v][li][lj] = q[v];
  }
  if constexpr (VISC > 0) {
    const int CI = NI + 2, CJ = NJ + 2;
    for (int e = tid; e < (TILE_I + 2) * (TILE_J + 2); e += TILE_THREADS) {
      int li = e / (TILE_J + 2), lj = e % (TILE_J + 2);
      int i = i0 - 1 + li, j = j0 - 1 + lj;   // canvas cell; centres carry one more ring
      int ci = min(max(i + 1, 0), CI - 1), cj = min(max(j + 1, 0), CJ - 1);
      s.cx[li][lj] = c.centres[ci * CJ + cj];
      s.cy[li][lj] = c.centres[CI * CJ + ci * CJ + cj];
    }
  }
  __syncthreads();
  // 2. i-faces of the tile: face (i, j) lies between canvas cells (i-1, j) and (i, j)
  for (int e = tid; e < (TILE_I + 1) * TILE_J; e += TILE_THREADS) {
    int fi = e / TILE_J, fj = e % TILE_J;
    int i = i0 + fi, j = j0 + fj;
    T F[5];
    bool live = j < NJ && (interior_at(c, i - 1, j) || interior_at(c, i, j));
    if (live) {
      int f = i * NJ + j;
      face_flux<T, NV, SECOND, VISC>(P, s, 0, fi + 1, fj + 2, c.fi[f], c.fi[c.nfi() + f], F);
    }
    for (int v = 0; v < NV; ++v) s.Fi[v][fi][fj] = live ? tangent_or_value(F[v]) : 0.0;
  }
  // 3. j-faces: face (i, j) lies between (i, j-1) and (i, j)
  for (int e = tid; e < TILE_I * (TILE_J + 1); e += TILE_THREADS) {
    int fi = e / (TILE_J + 1), fj = e % (TILE_J + 1);
    int i = i0 + fi, j = j0 + fj;
    T F[5];
    bool live = i < NI && (interior_at(c, i, j - 1) || interior_at(c, i, j));
    if (live) {
      int f = i * (NJ + 1) + j;
      face_flux<T, NV, SECOND, VISC>(P, s, 1, fi + 2, fj + 1, c.fj[f], c.fj[c.nfj() + f], F);
    }
    for (int v = 0; v < NV; ++v) s.Fj[v][fi][fj] = live ? tangent_or_value(F[v]) : 0.0;
  }
  __syncthreads();
  // 4. cells: the net flux, the SA source, the output
  double acc = 0.0;
  if (tid < TILE_I * TILE_J) {
    int li = tid / TILE_J, lj = tid % TILE_J;
    int i = i0 + li, j = j0 + lj;
    if (i < NI && j < NJ) {
      int idx = i * NJ + j;
      if (c.interior[idx]) {
        double R[NV];
        for (int v = 0; v < NV; ++v)
          R[v] = (s.Fi[v][li + 1][lj] - s.Fi[v][li][lj]) + (s.Fj[v][li][lj + 1] - s.Fj[v][li][lj]);
        if constexpr (VISC == 2) {
          const int si = li + 2, sj = lj + 2;
          const double vol = c.volume[idx];
          const int fl = i * NJ + j, fh = (i + 1) * NJ + j;
          const int gl = i * (NJ + 1) + j, gh = i * (NJ + 1) + j + 1;
          double sxl = c.fi[fl], syl = c.fi[c.nfi() + fl], sxh = c.fi[fh], syh = c.fi[c.nfi() + fh];
          double txl = c.fj[gl], tyl = c.fj[c.nfj() + gl], txh = c.fj[gh], tyh = c.fj[c.nfj() + gh];
          auto avg = [&](int v, int a, int b2, int cc, int dd) { return 0.5 * (s.q[v][a][b2] + s.q[v][cc][dd]); };
          // Green-Gauss over face-averaged values: g[c][v] = (1/V) sum phi_f S_f,c
          T gg[2][3];
          for (int v = 0; v < 3; ++v) {
            int row = v < 2 ? 1 + v : 4;
            T pil = avg(row, si - 1, sj, si, sj), pih = avg(row, si, sj, si + 1, sj);
            T pjl = avg(row, si, sj - 1, si, sj), pjh = avg(row, si, sj, si, sj + 1);
            gg[0][v] = ((pih * sxh - pil * sxl) + (pjh * txh - pjl * txl)) / vol;
            gg[1][v] = ((pih * syh - pil * syl) + (pjh * tyh - pjl * tyl)) / vol;
          }
          const T y[7] = {s.q[0][si][sj], s.q[3][si][sj], s.q[4][si][sj], gg[0][1], gg[1][0], gg[0][2], gg[1][2]};
          T src = sa_cell_source(P, y, c.distance[idx]);
          R[4] = R[4] - tangent_or_value(src) * vol;
        }
        for (int v = 0; v < NV; ++v) out[v * N + idx] = R[v];
        acc = c.volume[idx] * (R[0] * R[0]);
      } else {
        for (int v = 0; v < NV; ++v) out[v * N + idx] = U[v * N + idx] - P.U_inf[v];
      }
    }
  }
  {
    if (partial != nullptr) {
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if ((tid & 31) == 0) s.red[tid >> 5] = acc;
      __syncthreads();
      if (tid == 0) {
        double t = 0.0;
        for (int k = 0; k < TILE_THREADS / 32; ++k) t += s.red[k];
        partial[blockIdx.y * cd.tiles_x + blockIdx.x] = t;
      }
    }
  }
}

// ------------------------------------------------------------------------------------
// The linearised J.v.  One linearisation serves every J.v of a Newton step, as in the
// reference, where jax.linearize evaluates the primal once and keeps what the tangent map
// needs (src/jaxrans/solvers/implicit.py:102-108).  k_linearize runs once per step at U:
// for every live face of the first-order residual it stores the face flux's derivatives
// in factored form -- the inviscid flux with respect to the primitive states either side
// (AL, AR: 4 x 4 each), the SA convection's upwind value and mass flux, the viscous
// tail with respect to its intermediates -- and for every interior cell the SA source's
// derivatives.  Each is one forward-mode (dual-number) evaluation per input direction of
// the same physics code the residual runs.  k_jv applies them to a tangent: it stages
// the tangents of (rho, u, v, p[, nu_hat], T) of the tile and its 1-cell halo, maps them
// to the face intermediates' tangents by the (linear) face_intermediates, and sums
// coefficient times tangent.  The tangent map is linear in the direction, so the result
// is the dual-number J.v up to rounding order.
// ------------------------------------------------------------------------------------

template <int VISC> struct JacShape {
  static constexpr int SA0 = 32;                      // SA convection: up, mass if A is upwind, mass if B is
  static constexpr int VBASE = VISC == 2 ? 35 : 32;   // the viscous tail's [r][k] at VBASE + r * NX + k
  static constexpr int NCOEF = VISC == 0 ? 32 : VBASE + ViscShape<VISC>::NSTORED;
};
constexpr int JCELL = 7;   // the SA source's derivatives per interior cell

int jac_coefficients(int visc) {
  return visc == 2 ? JacShape<2>::NCOEF : (visc == 1 ? JacShape<1>::NCOEF : JacShape<0>::NCOEF);
}
int jac_cell_coefficients(int visc) { return visc == 2 ? JCELL : 0; }

// Coefficients of one face at flat face index f (i-faces first, then j-faces); the face
// lies between staged cells (ai, aj) and the next along `axis` of a double tile.
template <int NV, int VISC, class TJ>
__device__ __forceinline__ void linearize_face(const Physics& P, TileSmem<double, NV>& s, int axis, int ai, int aj,
                                               double sx, double sy, TJ* __restrict__ jac, size_t stride,
                                               int f) {
  using J = JacShape<VISC>;
  const double g = P.gamma;
  const int bi = ai + (axis == 0 ? 1 : 0), bj = aj + (axis == 0 ? 0 : 1);
  double qa[4], qb[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    qa[v] = s.q[v][ai][aj];
    qb[v] = s.q[v][bi][bj];
  }
  double mass = 0.0;
#pragma unroll 1
  for (int seed = 0; seed < 8; ++seed) {
    Dual qL[4], qR[4], F[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      qL[v] = Dual{qa[v], seed == v ? 1.0 : 0.0};
      qR[v] = Dual{qb[v], seed == 4 + v ? 1.0 : 0.0};
    }
    riemann(P.flux, qL, qR, sx, sy, g, F);
    const int base = seed < 4 ? seed : 12 + seed;   // AL[r][v] at r * 4 + v, AR[r][v] at 16 + r * 4 + v
#pragma unroll
    for (int r = 0; r < 4; ++r) jac[(size_t)(base + 4 * r) * stride + f] = TJ(F[r].d);
    mass = F[0].v;
  }
  if constexpr (VISC == 2) {
    const bool a_up = mass > 0.0;
    jac[(size_t)J::SA0 * stride + f] = TJ(a_up ? s.q[4][ai][aj] : s.q[4][bi][bj]);
    jac[(size_t)(J::SA0 + 1) * stride + f] = TJ(a_up ? mass : 0.0);
    jac[(size_t)(J::SA0 + 2) * stride + f] = TJ(a_up ? 0.0 : mass);
  }
  if constexpr (VISC > 0) {
    constexpr int NX = ViscShape<VISC>::NX, NR = ViscShape<VISC>::NR;
    auto q = [&](int v, int i, int j) -> double { return s.q[v][i][j]; };
    auto phi = [&](int i, int j, int k) -> double {
      if (k < 2) return s.q[1 + k][i][j];
      if (k == 2) return g * s.q[3][i][j] / s.q[0][i][j];
      return s.q[NV == 5 ? 4 : 0][i][j];
    };
    auto cxv = [&](int i, int j) { return s.cx[i - 1][j - 1]; };
    auto cyv = [&](int i, int j) { return s.cy[i - 1][j - 1]; };
    double x[NX];
    face_intermediates<double, VISC>(q, phi, cxv, cyv, axis, ai, aj, x);
    using S = ViscShape<VISC>;
#pragma unroll 1
    for (int k = 0; k < NX; ++k) {
      Dual xd[NX], out[NR];
#pragma unroll
      for (int m = 0; m < NX; ++m) xd[m] = Dual{x[m], m == k ? 1.0 : 0.0};
      viscous_tail<Dual, VISC>(P, xd, sx, sy, out);
#pragma unroll
      for (int r = 0; r < NR; ++r)
        if ((S::depends(r) >> k) & 1u) jac[(size_t)(J::VBASE + S::slot(r, k)) * stride + f] = TJ(out[r].d);
    }
  }
}

// Three CTAs per SM (at most 168 registers, some spilled to local memory): a single
// 385 x 97 case's tiles then run in one wave instead of two; measured 262 against 368 us.
template <int NV, int VISC, class TJ>
__global__ void __launch_bounds__(TILE_THREADS, 3) k_linearize(const CaseDev* __restrict__ cases) {
  __shared__ CaseDev scase;
  if (idle_block(cases[blockIdx.z],
                 (int)blockIdx.x >= cases[blockIdx.z].tiles_x || (int)blockIdx.y >= cases[blockIdx.z].tiles_y, 0))
    return;
  const CaseDev& cd = stage_case(cases, blockIdx.z, &scase);
  if (!cd.enabled) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ qg = cd.qg;
  TJ* __restrict__ jac = static_cast<TJ*>(cd.jac);
  const size_t stride = (size_t)cd.jstride;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileSmem<double, NV>& s = *reinterpret_cast<TileSmem<double, NV>*>(smem_raw);
  const int NI = c.NI, NJ = c.NJ, N = c.ncanvas();
  const int i0 = blockIdx.y * TILE_I, j0 = blockIdx.x * TILE_J;
  const int tid = threadIdx.x;
  for (int e = tid; e < HI * HJ; e += TILE_THREADS) {
    int li = e / HJ, lj = e % HJ;
    int i = i0 - 2 + li, j = j0 - 2 + lj;
    double q[5];
    if (i >= 0 && i < NI && j >= 0 && j < NJ) {
      load_prim_n<NV, double>(c, P, i * NJ + j, U, nullptr, qg, nullptr, q);
    } else {
      for (int v = 0; v < NV; ++v) q[v] = 1.0;
    }
    for (int v = 0; v < NV; ++v) s.q[v][li][lj] = q[v];
  }
  if constexpr (VISC > 0) {
    const int CI = NI + 2, CJ = NJ + 2;
    for (int e = tid; e < (TILE_I + 2) * (TILE_J + 2); e += TILE_THREADS) {
      int li = e / (TILE_J + 2), lj = e % (TILE_J + 2);
      int i = i0 - 1 + li, j = j0 - 1 + lj;
      int ci = min(max(i + 1, 0), CI - 1), cj = min(max(j + 1, 0), CJ - 1);
      s.cx[li][lj] = c.centres[ci * CJ + cj];
      s.cy[li][lj] = c.centres[CI * CJ + ci * CJ + cj];
    }
  }
  __syncthreads();
  const int nfi = c.nfi();
  for (int e = tid; e < (TILE_I + 1) * TILE_J; e += TILE_THREADS) {
    int fi = e / TILE_J, fj = e % TILE_J;
    int i = i0 + fi, j = j0 + fj;
    if (j < NJ && (interior_at(c, i - 1, j) || interior_at(c, i, j))) {
      int f = i * NJ + j;
      linearize_face<NV, VISC, TJ>(P, s, 0, fi + 1, fj + 2, c.fi[f], c.fi[nfi + f], jac, stride, f);
    }
  }
  for (int e = tid; e < TILE_I * (TILE_J + 1); e += TILE_THREADS) {
    int fi = e / (TILE_J + 1), fj = e % (TILE_J + 1);
    int i = i0 + fi, j = j0 + fj;
    if (i < NI && (interior_at(c, i, j - 1) || interior_at(c, i, j))) {
      int f = i * (NJ + 1) + j;
      linearize_face<NV, VISC, TJ>(P, s, 1, fi + 2, fj + 1, c.fj[f], c.fj[c.nfj() + f], jac, stride, nfi + f);
    }
  }
  if constexpr (VISC == 2) {
    double* __restrict__ jcell = cd.jcell;
    if (tid < TILE_I * TILE_J) {
      int li = tid / TILE_J, lj = tid % TILE_J;
      int i = i0 + li, j = j0 + lj;
      if (i < NI && j < NJ && c.interior[i * NJ + j]) {
        const int idx = i * NJ + j, si = li + 2, sj = lj + 2;
        const double vol = c.volume[idx];
        const int fl = i * NJ + j, fh = (i + 1) * NJ + j;
        const int gl = i * (NJ + 1) + j, gh = i * (NJ + 1) + j + 1;
        double sxl = c.fi[fl], syl = c.fi[nfi + fl], sxh = c.fi[fh], syh = c.fi[nfi + fh];
        double txl = c.fj[gl], tyl = c.fj[c.nfj() + gl], txh = c.fj[gh], tyh = c.fj[c.nfj() + gh];
        auto avg = [&](int v, int a, int b2, int cc, int dd) { return 0.5 * (s.q[v][a][b2] + s.q[v][cc][dd]); };
        double gg[2][3];
        for (int v = 0; v < 3; ++v) {
          int row = v < 2 ? 1 + v : 4;
          double pil = avg(row, si - 1, sj, si, sj), pih = avg(row, si, sj, si + 1, sj);
          double pjl = avg(row, si, sj - 1, si, sj), pjh = avg(row, si, sj, si, sj + 1);
          gg[0][v] = ((pih * sxh - pil * sxl) + (pjh * txh - pjl * txl)) / vol;
          gg[1][v] = ((pih * syh - pil * syl) + (pjh * tyh - pjl * tyl)) / vol;
        }
        const double y[JCELL] = {s.q[0][si][sj], s.q[3][si][sj], s.q[NV == 5 ? 4 : 0][si][sj], gg[0][1], gg[1][0],
                                 gg[0][2], gg[1][2]};
        const double d = c.distance[idx];
#pragma unroll 1
        for (int k = 0; k < JCELL; ++k) {
          Dual yd[JCELL];
#pragma unroll
          for (int m = 0; m < JCELL; ++m) yd[m] = Dual{y[m], m == k ? 1.0 : 0.0};
          jcell[(size_t)k * N + idx] = sa_cell_source(P, yd, d).d;
        }
      }
    }
  }
}

// The tangent of every ghost record as a map of its source cell's primitive tangent:
// record t (stage-1 records first) fills its ghost from source cell src(t) -- for a
// stage-2 record whose source is a stage-1 ghost (a corner), through that record too --
// so dq_ghost = G_t dq_src, G_t = d(record)/d(q_src), one dual-number evaluation of the
// condition per source component, at the state of the linearisation.  The uniform
// far field and the wall, symmetry, inflow, outflow and copy conditions are functions of
// the source state alone; the point-vortex far field (its circulation a sum over the
// wall) is not, and its cases fill their tangent ghosts every J.v (k_ghosts) instead.
__device__ __forceinline__ int ghost_source(const Canvas& c, int t) {
  const int n0 = c.n_ghost[0];
  if (t < n0) return c.g_source[0][t];
  const int r = t - n0, r1 = c.g_src_rec[r];
  return r1 >= 0 ? c.g_source[0][r1] : c.g_source[1][r];
}

// One thread per (record, source component): column k of G_t.
template <int NV>
__global__ void k_ghost_maps(const CaseDev* __restrict__ cases) {
  const CaseDev& cd = cases[blockIdx.y];
  if (!cd.enabled || cd.P.far_field == 1) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const int n0 = c.n_ghost[0], total = n0 + c.n_ghost[1];
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total * NV; e += gridDim.x * blockDim.x) {
    const int t = e / NV, k = e % NV;
    const int s = t < n0 ? 0 : 1, r = t < n0 ? t : t - n0;
    const int r1 = s == 1 ? c.g_src_rec[r] : -1;
    double qs[5];
    load_prim<double>(c, P, ghost_source(c, t), cd.U, nullptr, cd.qg, nullptr, qs);
    double* G = cd.gmap + (size_t)t * NV * NV;
    Dual q[5], q1[5], out[5];
    for (int v = 0; v < NV; ++v) q[v] = Dual{qs[v], v == k ? 1.0 : 0.0};
    if (r1 >= 0) {
      eval_record<Dual>(c, P, 0, r1, q, cst<Dual>(0.0), q1);
      eval_record<Dual>(c, P, s, r, q1, cst<Dual>(0.0), out);
    } else {
      eval_record<Dual>(c, P, s, r, q, cst<Dual>(0.0), out);
    }
    for (int v = 0; v < NV; ++v) G[v * NV + k] = out[v].d;
  }
}

// The tangent pass: tangents of the tile and a 1-cell halo, face tangent fluxes from the
// stored coefficients, per-cell sums.
constexpr int JHI = TILE_I + 2, JHJ = TILE_J + 2;

template <int NV> struct JvSmem {
  double dq[NV + 1][JHI][JHJ];   // tangents of (rho, u, v, p[, nu_hat]) and of T = gamma p / rho
  double cx[JHI][JHJ], cy[JHI][JHJ];
  double Fi[NV][TILE_I + 1][TILE_J];
  double Fj[NV][TILE_I][TILE_J + 1];
};

template <int NV, int VISC, class TJ>
__device__ __forceinline__ void jv_face(const JvSmem<NV>& s, int axis, int ai, int aj,
                                        const TJ* __restrict__ jf, size_t stride, double* dF) {
  using J = JacShape<VISC>;
  const int bi = ai + (axis == 0 ? 1 : 0), bj = aj + (axis == 0 ? 0 : 1);
  double a[4], b[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    a[v] = s.dq[v][ai][aj];
    b[v] = s.dq[v][bi][bj];
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int v = 0; v < 4; ++v) acc += double(jf[(size_t)(4 * r + v) * stride]) * a[v];
#pragma unroll
    for (int v = 0; v < 4; ++v) acc += double(jf[(size_t)(16 + 4 * r + v) * stride]) * b[v];
    dF[r] = acc;
  }
  if constexpr (VISC == 2) {
    dF[NV - 1] = (double(jf[(size_t)J::SA0 * stride]) * dF[0] +
                  double(jf[(size_t)(J::SA0 + 1) * stride]) * s.dq[NV - 1][ai][aj]) +
                 double(jf[(size_t)(J::SA0 + 2) * stride]) * s.dq[NV - 1][bi][bj];
  }
  if constexpr (VISC > 0) {
    constexpr int NX = ViscShape<VISC>::NX, NR = ViscShape<VISC>::NR;
    auto q = [&](int v, int i, int j) -> double { return s.dq[v][i][j]; };
    auto phi = [&](int i, int j, int k) -> double {
      if (k < 2) return s.dq[1 + k][i][j];
      if (k == 2) return s.dq[NV][i][j];
      return s.dq[NV - 1][i][j];
    };
    auto cxv = [&](int i, int j) { return s.cx[i][j]; };
    auto cyv = [&](int i, int j) { return s.cy[i][j]; };
    double x[NX];
    face_intermediates<double, VISC>(q, phi, cxv, cyv, axis, ai, aj, x);
    using S = ViscShape<VISC>;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < NX; ++k)
        if ((S::depends(r) >> k) & 1u) acc += double(jf[(size_t)(J::VBASE + S::slot(r, k)) * stride]) * x[k];
      dF[r < 3 ? 1 + r : NV - 1] -= acc;
    }
  }
}

// out = vdt * v + dR1/dU . v with v = buffer `tangent_id` (vdt_id < 0: the bare J.v),
// from the case's linearisation; own_ghosts: the tile evaluates its halo's tangent
// ghosts (no tangent ghost fill needed)
template <int NV, int VISC, class TJ>
__global__ void __launch_bounds__(TILE_THREADS) k_jv(const CaseDev* __restrict__ cases, int out_id, int tangent_id,
                                                     int vdt_id, int check_active, int own_ghosts) {
  __shared__ CaseDev scase;
  if (idle_block(cases[blockIdx.z],
                 (int)blockIdx.x >= cases[blockIdx.z].tiles_x || (int)blockIdx.y >= cases[blockIdx.z].tiles_y,
                 check_active))
    return;
  const CaseDev& cd = stage_case(cases, blockIdx.z, &scase);
  if (!cd.enabled || (check_active && cd.sc->active == 0)) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ qg = cd.qg;
  const double* __restrict__ V = buf(cd, tangent_id);
  const double* __restrict__ dqg = cd.dqg;
  const double* __restrict__ vdt = vdt_id >= 0 ? buf(cd, vdt_id) : nullptr;
  const TJ* __restrict__ jac = static_cast<const TJ*>(cd.jac);
  const size_t stride = (size_t)cd.jstride;
  double* __restrict__ out = buf(cd, out_id);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  JvSmem<NV>& s = *reinterpret_cast<JvSmem<NV>*>(smem_raw);
  const int NI = c.NI, NJ = c.NJ, N = c.ncanvas();
  const int i0 = blockIdx.y * TILE_I, j0 = blockIdx.x * TILE_J;
  const int tid = threadIdx.x;
  // 1. the tangents of the tile and its halo
  for (int e = tid; e < JHI * JHJ; e += TILE_THREADS) {
    int li = e / JHJ, lj = e % JHJ;
    int i = i0 - 1 + li, j = j0 - 1 + lj;
    double t[NV + 1];
    if (i >= 0 && i < NI && j >= 0 && j < NJ) {
      const int idx = i * NJ + j;
      Dual q[5];
      const int rec = own_ghosts && P.far_field != 1 && !c.interior[idx] ? c.ghost_rec[idx] : -1;
      if (rec >= 0) {
        // the ghost's tangent from its source cell's, through the record's map; its
        // state from the ghost-filled canvas
        Dual qs[5];
        load_prim_n<NV, Dual>(c, P, ghost_source(c, rec), U, V, qg, dqg, qs);
        const double* G = cd.gmap + (size_t)rec * NV * NV;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          double d = 0.0;
#pragma unroll
          for (int k = 0; k < NV; ++k) d += G[v * NV + k] * qs[k].d;
          q[v] = Dual{qg[v * N + idx], d};
        }
      } else {
        load_prim_n<NV, Dual>(c, P, idx, U, V, qg, dqg, q);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) t[v] = q[v].d;
      t[NV] = (P.gamma * q[3] / q[0]).d;
    } else {
#pragma unroll
      for (int v = 0; v <= NV; ++v) t[v] = 0.0;
    }
#pragma unroll
    for (int v = 0; v <= NV; ++v) s.dq[v][li][lj] = t[v];
  }
  if constexpr (VISC > 0) {
    const int CI = NI + 2, CJ = NJ + 2;
    for (int e = tid; e < JHI * JHJ; e += TILE_THREADS) {
      int li = e / JHJ, lj = e % JHJ;
      int i = i0 - 1 + li, j = j0 - 1 + lj;
      int ci = min(max(i + 1, 0), CI - 1), cj = min(max(j + 1, 0), CJ - 1);
      s.cx[li][lj] = c.centres[ci * CJ + cj];
      s.cy[li][lj] = c.centres[CI * CJ + ci * CJ + cj];
    }
  }
  __syncthreads();
  const int nfi = c.nfi();
  // 2. i-faces: face (i, j) lies between canvas cells (i-1, j) and (i, j)
  for (int e = tid; e < (TILE_I + 1) * TILE_J; e += TILE_THREADS) {
    int fi = e / TILE_J, fj = e % TILE_J;
    int i = i0 + fi, j = j0 + fj;
    double dF[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) dF[v] = 0.0;
    if (j < NJ && (interior_at(c, i - 1, j) || interior_at(c, i, j)))
      jv_face<NV, VISC, TJ>(s, 0, fi, fj + 1, jac + i * NJ + j, stride, dF);
#pragma unroll
    for (int v = 0; v < NV; ++v) s.Fi[v][fi][fj] = dF[v];
  }
  // 3. j-faces: face (i, j) lies between (i, j-1) and (i, j)
  for (int e = tid; e < TILE_I * (TILE_J + 1); e += TILE_THREADS) {
    int fi = e / (TILE_J + 1), fj = e % (TILE_J + 1);
    int i = i0 + fi, j = j0 + fj;
    double dF[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) dF[v] = 0.0;
    if (i < NI && (interior_at(c, i, j - 1) || interior_at(c, i, j)))
      jv_face<NV, VISC, TJ>(s, 1, fi + 1, fj, jac + nfi + i * (NJ + 1) + j, stride, dF);
#pragma unroll
    for (int v = 0; v < NV; ++v) s.Fj[v][fi][fj] = dF[v];
  }
  __syncthreads();
  // 4. cells: the net tangent flux, the SA source's tangent, the output
  if (tid < TILE_I * TILE_J) {
    int li = tid / TILE_J, lj = tid % TILE_J;
    int i = i0 + li, j = j0 + lj;
    if (i < NI && j < NJ) {
      const int idx = i * NJ + j;
      const double w = vdt != nullptr ? vdt[idx] : 0.0;
      if (c.interior[idx]) {
        double R[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v)
          R[v] = (s.Fi[v][li + 1][lj] - s.Fi[v][li][lj]) + (s.Fj[v][li][lj + 1] - s.Fj[v][li][lj]);
        if constexpr (VISC == 2) {
          const int si = li + 1, sj = lj + 1;
          const double vol = c.volume[idx];
          const int fl = i * NJ + j, fh = (i + 1) * NJ + j;
          const int gl = i * (NJ + 1) + j, gh = i * (NJ + 1) + j + 1;
          double sxl = c.fi[fl], syl = c.fi[nfi + fl], sxh = c.fi[fh], syh = c.fi[nfi + fh];
          double txl = c.fj[gl], tyl = c.fj[c.nfj() + gl], txh = c.fj[gh], tyh = c.fj[c.nfj() + gh];
          auto avg = [&](int v, int a, int b2, int cc, int dd) { return 0.5 * (s.dq[v][a][b2] + s.dq[v][cc][dd]); };
          double gg[2][3];
#pragma unroll
          for (int v = 0; v < 3; ++v) {
            int row = v < 2 ? 1 + v : NV - 1;
            double pil = avg(row, si - 1, sj, si, sj), pih = avg(row, si, sj, si + 1, sj);
            double pjl = avg(row, si, sj - 1, si, sj), pjh = avg(row, si, sj, si, sj + 1);
            gg[0][v] = ((pih * sxh - pil * sxl) + (pjh * txh - pjl * txl)) / vol;
            gg[1][v] = ((pih * syh - pil * syl) + (pjh * tyh - pjl * tyl)) / vol;
          }
          const double y[JCELL] = {s.dq[0][si][sj], s.dq[3][si][sj], s.dq[NV - 1][si][sj], gg[0][1], gg[1][0],
                                   gg[0][2], gg[1][2]};
          const double* __restrict__ jcell = cd.jcell;
          double src = 0.0;
#pragma unroll
          for (int k = 0; k < JCELL; ++k) src += jcell[(size_t)k * N + idx] * y[k];
          R[NV - 1] = R[NV - 1] - src * vol;
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v * N + idx] = w * V[v * N + idx] + R[v];
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) out[v * N + idx] = w * V[v * N + idx] + V[v * N + idx];
      }
    }
  }
}
// ------------------------------------------------------------------------------------
// Wave speeds and the per-face terms of the preconditioner (residual.py:169-203,
// preconditioners.py:557-563): lambda from face-averaged states (a block face's
// partner from the neighbour map), the SA mass flux and diffusion per face.
// ------------------------------------------------------------------------------------

__device__ __forceinline__ void prim_raw(const Canvas& c, const Physics& P, const double* U, int idx, double* q) {
  const int N = c.ncanvas();
  double u[5];
  for (int v = 0; v < c.nvar; ++v) u[v] = U[v * N + idx];
  to_prim(u, q, c.nvar, P.gamma);
}

template <int VISC>
__global__ void k_faces(const CaseDev* __restrict__ cases) {
  __shared__ CaseDev scase;
  {
    const Canvas& g = cases[blockIdx.y].c;
    const int nf = (g.NI + 1) * g.NJ + g.NI * (g.NJ + 1);
    if (idle_block(cases[blockIdx.y], (int)(blockIdx.x * blockDim.x) >= nf, 0)) return;
  }
  const CaseDev& cd = stage_case(cases, blockIdx.y, &scase);
  if (!cd.enabled) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  double* __restrict__ lam = cd.lam;
  double* __restrict__ mflux = cd.mflux;
  double* __restrict__ dflux = cd.dflux;
  const int nfi = c.nfi(), nf = nfi + c.nfj();
  const int NI = c.NI, NJ = c.NJ;
  const double g = P.gamma;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    // every canvas face, as the reference computes them: the canvas edge copied
    // (a face on the edge averages the edge cell with itself)
    int a, b;
    double sx, sy;
    if (f < nfi) {
      int i = f / NJ, j = f % NJ;
      a = max(i - 1, 0) * NJ + j;
      b = min(i, NI - 1) * NJ + j;
      sx = c.fi[f];
      sy = c.fi[nfi + f];
    } else {
      int ff = f - nfi;
      int i = ff / (NJ + 1), j = ff % (NJ + 1);
      a = i * NJ + max(j - 1, 0);
      b = i * NJ + min(j, NJ - 1);
      sx = c.fj[ff];
      sy = c.fj[c.nfj() + ff];
    }
    int na = c.neighbours[a], nb = c.neighbours[b];
    double qa[5], qb[5], qf[5];
    prim_raw(c, P, U, na, qa);
    prim_raw(c, P, U, nb, qb);
    for (int v = 0; v < c.nvar; ++v) qf[v] = 0.5 * (qa[v] + qb[v]);
    double vn = qf[1] * sx + qf[2] * sy;
    double l = fabs(vn) + sqrt(g * qf[3] / qf[0]) * hypot(sx, sy);
    if (VISC > 0) {
      double vol = 0.5 * (c.volume[na] + c.volume[nb]);
      double mu = viscosity(P, g * qf[3] / qf[0]);
      double mu_all = mu;
      if (VISC == 2) mu_all = mu + eddy_viscosity(P.sa, qf[0], qf[4] * P.mu_inf, mu / qf[0]);
      double factor = 2.0 * g / PR_LAM;
      l = l + factor * mu_all * (sx * sx + sy * sy) / (qf[0] * vol);
      if (VISC == 2) {
        double kap = diffusion_coefficient(P.sa, qf[0], qf[4] * P.mu_inf, mu);
        mflux[f] = qf[0] * (qf[1] * sx + qf[2] * sy);
        dflux[f] = kap * (sx * sx + sy * sy) / vol;
      }
    }
    lam[f] = l;
  }
}

// Per cell: V/dt = sum lambda / CFL; the flow chains' diagonal scalar sum lambda (1/CFL + 1/2);
// the SA chains' diagonal (preconditioners.py:564-578).
template <int VISC>
__global__ void k_cells(const CaseDev* __restrict__ cases) {
  __shared__ CaseDev scase;
  {
    const Canvas& g = cases[blockIdx.y].c;
    if (idle_block(cases[blockIdx.y], (int)(blockIdx.x * blockDim.x) >= g.NI * g.NJ, 0)) return;
  }
  const CaseDev& cd = stage_case(cases, blockIdx.y, &scase);
  if (!cd.enabled) return;
  const Canvas& c = cd.c;
  const Physics& P = cd.P;
  const double* __restrict__ U = cd.U;
  const double* __restrict__ lam = cd.lam;
  const double* __restrict__ mflux = cd.mflux;
  const double* __restrict__ dflux = cd.dflux;
  const Scalars* __restrict__ sc = cd.sc;
  double* __restrict__ vdt = cd.vdt;
  double* __restrict__ dflow = cd.dflow;
  double* __restrict__ dsa = cd.dsa;
  const int NI = c.NI, NJ = c.NJ, N = c.ncanvas(), nfi = c.nfi();
  const double cfl = sc->cfl, g = P.gamma;
  // every canvas cell: V/dt enters the Krylov operator on ghost cells too (there the
  // residual is U - U_inf, its tangent the identity)
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < N; idx += gridDim.x * blockDim.x) {
    int i = idx / NJ, j = idx % NJ;
    int fl = i * NJ + j, fh = (i + 1) * NJ + j;
    int gl = nfi + i * (NJ + 1) + j, gh = gl + 1;
    double sum = ((lam[fl] + lam[fh]) + lam[gl]) + lam[gh];
    vdt[idx] = sum / cfl;
    dflow[idx] = sum * (1.0 / cfl + 0.5);
    if constexpr (VISC == 2) {
      auto out_f = [&](int f) { return fmax(mflux[f], 0.0) + dflux[f]; };
      auto in_f = [&](int f) { return fmax(-mflux[f], 0.0) + dflux[f]; };
      double q[5];
      prim_raw(c, P, U, idx, q);
      double diag = ((out_f(fh) + in_f(fl)) + out_f(gh)) + in_f(gl);
      diag = diag / q[0];
      // vorticity from face-averaged velocities (neighbour-filled raw states)
      double sxl = c.fi[fl], syl = c.fi[nfi + fl], sxh = c.fi[fh], syh = c.fi[nfi + fh];
      int jl = i * (NJ + 1) + j, jh = jl + 1;
      double txl = c.fj[jl], tyl = c.fj[c.nfj() + jl], txh = c.fj[jh], tyh = c.fj[c.nfj() + jh];
      auto favg = [&](int a, int b, int v) {
        double qa[5], qb[5];
        prim_raw(c, P, U, c.neighbours[a], qa);
        prim_raw(c, P, U, c.neighbours[b], qb);
        return 0.5 * (qa[v] + qb[v]);
      };
      int im = max(i - 1, 0) * NJ + j, ip = min(i + 1, NI - 1) * NJ + j;
      int jm = i * NJ + max(j - 1, 0), jp = i * NJ + min(j + 1, NJ - 1);
      double vol = c.volume[idx];
      double gxv[2], gyv[2];
      for (int v = 0; v < 2; ++v) {
        double pil = favg(im, idx, 1 + v), pih = favg(idx, ip, 1 + v);
        double pjl = favg(jm, idx, 1 + v), pjh = favg(idx, jp, 1 + v);
        gxv[v] = ((pih * sxh - pil * sxl) + (pjh * txh - pjl * txl)) / vol;
        gyv[v] = ((pih * syh - pil * syl) + (pjh * tyh - pjl * tyl)) / vol;
      }
      double omega = fabs(gxv[1] - gyv[0]);
      double nu = viscosity(P, g * q[3] / q[0]) / q[0];
      double d = c.distance[idx];
      double nut = q[4] * P.mu_inf;
      double st = s_tilde(P.sa, omega, nut, nu, d);
      double fw = f_w(P.sa, r_of(P.sa, nut, st, d));
      double dest = q[4] > 0.0 ? 2.0 * P.sa.c_w1 * fw * P.mu_inf * q[4] / (d * d) : 0.0;
      dsa[idx] = diag + dest * vol + sum / cfl;
    }
  }
}

// ------------------------------------------------------------------------------------
// Launch wrappers
// ------------------------------------------------------------------------------------


dim3 tile_grid(const Canvas& c) { return dim3((c.NJ + TILE_J - 1) / TILE_J, (c.NI + TILE_I - 1) / TILE_I); }

template <class T, int NV, bool SECOND, int VISC> static void configure_one() {
  cudaFuncSetAttribute(k_residual<T, NV, SECOND, VISC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(TileSmem<T, NV>));
}

template <class TJ> static void configure_lin() {
  cudaFuncSetAttribute(k_linearize<5, 2, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(TileSmem<double, 5>));
  cudaFuncSetAttribute(k_linearize<4, 1, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(TileSmem<double, 4>));
  cudaFuncSetAttribute(k_linearize<4, 0, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(TileSmem<double, 4>));
  cudaFuncSetAttribute(k_jv<5, 2, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(JvSmem<5>));
  cudaFuncSetAttribute(k_jv<4, 1, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(JvSmem<4>));
  cudaFuncSetAttribute(k_jv<4, 0, TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(JvSmem<4>));
}

// the tile kernels' dynamic shared memory limits, set once before any launch or capture
void configure_kernels() {
  static bool done = false;
  if (done) return;
  configure_one<double, 5, true, 2>();
  configure_one<double, 5, false, 2>();
  configure_one<double, 4, true, 1>();
  configure_one<double, 4, false, 1>();
  configure_one<double, 4, true, 0>();
  configure_one<double, 4, false, 0>();
  configure_lin<double>();
  configure_lin<float>();
  done = true;
}

// One launch over every case of a batch: grid z = the case, x/y = the tiles (a case
// with fewer tiles returns at once from the excess ones).
template <class T, int NV, bool SECOND, int VISC>
static void launch_tile(const CaseDev* cases, const BatchDims& d, int out_id, int with_partial, int check_active,
                        cudaStream_t st) {
  dim3 grid(d.tiles_x, d.tiles_y, d.n_cases);
  k_residual<T, NV, SECOND, VISC><<<grid, TILE_THREADS, sizeof(TileSmem<T, NV>), st>>>(cases, out_id, with_partial,
                                                                                     check_active);
}

// R(U) of every case into `out_id` (second or first order), with the norm partials
void launch_residual(const CaseDev* cases, const BatchDims& d, int visc, bool second, int out_id, cudaStream_t st) {
  if (visc == 2) {
    if (second) launch_tile<double, 5, true, 2>(cases, d, out_id, 1, 0, st);
    else launch_tile<double, 5, false, 2>(cases, d, out_id, 1, 0, st);
  } else if (visc == 1) {
    if (second) launch_tile<double, 4, true, 1>(cases, d, out_id, 1, 0, st);
    else launch_tile<double, 4, false, 1>(cases, d, out_id, 1, 0, st);
  } else {
    if (second) launch_tile<double, 4, true, 0>(cases, d, out_id, 1, 0, st);
    else launch_tile<double, 4, false, 0>(cases, d, out_id, 1, 0, st);
  }
}

// The linearisation of every case's first-order residual at its U (ghosts of U filled);
// fp32: its face coefficients stored in single precision (the mixed form)
template <class TJ>
static void linearize_t(const CaseDev* cases, const BatchDims& d, int visc, cudaStream_t st) {
  dim3 grid(d.tiles_x, d.tiles_y, d.n_cases);
  if (visc == 2) k_linearize<5, 2, TJ><<<grid, TILE_THREADS, sizeof(TileSmem<double, 5>), st>>>(cases);
  else if (visc == 1) k_linearize<4, 1, TJ><<<grid, TILE_THREADS, sizeof(TileSmem<double, 4>), st>>>(cases);
  else k_linearize<4, 0, TJ><<<grid, TILE_THREADS, sizeof(TileSmem<double, 4>), st>>>(cases);
}

void launch_linearize(const CaseDev* cases, const BatchDims& d, int visc, bool fp32, cudaStream_t st) {
  dim3 ggrid(max(1, (d.ghost_records * 5 + GHOST_THREADS - 1) / GHOST_THREADS), d.n_cases);
  if (visc == 2) k_ghost_maps<5><<<ggrid, GHOST_THREADS, 0, st>>>(cases);
  else k_ghost_maps<4><<<ggrid, GHOST_THREADS, 0, st>>>(cases);
  if (fp32) linearize_t<float>(cases, d, visc, st);
  else linearize_t<double>(cases, d, visc, st);
}

// out = vdt * v + dR1/dU . v with v = buffer `tangent_id` (vdt_id < 0: the bare J.v), from
// the linearisation launch_linearize stored (fp32: its coefficients in single precision,
// every product and sum in double); own_ghosts: the tiles map their halo's tangent ghosts
// through the linearisation's ghost maps, but in a case with the point-vortex far field,
// whose tangent ghosts a ghost fill (launch_ghosts) must provide
template <class TJ>
static void jvp_t(const CaseDev* cases, const BatchDims& d, int visc, int tangent_id, int vdt_id, int out_id,
                  int check_active, int own_ghosts, cudaStream_t st) {
  dim3 grid(d.tiles_x, d.tiles_y, d.n_cases);
  if (visc == 2)
    k_jv<5, 2, TJ><<<grid, TILE_THREADS, sizeof(JvSmem<5>), st>>>(cases, out_id, tangent_id, vdt_id, check_active,
                                                                  own_ghosts);
  else if (visc == 1)
    k_jv<4, 1, TJ><<<grid, TILE_THREADS, sizeof(JvSmem<4>), st>>>(cases, out_id, tangent_id, vdt_id, check_active,
                                                                  own_ghosts);
  else
    k_jv<4, 0, TJ><<<grid, TILE_THREADS, sizeof(JvSmem<4>), st>>>(cases, out_id, tangent_id, vdt_id, check_active,
                                                                  own_ghosts);
}

void launch_jvp(const CaseDev* cases, const BatchDims& d, int visc, bool fp32, int tangent_id, int vdt_id,
                int out_id, int check_active, int own_ghosts, cudaStream_t st) {
  if (fp32) jvp_t<float>(cases, d, visc, tangent_id, vdt_id, out_id, check_active, own_ghosts, st);
  else jvp_t<double>(cases, d, visc, tangent_id, vdt_id, out_id, check_active, own_ghosts, st);
}

// the ghosts of U (tangent_id < 0) or of the tangent in buffer `tangent_id`
void launch_ghosts(const CaseDev* cases, const BatchDims& d, int tangent_id, int check_active, cudaStream_t st) {
  dim3 grid(max(1, (d.ghost_records + GHOST_THREADS - 1) / GHOST_THREADS), d.n_cases);
  if (tangent_id >= 0) k_ghosts<Dual><<<grid, GHOST_THREADS, 0, st>>>(cases, tangent_id, check_active);
  else k_ghosts<double><<<grid, GHOST_THREADS, 0, st>>>(cases, -1, check_active);
}

void launch_faces(const CaseDev* cases, const BatchDims& d, int visc, cudaStream_t st) {
  dim3 grid(max(1, min((d.faces + 255) / 256, 148 * 8)), d.n_cases);
  if (visc == 2) k_faces<2><<<grid, 256, 0, st>>>(cases);
  else if (visc == 1) k_faces<1><<<grid, 256, 0, st>>>(cases);
  else k_faces<0><<<grid, 256, 0, st>>>(cases);
}

void launch_cells(const CaseDev* cases, const BatchDims& d, int visc, cudaStream_t st) {
  dim3 grid(max(1, min((d.cells + 255) / 256, 148 * 8)), d.n_cases);
  if (visc == 2) k_cells<2><<<grid, 256, 0, st>>>(cases);
  else if (visc == 1) k_cells<1><<<grid, 256, 0, st>>>(cases);
  else k_cells<0><<<grid, 256, 0, st>>>(cases);
}

}  // namespace jr
