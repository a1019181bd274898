// The 3D path's device types and pointwise physics: the plan of one 3D case as the
// kernels read it, and the vector-normal forms of the Euler flux, Roe average, HLLC and
// Roe fluxes and boundary conditions (src/jaxrans/numerics/riemann.py:47-203,
// boundary.py:54-130, physics/euler.py:28-94).  The scalar pieces (Dual arithmetic with
// JAX's JVP rules, limiters, the SA functions) are those of physics.cuh.
#pragma once
#include <cuda_runtime.h>

#include "physics.cuh"

namespace jr {

constexpr int NV3_MAX = 6;            // rho, rho u, rho v, rho w, E, rho nu~
constexpr int MAX_STAGES3 = 12;       // three stages per pass, at most four passes
constexpr double PR_LAMINAR = 0.72, PR_TURBULENT = 0.9;

struct Physics3 {
  double gamma;
  double mu_inf;       // M / Re (<= 0: inviscid)
  double sutherland;   // S / T_inf, < 0: constant viscosity
  double kappa;        // MUSCL kappa (limiter 4)
  double c_cr1;        // QCR2000 (0: off)
  int flux;            // 0 hllc, 1 roe
  int limiter;         // 0 none, 1 minmod, 2 van_albada, 3 van_albada_smooth, 4 kappa family
  double q_inf[NV3_MAX];   // primitive freestream
  double U_inf[NV3_MAX];   // its conservative state
  SAConst sa;
};

// One 3D case on the device: canvas (NI, NJ, NK), j... k fastest; fields variable-major.
struct Plan3Dev {
  int NI, NJ, NK, nvar;
  const uint8_t* interior;     // canvas
  const double* volume;        // canvas
  const double* faces[3];      // family a: 3 planes of (NI + (a==0)) (NJ + (a==1)) (NK + (a==2))
  const double* centres;       // 3 planes of (NI+2)(NJ+2)(NK+2): one ring beyond the canvas
  const double* distance;      // canvas (SA) or null
  int n_stages;
  int stage_off[MAX_STAGES3 + 1];   // records of stage s: [stage_off[s], stage_off[s+1])
  const int* g_ghost;
  const int* g_source;
  const int* g_kind;           // 0 copy, 1 slip wall, 2 no-slip wall, 3 symmetry, 4 far field
  const double* g_normal;      // 3 per record: the outward unit normal of the face
  const int* neighbours;       // canvas: the partner across a block face, or the cell itself
  int n_chains, chain_L;       // line chains along each block's wall-normal index
  int line_fp32;               // the line factor and apply in FP32 (the mixed form)
  int line_coupled;            // the SA row coupled to the neighbours' mean flow (6x6 blocks)
  double* face_buf;            // the residual's face fluxes: nvar x (all three families' faces)
  void* ghost_buf;             // one ghost stage's values: nvar x (the largest stage's records), Dual-sized
  const double* face_geo;      // viscous: per face (flat over the families) its diamond gradient's
                               // geometry, 10 planes: the cross products c23, c31, c12 (3 each), det
  void* node_buf;              // viscous: per node (NI+1)(NJ+1)(NK+1) the mean of its eight cells'
                               // (u, v, w, T[, nu~]), 5 planes, Dual-sized
  const int* ch_cells;         // [chain * chain_L + k], -1 past the chain's end
  const int* ch_face;          // link k -> k+1: flat index into the three face families, concatenated
  const int* ch_sign;          // +1 / -1: the link face's vector points out of / into cell k; 0 none
  int n_walls;                 // wall faces: the cell on each, the face's family and index in it,
  const int* w_cell;           // +1 where its vector points into the fluid
  const int* w_family;
  const int* w_face;
  const double* w_into;
  Physics3 P;
};

template <class T> __host__ __device__ __forceinline__ T mk(double v, double d);
template <> __host__ __device__ __forceinline__ double mk<double>(double v, double) { return v; }
template <> __host__ __device__ __forceinline__ Dual mk<Dual>(double v, double d) { return Dual{v, d}; }

__host__ __device__ __forceinline__ double tangent_or_value(double x) { return x; }
__host__ __device__ __forceinline__ double tangent_or_value(const Dual& x) { return x.d; }

template <class T> __host__ __device__ __forceinline__ T viscosity3(const Physics3& P, T Tt) {
  if (P.sutherland < 0.0) return cst<T>(P.mu_inf);
  double s = P.sutherland;
  return P.mu_inf * Tt * dsqrt(Tt) * (1.0 + s) / (Tt + s);
}

// (rho, u, v, w, p[, nu~]) from (rho, rho u, rho v, rho w, E[, rho nu~])
template <class T> __host__ __device__ __forceinline__ void to_prim3(const T* U, T* q, int nvar, double g) {
  T rho = U[0];
  T u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
  q[0] = rho;
  q[1] = u;
  q[2] = v;
  q[3] = w;
  q[4] = (g - 1.0) * (U[4] - 0.5 * rho * ((u * u + v * v) + w * w));
  if (nvar > 5) q[5] = U[5] / rho;
}

template <class T> __host__ __device__ __forceinline__ T dot3(const T* a, const double* n) {
  return (a[0] * n[0] + a[1] * n[1]) + a[2] * n[2];
}

template <class T> __host__ __device__ __forceinline__ T sq3(const T* a) { return (a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]; }

template <class T> __host__ __device__ __forceinline__ void normal_flux3(const T* q, const double* n, double g, T* F) {
  T vn = dot3(q + 1, n);
  T E = q[4] / (g - 1.0) + 0.5 * q[0] * sq3(q + 1);
  F[0] = q[0] * vn;
  for (int m = 0; m < 3; ++m) F[1 + m] = q[0] * q[1 + m] * vn + q[4] * n[m];
  F[4] = (E + q[4]) * vn;
}

template <class T>
__host__ __device__ __forceinline__ void roe_average3(const T* qL, const T* qR, double g, T& rho, T* vel, T& H, T& a) {
  T hl = g / (g - 1.0) * qL[4] / qL[0] + 0.5 * sq3(qL + 1);
  T hr = g / (g - 1.0) * qR[4] / qR[0] + 0.5 * sq3(qR + 1);
  T w = dsqrt(qR[0] / qL[0]);
  T den = 1.0 + w;
  rho = dsqrt(qL[0] * qR[0]);
  for (int m = 0; m < 3; ++m) vel[m] = (qL[1 + m] + w * qR[1 + m]) / den;
  H = (hl + w * hr) / den;
  T a2 = (g - 1.0) * (H - 0.5 * sq3(vel));
  a = dsqrt(dmax(a2, 1e-30));
}

__host__ __device__ __forceinline__ double unit3(const double* s, double* n) {
  const double len = sqrt((s[0] * s[0] + s[1] * s[1]) + s[2] * s[2]);
  const double safe = fmax(len, 1e-300);
  for (int m = 0; m < 3; ++m) n[m] = s[m] / safe;
  return len;
}

template <class T> __host__ __device__ __forceinline__ void hllc3(const T* qL, const T* qR, const double* s, double g, T* F) {
  double n[3];
  const double len = unit3(s, n);
  T vnl = dot3(qL + 1, n), vnr = dot3(qR + 1, n);
  T al = dsqrt(g * qL[4] / qL[0]), ar = dsqrt(g * qR[4] / qR[0]);
  T rho_ro, v_ro[3], H_ro, a_ro;
  roe_average3(qL, qR, g, rho_ro, v_ro, H_ro, a_ro);
  T vn_ro = dot3(v_ro, n);
  T sl = dmin(vnl - al, vn_ro - a_ro);
  T sr = dmax(vnr + ar, vn_ro + a_ro);
  T ml = qL[0] * (sl - vnl);
  T mr = qR[0] * (sr - vnr);
  T sm = (qR[4] - qL[4] + ml * vnl - mr * vnr) / dmin(ml - mr, -1e-300);
  T f[5];
  if (val(sl) >= 0.0) {
    normal_flux3(qL, n, g, f);
  } else if (!(val(sm) >= 0.0) && !(val(sr) >= 0.0)) {
    normal_flux3(qR, n, g, f);
  } else {
    const bool left = val(sm) >= 0.0;
    T q[5];   // the star side's state, selected by value (a selected pointer would put both in local memory)
#pragma unroll
    for (int k = 0; k < 5; ++k) q[k] = left ? qL[k] : qR[k];
    T sk = left ? sl : sr;
    T vn = left ? vnl : vnr;
    T wide = left ? dmin(sl - sm, -1e-300) : dmax(sr - sm, 1e-300);
    normal_flux3(q, n, g, f);
    T E = q[4] / (g - 1.0) + 0.5 * q[0] * sq3(q + 1);
    T Uk[5] = {q[0], q[0] * q[1], q[0] * q[2], q[0] * q[3], E};
    T pstar = q[4] + q[0] * (vn - sk) * (vn - sm);
    T rstar = q[0] * (sk - vn) / wide;
    T estar = ((sk - vn) * E - q[4] * vn + pstar * sm) / wide;
    T us[5] = {rstar, rstar * (q[1] + (sm - vn) * n[0]), rstar * (q[2] + (sm - vn) * n[1]),
               rstar * (q[3] + (sm - vn) * n[2]), estar};
    for (int k = 0; k < 5; ++k) f[k] = f[k] + sk * (us[k] - Uk[k]);
  }
  for (int k = 0; k < 5; ++k) F[k] = len * f[k];
}

template <class T> __host__ __device__ __forceinline__ void roe3(const T* qL, const T* qR, const double* s, double g, T* F) {
  double n[3];
  const double len = unit3(s, n);
  T rho, vel[3], H, a;
  roe_average3(qL, qR, g, rho, vel, H, a);
  T vn = dot3(vel, n);
  T drho = qR[0] - qL[0], dp = qR[4] - qL[4];
  T dv[3] = {qR[1] - qL[1], qR[2] - qL[2], qR[3] - qL[3]};
  T dvn = dot3(dv, n);
  T dvt[3];
  for (int m = 0; m < 3; ++m) dvt[m] = dv[m] - dvn * n[m];
  T a2 = a * a;
  T am = (dp - rho * a * dvn) / (2.0 * a2);
  T ae = drho - dp / a2;
  T ap = (dp + rho * a * dvn) / (2.0 * a2);
  T lm = dabs(vn - a), l0 = dabs(vn), lp = dabs(vn + a);
  T kin = 0.5 * sq3(vel);
  T vdt = (vel[0] * dvt[0] + vel[1] * dvt[1]) + vel[2] * dvt[2];
  T rm[5] = {cst<T>(1.0), vel[0] - a * n[0], vel[1] - a * n[1], vel[2] - a * n[2], H - a * vn};
  T re_[5] = {cst<T>(1.0), vel[0], vel[1], vel[2], kin};
  T sh[5] = {cst<T>(0.0), rho * dvt[0], rho * dvt[1], rho * dvt[2], rho * vdt};
  T rp[5] = {cst<T>(1.0), vel[0] + a * n[0], vel[1] + a * n[1], vel[2] + a * n[2], H + a * vn};
  T fl[5], fr[5];
  normal_flux3(qL, n, g, fl);
  normal_flux3(qR, n, g, fr);
  for (int k = 0; k < 5; ++k) {
    T diss = lm * am * rm[k] + l0 * ae * re_[k] + l0 * sh[k] + lp * ap * rp[k];
    F[k] = len * (0.5 * (fl[k] + fr[k]) - 0.5 * diss);
  }
}

template <class T> __host__ __device__ __forceinline__ void riemann3(int kind, const T* qL, const T* qR, const double* s,
                                                             double g, T* F) {
  if (kind == 0)
    hllc3(qL, qR, s, g, F);
  else
    roe3(qL, qR, s, g, F);
}

// a ghost's primitive state from its source cell's (src/jaxrans/numerics/boundary.py:54-130)
template <class T>
__host__ __device__ __forceinline__ void condition3(int kind, const T* q, double nx, double ny, double nz, const Physics3& P,
                                           int nvar, T* o) {
  const double n[3] = {nx, ny, nz};
  for (int v = 0; v < nvar; ++v) o[v] = q[v];
  if (kind == 1 || kind == 3) {   // slip wall / symmetry: the velocity mirrored
    T vn = dot3(q + 1, n);
    for (int m = 0; m < 3; ++m) o[1 + m] = q[1 + m] - 2.0 * vn * n[m];
    if (kind == 1 && nvar > 5) o[5] = -q[5];
  } else if (kind == 2) {         // no-slip wall: velocity and scalars reversed
    for (int m = 0; m < 3; ++m) o[1 + m] = -q[1 + m];
    if (nvar > 5) o[5] = -q[5];
  } else if (kind == 4) {         // far field: Riemann invariants against the freestream
    const double g = P.gamma;
    const double* qf = P.q_inf;
    T ai = dsqrt(g * q[4] / q[0]);
    const double af = sqrt(g * qf[4] / qf[0]);
    const double two = 2.0 / (g - 1.0);
    T vni = dot3(q + 1, n);
    const double vnf = (qf[1] * n[0] + qf[2] * n[1]) + qf[3] * n[2];
    T rp = vni + two * ai;
    T rm = cst<T>(vnf - two * af);
    T vnb = 0.5 * (rp + rm);
    T ab = 0.25 * (g - 1.0) * (rp - rm);
    const bool outflow = val(vnb) > 0.0;
    T sb = outflow ? q[4] / dpow(q[0], g) : cst<T>(qf[4] / pow(qf[0], g));
    T rb = dpow(ab * ab / (g * sb), 1.0 / (g - 1.0));
    o[0] = rb;
    for (int m = 0; m < 3; ++m) {
      T tang = outflow ? q[1 + m] - vni * n[m] : cst<T>(qf[1 + m] - vnf * n[m]);
      o[1 + m] = vnb * n[m] + tang;
    }
    o[4] = rb * ab * ab / g;
    if (nvar > 5) o[5] = outflow ? q[5] : cst<T>(qf[5]);
  }
}

void launch_residual3(const Plan3Dev& p, const double* U, double* R, void* A, bool first_order, cudaStream_t st);
// the exact tangent of the first-order residual at U along v (A: a Dual-sized canvas)
void launch_jvp3(const Plan3Dev& p, const double* U, const double* v, double* Jv, void* A, cudaStream_t st);
void launch_wave_speeds3(const Plan3Dev& p, const double* U, double* lam, cudaStream_t st);
void launch_wall_loads3(const Plan3Dev& p, const double* U, double* loads, void* A, cudaStream_t st);
// the viscous faces' diamond-gradient geometry into geo (10 x all faces), once per plan
void launch_face_geometry3(const Plan3Dev& p, double* geo, cudaStream_t st);
void launch_line_factor3(const Plan3Dev& p, const double* U, double cfl, void* F, cudaStream_t st);
void launch_line_apply3(const Plan3Dev& p, const void* F, const double* r, double* z, cudaStream_t st);
void launch_precondition3(const Plan3Dev& p, const double* U, double cfl, const double* r, double* z, void* F,
                          cudaStream_t st);
// words per chain element of the line factor (linesolve3d.cuh): three 5x5 blocks, three
// SA scalars and the SA row's two coupling rows to the mean flow (the coupled form)
constexpr int FACTOR3 = 88;

// Kernels the 3D path has launched since the library was loaded (counted on the host at
// each launch site; the benchmark's launch figure).
long long& launches3();
inline void counted3(int n = 1) { launches3() += n; }

void launch_wall_distance3(const double* points, long long n_points, const double* quads, int n_faces, double* spheres,
                           double* out, cudaStream_t st);

}  // namespace jr
