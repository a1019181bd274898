// Pointwise physics of the 2D Euler / Navier-Stokes / SA-RANS residual, templated on
// the scalar: `double` for R(U), `Dual` (value + tangent) for the exact J.v of the
// first-order residual.  The formulas follow the reference's own
// (src/jaxrans/numerics/riemann.py, limiters.py, boundary.py, physics/*.py), with the
// same branch choices; non-smooth primitives carry JAX's JVP rules so that the
// tangent equals what jax.linearize gives on the same state:
//   abs:      select(x >= 0, +t, -t)
//   min/max:  the selected operand's tangent, the mean of both at an exact tie
//   where:    the selected branch's tangent; comparisons read the value only.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace jr {

struct Dual {
  double v, d;
};

__host__ __device__ __forceinline__ double val(double x) { return x; }
__host__ __device__ __forceinline__ double val(const Dual& x) { return x.v; }

template <class T> __host__ __device__ __forceinline__ T cst(double x);
template <> __host__ __device__ __forceinline__ double cst<double>(double x) { return x; }
template <> __host__ __device__ __forceinline__ Dual cst<Dual>(double x) { return Dual{x, 0.0}; }

__host__ __device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__host__ __device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__host__ __device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__host__ __device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__host__ __device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__host__ __device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__host__ __device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__host__ __device__ __forceinline__ Dual operator/(double a, Dual b) {
  double q = a / b.v;
  return {q, -q * b.d / b.v};
}

__host__ __device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__host__ __device__ __forceinline__ Dual dsqrt(Dual x) {
  double s = sqrt(x.v);
  return {s, x.d * (0.5 / s)};
}
// x**c for a constant exponent (pow's JVP: c x^(c-1) t)
__host__ __device__ __forceinline__ double dpow(double x, double c) { return pow(x, c); }
__host__ __device__ __forceinline__ Dual dpow(Dual x, double c) {
  return {pow(x.v, c), x.d * (c * pow(x.v, c - 1.0))};
}
__host__ __device__ __forceinline__ double dabs(double x) { return x >= 0.0 ? x : -x; }
__host__ __device__ __forceinline__ Dual dabs(Dual x) { return x.v >= 0.0 ? x : -x; }
__host__ __device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : (b > a ? b : a); }
__host__ __device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : (b < a ? b : a); }
__host__ __device__ __forceinline__ Dual dmax(Dual a, Dual b) {
  return a.v > b.v ? a : (b.v > a.v ? b : Dual{a.v, 0.5 * (a.d + b.d)});
}
__host__ __device__ __forceinline__ Dual dmin(Dual a, Dual b) {
  return a.v < b.v ? a : (b.v < a.v ? b : Dual{a.v, 0.5 * (a.d + b.d)});
}
__host__ __device__ __forceinline__ Dual dmax(Dual a, double b) { return dmax(a, Dual{b, 0.0}); }
__host__ __device__ __forceinline__ Dual dmin(Dual a, double b) { return dmin(a, Dual{b, 0.0}); }
template <class T> __host__ __device__ __forceinline__ T sel(bool c, const T& a, const T& b) { return c ? a : b; }
__host__ __device__ __forceinline__ Dual sel(bool c, const Dual& a, double b) { return c ? a : Dual{b, 0.0}; }
__host__ __device__ __forceinline__ Dual sel(bool c, double a, const Dual& b) { return c ? Dual{a, 0.0} : b; }
__host__ __device__ __forceinline__ double sel(bool c, double a, double b) { return c ? a : b; }
template <class T> __host__ __device__ __forceinline__ T ipow3(T x) { return x * (x * x); }
template <class T> __host__ __device__ __forceinline__ T ipow6(T x) {
  T x2 = x * x;
  return x2 * (x2 * x2);
}

// ---- model constants (SA-noft2 / SA-neg: src/jaxrans/physics/spalart_allmaras.py:66-89)
struct SAConst {
  double c_b1, sigma, c_b2, kappa, c_w2, c_w3, c_v1, c_2, c_3, c_n1, r_max;
  double c_w1, c_v1_3, c_w3_6, c_2_2;  // derived, evaluated on the host
};

// SA-noft2 constants (src/jaxrans/physics/spalart_allmaras.py:66-89) and the derived ones
inline void sa_constants(SAConst& s) {
  s.c_b1 = 0.1355;
  s.sigma = 2.0 / 3.0;
  s.c_b2 = 0.622;
  s.kappa = 0.41;
  s.c_w2 = 0.3;
  s.c_w3 = 2.0;
  s.c_v1 = 7.1;
  s.c_2 = 0.7;
  s.c_3 = 0.9;
  s.c_n1 = 16.0;
  s.r_max = 10.0;
  s.c_w1 = s.c_b1 / (s.kappa * s.kappa) + (1.0 + s.c_b2) / s.sigma;
  s.c_v1_3 = s.c_v1 * s.c_v1 * s.c_v1;
  s.c_w3_6 = s.c_w3 * s.c_w3 * s.c_w3 * s.c_w3 * s.c_w3 * s.c_w3;
  s.c_2_2 = s.c_2 * s.c_2;
}

// Everything a residual evaluation needs that is not per cell.
struct Physics {
  double gamma;
  double mu_inf;       // M / Re (0: inviscid)
  double sutherland;   // S / T_inf, < 0: constant viscosity
  double c_cr1;        // QCR2000 (0: off)
  double kappa;        // MUSCL kappa (limiter 4)
  int flux;            // 0 hllc, 1 roe
  int limiter;         // 0 none, 1 minmod, 2 van_albada, 3 van_albada_smooth, 4 kappa family
  int nvar;            // 4 or 5
  int far_field;       // 0 characteristic, 1 characteristic + point vortex
  double q_inf[5];     // primitive freestream
  double U_inf[5];     // its conservative state (the canvas initial value)
  double quarter_chord[2];
  SAConst sa;
};

template <class T> __host__ __device__ __forceinline__ T viscosity(const Physics& P, T Tt) {
  if (P.sutherland < 0.0) return cst<T>(P.mu_inf);
  double s = P.sutherland;
  return P.mu_inf * Tt * dsqrt(Tt) * (1.0 + s) / (Tt + s);
}

// primitive (rho, u, v, p[, nu_hat]) from conservative
template <class T> __host__ __device__ __forceinline__ void to_prim(const T* U, T* q, int nvar, double g) {
  T rho = U[0];
  T u = U[1] / rho, v = U[2] / rho;
  q[0] = rho;
  q[1] = u;
  q[2] = v;
  q[3] = (g - 1.0) * (U[3] - 0.5 * rho * (u * u + v * v));
  if (nvar > 4) q[4] = U[4] / rho;
}

// ---- limiters on differences (src/jaxrans/numerics/limiters.py:61-116)
template <class T> __host__ __device__ __forceinline__ T limit(const T& a, const T& b, int kind) {
  if (kind == 1) {  // minmod
    double ab = val(a * b);
    if (!(ab > 0.0)) return cst<T>(0.0);
    double sg = val(a) > 0.0 ? 1.0 : (val(a) < 0.0 ? -1.0 : 0.0);
    return sg * dmin(dabs(a), dabs(b));
  }
  if (kind == 2) {  // van Albada, cut at extrema
    T ab = a * b;
    if (!(val(ab) > 0.0)) return cst<T>(0.0);
    return ab * (a + b) / (a * a + b * b);
  }
  if (kind == 3) {  // van Albada, smooth
    const double e = 1e-12;
    return ((b * b + e) * a + (a * a + e) * b) / (a * a + b * b + 2.0 * e);
  }
  return 0.5 * (a + b);  // none
}

// ---- Euler flux and Riemann solvers (src/jaxrans/numerics/riemann.py:47-198)
template <class T>
__host__ __device__ __forceinline__ void normal_flux(const T* q, double nx, double ny, double g, T* F) {
  T vn = q[1] * nx + q[2] * ny;
  T E = q[3] / (g - 1.0) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
  F[0] = q[0] * vn;
  F[1] = q[0] * q[1] * vn + q[3] * nx;
  F[2] = q[0] * q[2] * vn + q[3] * ny;
  F[3] = (E + q[3]) * vn;
}

template <class T>
__host__ __device__ __forceinline__ void roe_average(const T* qL, const T* qR, double g, T& rho, T& u, T& v, T& H, T& a) {
  T hl = g / (g - 1.0) * qL[3] / qL[0] + 0.5 * (qL[1] * qL[1] + qL[2] * qL[2]);
  T hr = g / (g - 1.0) * qR[3] / qR[0] + 0.5 * (qR[1] * qR[1] + qR[2] * qR[2]);
  T w = dsqrt(qR[0] / qL[0]);
  T den = 1.0 + w;
  rho = dsqrt(qL[0] * qR[0]);
  u = (qL[1] + w * qR[1]) / den;
  v = (qL[2] + w * qR[2]) / den;
  H = (hl + w * hr) / den;
  T a2 = (g - 1.0) * (H - 0.5 * (u * u + v * v));
  a = dsqrt(dmax(a2, 1e-30));
}

template <class T>
__host__ __device__ __forceinline__ void hllc_flux(const T* qL, const T* qR, double sx, double sy, double g, T* F) {
  double len = hypot(sx, sy);
  double safe = fmax(len, 1e-300);
  double nx = sx / safe, ny = sy / safe;
  T vnl = qL[1] * nx + qL[2] * ny, vnr = qR[1] * nx + qR[2] * ny;
  T al = dsqrt(g * qL[3] / qL[0]), ar = dsqrt(g * qR[3] / qR[0]);
  T rho_ro, u_ro, v_ro, H_ro, a_ro;
  roe_average(qL, qR, g, rho_ro, u_ro, v_ro, H_ro, a_ro);
  T vn_ro = u_ro * nx + v_ro * ny;
  T sl = dmin(vnl - al, vn_ro - a_ro);
  T sr = dmax(vnr + ar, vn_ro + a_ro);
  T ml = qL[0] * (sl - vnl);
  T mr = qR[0] * (sr - vnr);
  T sm = (qR[3] - qL[3] + ml * vnl - mr * vnr) / dmin(ml - mr, -1e-300);
  T f[4];
  // the region the face sits in, tested in the reference's order: S_L, S_M, S_R
  if (val(sl) >= 0.0) {
    normal_flux(qL, nx, ny, g, f);
  } else if (!(val(sm) >= 0.0) && !(val(sr) >= 0.0)) {
    normal_flux(qR, nx, ny, g, f);
  } else {
    // star flux of one side of the contact: F_K + S_K (U*_K - U_K)
    const bool left = val(sm) >= 0.0;
    T q[4];   // the star side's state, selected by value (a selected pointer would put both in local memory)
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = left ? qL[k] : qR[k];
    T sk = left ? sl : sr;
    T vn = left ? vnl : vnr;
    T wide = left ? dmin(sl - sm, -1e-300) : dmax(sr - sm, 1e-300);
    normal_flux(q, nx, ny, g, f);
    T E = q[3] / (g - 1.0) + 0.5 * q[0] * (q[1] * q[1] + q[2] * q[2]);
    T Uk[4] = {q[0], q[0] * q[1], q[0] * q[2], E};
    T pstar = q[3] + q[0] * (vn - sk) * (vn - sm);
    T rstar = q[0] * (sk - vn) / wide;
    T estar = ((sk - vn) * E - q[3] * vn + pstar * sm) / wide;
    T us[4] = {rstar, rstar * (q[1] + (sm - vn) * nx), rstar * (q[2] + (sm - vn) * ny), estar};
#pragma unroll
    for (int k = 0; k < 4; ++k) f[k] = f[k] + sk * (us[k] - Uk[k]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) F[k] = len * f[k];
}

template <class T>
__host__ __device__ __forceinline__ void roe_flux(const T* qL, const T* qR, double sx, double sy, double g, T* F) {
  double len = hypot(sx, sy);
  double safe = fmax(len, 1e-300);
  double nx = sx / safe, ny = sy / safe;
  T rho, u, v, H, a;
  roe_average(qL, qR, g, rho, u, v, H, a);
  T vn = u * nx + v * ny;
  T drho = qR[0] - qL[0], dp = qR[3] - qL[3];
  T du = qR[1] - qL[1], dv = qR[2] - qL[2];
  T dvn = du * nx + dv * ny;
  T dut = du - dvn * nx, dvt = dv - dvn * ny;
  T a2 = a * a;
  T am = (dp - rho * a * dvn) / (2.0 * a2);
  T ae = drho - dp / a2;
  T ap = (dp + rho * a * dvn) / (2.0 * a2);
  T lm = dabs(vn - a), l0 = dabs(vn), lp = dabs(vn + a);
  T kin = 0.5 * (u * u + v * v);
  T rm[4] = {cst<T>(1.0), u - a * nx, v - a * ny, H - a * vn};
  T re_[4] = {cst<T>(1.0), u, v, kin};
  T sh[4] = {cst<T>(0.0), rho * dut, rho * dvt, rho * (u * dut + v * dvt)};
  T rp[4] = {cst<T>(1.0), u + a * nx, v + a * ny, H + a * vn};
  T fl[4], fr[4];
  normal_flux(qL, nx, ny, g, fl);
  normal_flux(qR, nx, ny, g, fr);
  T cm = lm * am, ce = l0 * ae, cp = lp * ap;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    T diss = cm * rm[k] + ce * re_[k] + l0 * sh[k] + cp * rp[k];
    F[k] = len * (0.5 * (fl[k] + fr[k]) - 0.5 * diss);
  }
}

template <class T>
__host__ __device__ __forceinline__ void riemann(int kind, const T* qL, const T* qR, double sx, double sy, double g, T* F) {
  if (kind == 0)
    hllc_flux(qL, qR, sx, sy, g, F);
  else
    roe_flux(qL, qR, sx, sy, g, F);
}

// ---- Spalart-Allmaras pieces (src/jaxrans/physics/spalart_allmaras.py:119-195)
template <class T> __host__ __device__ __forceinline__ T eddy_viscosity(const SAConst& c, T rho, T nut, T nu) {
  if (!(val(nut) > 0.0)) return cst<T>(0.0);
  T chi = nut / nu;
  T chi3 = ipow3(chi);
  return rho * nut * (chi3 / (chi3 + c.c_v1_3));
}

template <class T> __host__ __device__ __forceinline__ T f_n(const SAConst& c, T nut, T nu) {
  if (val(nut) >= 0.0) return cst<T>(1.0);
  T chi3 = ipow3(nut / nu);
  return (c.c_n1 + chi3) / (c.c_n1 - chi3);
}

template <class T> __host__ __device__ __forceinline__ T diffusion_coefficient(const SAConst& c, T rho, T nut, T mu) {
  T nu = mu / rho;
  return (mu + rho * nut * f_n(c, nut, nu)) / c.sigma;
}

template <class T> __host__ __device__ __forceinline__ T s_tilde(const SAConst& c, T omega, T nut, T nu, double d) {
  T chi = nut / nu;
  T chi3 = ipow3(chi);
  T fv1 = chi3 / (chi3 + c.c_v1_3);
  T fv2 = 1.0 - chi / (1.0 + chi * fv1);
  double kd = c.kappa * d;
  T sbar = nut * fv2 / (kd * kd);
  bool ordinary = val(sbar) >= val(-c.c_2 * omega);
  if (ordinary) return omega + sbar;
  T den = (c.c_3 - 2.0 * c.c_2) * omega - sbar;
  return omega + omega * (c.c_2_2 * omega + c.c_3 * sbar) / den;
}

template <class T> __host__ __device__ __forceinline__ T f_w(const SAConst& c, T r) {
  T gg = r + c.c_w2 * (ipow6(r) - r);
  return gg * dpow((1.0 + c.c_w3_6) / (ipow6(gg) + c.c_w3_6), 1.0 / 6.0);
}

template <class T> __host__ __device__ __forceinline__ T r_of(const SAConst& c, T nut, T st, double d) {
  double kd = c.kappa * d;
  T den = st * (kd * kd);
  if (!(val(den) > 0.0)) return cst<T>(c.r_max);
  return dmin(nut / den, c.r_max);
}

// (production, destruction) per unit mass (src/jaxrans/physics/spalart_allmaras.py:165-177)
template <class T>
__host__ __device__ __forceinline__ void sa_source(const SAConst& c, T nut, T nu, T omega, double d, T& P, T& D) {
  bool pos = val(nut) >= 0.0;
  T st = s_tilde(c, omega, pos ? nut : cst<T>(0.0), nu, d);
  T w = nut / d;
  T wall = w * w;
  P = (pos ? c.c_b1 * st : c.c_b1 * omega) * nut;
  D = (pos ? c.c_w1 * f_w(c, r_of(c, nut, st, d)) : cst<T>(-c.c_w1)) * wall;
}

// ---- boundary conditions on primitives (src/jaxrans/numerics/boundary.py:67-158)
template <class T>
__host__ __device__ __forceinline__ void characteristic(const T* e, double nx, double ny, const T* qf, int nvar, double g,
                                               T* out) {
  T ai = dsqrt(g * e[3] / e[0]);
  T af = dsqrt(g * qf[3] / qf[0]);
  double two = 2.0 / (g - 1.0);
  T vni = e[1] * nx + e[2] * ny;
  T vnf = qf[1] * nx + qf[2] * ny;
  T rp = vni + two * ai;
  T rm = vnf - two * af;
  T vnb = 0.5 * (rp + rm);
  T ab = 0.25 * (g - 1.0) * (rp - rm);
  bool outflow = val(vnb) > 0.0;
  T sb = outflow ? e[3] / dpow(e[0], g) : qf[3] / dpow(qf[0], g);
  T tu = outflow ? e[1] - vni * nx : qf[1] - vnf * nx;
  T tv = outflow ? e[2] - vni * ny : qf[2] - vnf * ny;
  T rb = dpow(ab * ab / (g * sb), 1.0 / (g - 1.0));
  out[0] = rb;
  out[1] = vnb * nx + tu;
  out[2] = vnb * ny + tv;
  out[3] = rb * ab * ab / g;
  if (nvar > 4) out[4] = outflow ? e[4] : qf[4];
}

}  // namespace jr
