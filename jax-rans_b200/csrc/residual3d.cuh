// The per-cell and per-record bodies of the 3D residual and J.v (residual3d.cu launches
// them, one thread each): host-and-device code, so the same arithmetic can also run on
// the host to check the kernels' indexing without a GPU.
#pragma once
#include <cstdint>

#include "device3d.cuh"

namespace jr {

// the primitive state of canvas cell c from conservative U (and the tangent dU for Dual)
template <class T>
__host__ __device__ __forceinline__ void prim_cell(const Plan3Dev& p, const double* U, const double* dU, T* Q, int c) {
  const int n = p.NI * p.NJ * p.NK;
  T u[NV3_MAX], q[NV3_MAX];
  for (int v = 0; v < p.nvar; ++v) u[v] = mk<T>(U[(size_t)v * n + c], dU ? dU[(size_t)v * n + c] : 0.0);
  to_prim3(u, q, p.nvar, p.P.gamma);
  for (int v = 0; v < p.nvar; ++v) Q[(size_t)v * n + c] = q[v];
}

// the same with the plan's variable count NV (== p.nvar) fixed at compile time
template <int NV, class T>
__host__ __device__ __forceinline__ void prim_cell_n(const Plan3Dev& p, const double* U, const double* dU, T* Q,
                                                     int c) {
  const int n = p.NI * p.NJ * p.NK;
  T u[NV3_MAX], q[NV3_MAX];
#pragma unroll
  for (int v = 0; v < NV; ++v) u[v] = mk<T>(U[(size_t)v * n + c], dU ? dU[(size_t)v * n + c] : 0.0);
  to_prim3(u, q, NV, p.P.gamma);
#pragma unroll
  for (int v = 0; v < NV; ++v) Q[(size_t)v * n + c] = q[v];
}

// ghost record r of a stage: out[ghost] = condition(in[source]) (or a copy across a cut)
template <class T>
__host__ __device__ __forceinline__ void ghost_record(const Plan3Dev& p, const T* in, T* out, int r) {
  const int n = p.NI * p.NJ * p.NK;
  const int ghost = p.g_ghost[r], src = p.g_source[r], kind = p.g_kind[r];
  if (ghost < 0 || ghost >= n || src < 0 || src >= n) return;   // validated on the host
  T q[NV3_MAX], o[NV3_MAX];
  for (int v = 0; v < p.nvar; ++v) q[v] = in[(size_t)v * n + src];
  condition3(kind, q, p.g_normal[3 * r], p.g_normal[3 * r + 1], p.g_normal[3 * r + 2], p.P, p.nvar, o);
  for (int v = 0; v < p.nvar; ++v) out[(size_t)v * n + ghost] = o[v];
}

// The same stage in place, in two passes: every record's value from the canvas as it was
// before the stage (into buf, slot r - r0 of count), then every value to its ghost.  A
// stage writes each ghost once, so the two passes give the double-buffered stage's canvas
// without copying the canvas.
template <class T>
__host__ __device__ __forceinline__ void ghost_value(const Plan3Dev& p, const T* Q, int r, int r0, int count, T* buf) {
  const int n = p.NI * p.NJ * p.NK;
  const int ghost = p.g_ghost[r], src = p.g_source[r], kind = p.g_kind[r];
  if (ghost < 0 || ghost >= n || src < 0 || src >= n) return;   // validated on the host
  T q[NV3_MAX], o[NV3_MAX];
  for (int v = 0; v < p.nvar; ++v) q[v] = Q[(size_t)v * n + src];
  condition3(kind, q, p.g_normal[3 * r], p.g_normal[3 * r + 1], p.g_normal[3 * r + 2], p.P, p.nvar, o);
  for (int v = 0; v < p.nvar; ++v) buf[(size_t)v * count + (r - r0)] = o[v];
}

template <class T>
__host__ __device__ __forceinline__ void ghost_store(const Plan3Dev& p, const T* buf, int r, int r0, int count, T* Q) {
  const int n = p.NI * p.NJ * p.NK;
  const int ghost = p.g_ghost[r], src = p.g_source[r];
  if (ghost < 0 || ghost >= n || src < 0 || src >= n) return;
  for (int v = 0; v < p.nvar; ++v) Q[(size_t)v * n + ghost] = buf[(size_t)v * count + (r - r0)];
}

// ---- geometry access
// faces of family a on the canvas (one more than the cells along a)
__host__ __device__ __forceinline__ int face_count(const Plan3Dev& p, int a) {
  return (p.NI + (a == 0)) * (p.NJ + (a == 1)) * (p.NK + (a == 2));
}

// a flat index into the three face families, concatenated, to (family, i, j, k)
__host__ __device__ __forceinline__ void face_of(const Plan3Dev& p, int flat, int& a, int& i, int& j, int& k) {
  a = 0;
  while (a < 2 && flat >= face_count(p, a)) flat -= face_count(p, a++);
  const int fj = p.NJ + (a == 1), fk = p.NK + (a == 2);
  i = flat / (fj * fk);
  j = (flat / fk) % fj;
  k = flat % fk;
}

// the flat index of face (i, j, k) of family a
__host__ __device__ __forceinline__ int face_flat(const Plan3Dev& p, int a, int i, int j, int k) {
  int off = 0;
  for (int b = 0; b < a; ++b) off += face_count(p, b);
  return off + (i * (p.NJ + (a == 1)) + j) * (p.NK + (a == 2)) + k;
}

__host__ __device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

struct Cell3 {
  int i, j, k;
};

__host__ __device__ __forceinline__ int cell_index(const Plan3Dev& p, int i, int j, int k) {
  i = clampi(i, 0, p.NI - 1);
  j = clampi(j, 0, p.NJ - 1);
  k = clampi(k, 0, p.NK - 1);
  return (i * p.NJ + j) * p.NK + k;
}

// face (i, j, k) of family a: between cells (i, j, k) - e_a and (i, j, k)
__host__ __device__ __forceinline__ void face_vector(const Plan3Dev& p, int a, int i, int j, int k, double s[3]) {
  const int fi = p.NI + (a == 0), fj = p.NJ + (a == 1), fk = p.NK + (a == 2);
  const size_t nf = (size_t)fi * fj * fk;
  const size_t f = ((size_t)i * fj + j) * fk + k;
  s[0] = p.faces[a][f];
  s[1] = p.faces[a][nf + f];
  s[2] = p.faces[a][2 * nf + f];
}

// centre of canvas cell (i, j, k), -1 <= i <= NI (one ring beyond the canvas)
__host__ __device__ __forceinline__ void centre(const Plan3Dev& p, int i, int j, int k, double x[3]) {
  const int ci = p.NI + 2, cj = p.NJ + 2, ck = p.NK + 2;
  i = clampi(i + 1, 0, ci - 1);
  j = clampi(j + 1, 0, cj - 1);
  k = clampi(k + 1, 0, ck - 1);
  const size_t nc = (size_t)ci * cj * ck;
  const size_t c = ((size_t)i * cj + j) * ck + k;
  x[0] = p.centres[c];
  x[1] = p.centres[nc + c];
  x[2] = p.centres[2 * nc + c];
}

// the mean of the eight cells round node (I, J, K) (cells I-1..I, J-1..J, K-1..K),
// averaged axis by axis: i, then j, then k
__host__ __device__ __forceinline__ void node_centre(const Plan3Dev& p, int I, int J, int K, double x[3]) {
  double c[2][2][2][3];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) centre(p, I - 1 + a, J - 1 + b, K - 1 + d, c[a][b][d]);
  for (int m = 0; m < 3; ++m) {
    double jk[2][2];
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) jk[b][d] = 0.5 * (c[0][b][d][m] + c[1][b][d][m]);
    double kk[2];
    for (int d = 0; d < 2; ++d) kk[d] = 0.5 * (jk[0][d] + jk[1][d]);
    x[m] = 0.5 * (kk[0] + kk[1]);
  }
}

// phi = (u, v, w, T[, nu~]) of a filled primitive cell
template <class T>
__host__ __device__ __forceinline__ void grad_vars(const Plan3Dev& p, const T* Q, int c, T phi[5]) {
  const int n = p.NI * p.NJ * p.NK;
  T rho = Q[c], pr = Q[(size_t)4 * n + c];
  phi[0] = Q[(size_t)n + c];
  phi[1] = Q[(size_t)2 * n + c];
  phi[2] = Q[(size_t)3 * n + c];
  phi[3] = p.P.gamma * pr / rho;
  if (p.nvar > 5) phi[4] = Q[(size_t)5 * n + c];
}

// component m of grad_vars at cell c (the same arithmetic, one component)
template <class T>
__host__ __device__ __forceinline__ T grad_var(const Plan3Dev& p, const T* Q, int c, int m) {
  const int n = p.NI * p.NJ * p.NK;
  if (m < 3) return Q[(size_t)(1 + m) * n + c];
  if (m == 3) return p.P.gamma * Q[(size_t)4 * n + c] / Q[c];
  return Q[(size_t)5 * n + c];
}

// component m of node_phi: the same three halvings of the eight cells' values, one
// component at a time (a face's gradient then never holds all eight cells' values)
template <class T>
__host__ __device__ __forceinline__ T node_phi_m(const Plan3Dev& p, const T* Q, int I, int J, int K, int m) {
  T jk[2][2];
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int d = 0; d < 2; ++d)
      jk[b][d] = 0.5 * (grad_var(p, Q, cell_index(p, I - 1, J - 1 + b, K - 1 + d), m) +
                        grad_var(p, Q, cell_index(p, I, J - 1 + b, K - 1 + d), m));
  T kk[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) kk[d] = 0.5 * (jk[0][d] + jk[1][d]);
  return 0.5 * (kk[0] + kk[1]);
}

template <class T>
__host__ __device__ __forceinline__ void node_phi(const Plan3Dev& p, const T* Q, int I, int J, int K, int nphi, T out[5]) {
  T c[2][2][2][5];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) grad_vars(p, Q, cell_index(p, I - 1 + a, J - 1 + b, K - 1 + d), c[a][b][d]);
  for (int m = 0; m < nphi; ++m) {
    T jk[2][2];
    for (int b = 0; b < 2; ++b)
      for (int d = 0; d < 2; ++d) jk[b][d] = 0.5 * (c[0][b][d][m] + c[1][b][d][m]);
    T kk[2];
    for (int d = 0; d < 2; ++d) kk[d] = 0.5 * (jk[0][d] + jk[1][d]);
    out[m] = 0.5 * (kk[0] + kk[1]);
  }
}

__host__ __device__ __forceinline__ void cross3(const double a[3], const double b[3], double out[3]) {
  out[0] = a[1] * b[2] - a[2] * b[1];
  out[1] = a[2] * b[0] - a[0] * b[2];
  out[2] = a[0] * b[1] - a[1] * b[0];
}

// The diamond gradient at face (fi, fj, fk) of family a: grad[d][m] = d phi_m / d x_d
// (src/jaxrans/numerics/gradients.py:59-95).
template <class T, int NPHI>
__host__ __device__ __forceinline__ void face_gradient(const Plan3Dev& p, const T* Q, int a, int fi, int fj, int fk,
                                                       T grad[3][5]) {
  int lo[3] = {fi, fj, fk}, hi[3] = {fi, fj, fk};
  lo[a] -= 1;
  double xl[3], xh[3];
  centre(p, lo[0], lo[1], lo[2], xl);
  centre(p, hi[0], hi[1], hi[2], xh);
  T pl[5], ph[5];
  grad_vars(p, Q, cell_index(p, lo[0], lo[1], lo[2]), pl);
  grad_vars(p, Q, cell_index(p, hi[0], hi[1], hi[2]), ph);
  // the face's nodes: (shift along the first other axis, along the second), ascending
  const int b1 = a == 0 ? 1 : 0, b2 = a == 2 ? 1 : 2;
  auto node = [&](int s1, int s2, int out[3]) {
    out[0] = fi;
    out[1] = fj;
    out[2] = fk;
    out[b1] += s1;
    out[b2] += s2;
  };
  int n00[3], n11[3], n10[3], n01[3];
  node(0, 0, n00);
  node(1, 1, n11);
  node(1, 0, n10);
  node(0, 1, n01);
  double x00[3], x11[3], x10[3], x01[3];
  node_centre(p, n00[0], n00[1], n00[2], x00);
  node_centre(p, n11[0], n11[1], n11[2], x11);
  node_centre(p, n10[0], n10[1], n10[2], x10);
  node_centre(p, n01[0], n01[1], n01[2], x01);
  double d1[3], d2[3], d3[3];
  for (int m = 0; m < 3; ++m) {
    d1[m] = xh[m] - xl[m];
    d2[m] = x11[m] - x00[m];
    d3[m] = x01[m] - x10[m];
  }
  double c23[3], c31[3], c12[3];
  cross3(d2, d3, c23);
  cross3(d3, d1, c31);
  cross3(d1, d2, c12);
  const double det = d1[0] * c23[0] + d1[1] * c23[1] + d1[2] * c23[2];
#pragma unroll
  for (int m = 0; m < NPHI; ++m) {
    const T f00 = node_phi_m(p, Q, n00[0], n00[1], n00[2], m), f11 = node_phi_m(p, Q, n11[0], n11[1], n11[2], m);
    const T f10 = node_phi_m(p, Q, n10[0], n10[1], n10[2], m), f01 = node_phi_m(p, Q, n01[0], n01[1], n01[2], m);
    T p1 = ph[m] - pl[m], p2 = f11 - f00, p3 = f01 - f10;
#pragma unroll
    for (int d = 0; d < 3; ++d) grad[d][m] = (p1 * c23[d] + p2 * c31[d] + p3 * c12[d]) / det;
  }
}

// the geometry of face (fi, fj, fk)'s diamond gradient, face_gradient's own arithmetic:
// out = c23 (3), c31 (3), c12 (3), det
__host__ __device__ __forceinline__ void face_gradient_geometry(const Plan3Dev& p, int a, int fi, int fj, int fk,
                                                                double out[10]) {
  int lo[3] = {fi, fj, fk}, hi[3] = {fi, fj, fk};
  lo[a] -= 1;
  double xl[3], xh[3];
  centre(p, lo[0], lo[1], lo[2], xl);
  centre(p, hi[0], hi[1], hi[2], xh);
  const int b1 = a == 0 ? 1 : 0, b2 = a == 2 ? 1 : 2;
  int n00[3] = {fi, fj, fk}, n11[3] = {fi, fj, fk}, n10[3] = {fi, fj, fk}, n01[3] = {fi, fj, fk};
  n11[b1] += 1;
  n11[b2] += 1;
  n10[b1] += 1;
  n01[b2] += 1;
  double x00[3], x11[3], x10[3], x01[3];
  node_centre(p, n00[0], n00[1], n00[2], x00);
  node_centre(p, n11[0], n11[1], n11[2], x11);
  node_centre(p, n10[0], n10[1], n10[2], x10);
  node_centre(p, n01[0], n01[1], n01[2], x01);
  double d1[3], d2[3], d3[3];
  for (int m = 0; m < 3; ++m) {
    d1[m] = xh[m] - xl[m];
    d2[m] = x11[m] - x00[m];
    d3[m] = x01[m] - x10[m];
  }
  cross3(d2, d3, out);
  cross3(d3, d1, out + 3);
  cross3(d1, d2, out + 6);
  out[9] = d1[0] * out[0] + d1[1] * out[1] + d1[2] * out[2];
}

__host__ __device__ __forceinline__ int node_flat(const Plan3Dev& p, int I, int J, int K) {
  return (I * (p.NJ + 1) + J) * (p.NK + 1) + K;
}
__host__ __device__ __forceinline__ int node_count(const Plan3Dev& p) { return (p.NI + 1) * (p.NJ + 1) * (p.NK + 1); }

// face_gradient from the plan's stored face geometry (p.face_geo) and this evaluation's
// node values (p.node_buf, filled by k3_node_phi): the same values in the same arithmetic
template <class T, int NPHI>
__host__ __device__ __forceinline__ void face_gradient_stored(const Plan3Dev& p, const T* Q, int a, int fi, int fj,
                                                              int fk, T grad[3][5]) {
  // (shifts by selects, not by indexing small arrays with the family: those would live in
  // local memory)
  T pl[5], ph[5];
  grad_vars(p, Q, cell_index(p, fi - (a == 0), fj - (a == 1), fk - (a == 2)), pl);
  grad_vars(p, Q, cell_index(p, fi, fj, fk), ph);
  const size_t nf = (size_t)face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  const size_t f = (size_t)face_flat(p, a, fi, fj, fk);
  double c23[3], c31[3], c12[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c23[d] = p.face_geo[(size_t)d * nf + f];
    c31[d] = p.face_geo[(size_t)(3 + d) * nf + f];
    c12[d] = p.face_geo[(size_t)(6 + d) * nf + f];
  }
  const double det = p.face_geo[(size_t)9 * nf + f];
  const int b1 = a == 0 ? 1 : 0, b2 = a == 2 ? 1 : 2;
  // node (fi, fj, fk) shifted by s1 along axis b1 and s2 along axis b2
  auto node_at = [&](int s1, int s2) {
    return node_flat(p, fi + (b1 == 0) * s1 + (b2 == 0) * s2, fj + (b1 == 1) * s1 + (b2 == 1) * s2,
                     fk + (b1 == 2) * s1 + (b2 == 2) * s2);
  };
  const int i00 = node_at(0, 0), i11 = node_at(1, 1), i10 = node_at(1, 0), i01 = node_at(0, 1);
  const T* nb = static_cast<const T*>(p.node_buf);
  const size_t nn = (size_t)node_count(p);
#pragma unroll
  for (int m = 0; m < NPHI; ++m) {
    const T f00 = nb[m * nn + i00], f11 = nb[m * nn + i11], f10 = nb[m * nn + i10], f01 = nb[m * nn + i01];
    T p1 = ph[m] - pl[m], p2 = f11 - f00, p3 = f01 - f10;
#pragma unroll
    for (int d = 0; d < 3; ++d) grad[d][m] = (p1 * c23[d] + p2 * c31[d] + p3 * c12[d]) / det;
  }
}

template <class T>
__host__ __device__ __forceinline__ void load_cell(const Plan3Dev& p, const T* Q, int c, T q[NV3_MAX]) {
  const int n = p.NI * p.NJ * p.NK;
  for (int v = 0; v < p.nvar; ++v) q[v] = Q[(size_t)v * n + c];
}

// the same with the variable count known at compile time (the plan's nvar: 6 with SA,
// else 5), so the cell's values stay in registers
template <int NV, class T>
__host__ __device__ __forceinline__ void load_cell_n(const Plan3Dev& p, const T* Q, int c, T q[NV3_MAX]) {
  const int n = p.NI * p.NJ * p.NK;
#pragma unroll
  for (int v = 0; v < NV; ++v) q[v] = Q[(size_t)v * n + c];
}

// The net flux through face (fi, fj, fk) of family a (inviscid minus viscous), and for
// SA the row's face flux (upwind on the mass flux, minus the diffusion).
// QCR2000's addition to the stress (src/jaxrans/physics/spalart_allmaras.py:197-216):
// -c_cr1 (O_ik tau_jk + O_jk tau_ik), O = (grad V - grad V^T) / |grad V| (0 where grad V
// is 0, and so its tangent), tau = mu_t (grad V + grad V^T - 2/3 div V I); with
// gv[a][b] = d v_a / d x_b = grad[b][a].
template <class T>
__host__ __device__ __forceinline__ void qcr_extra(const T grad[3][5], const T& mut, double c_cr1, T extra[3][3]) {
  T gv[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) gv[a][b] = grad[b][a];
  T square = gv[0][0] * gv[0][0];
  for (int e = 1; e < 9; ++e) square = square + gv[e / 3][e % 3] * gv[e / 3][e % 3];
  const bool positive = val(square) > 0.0;
  const T norm = positive ? dsqrt(square) : cst<T>(1.0);
  const T div = (gv[0][0] + gv[1][1]) + gv[2][2];
  T rot[3][3], tau[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      rot[a][b] = (gv[a][b] - gv[b][a]) / norm;
      tau[a][b] = mut * (gv[a][b] + gv[b][a] - (a == b ? (2.0 / 3.0) * div : cst<T>(0.0)));
    }
  T prod[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) prod[i][j] = (rot[i][0] * tau[j][0] + rot[i][1] * tau[j][1]) + rot[i][2] * tau[j][2];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) extra[a][b] = -c_cr1 * (prod[a][b] + prod[b][a]);
}

// FO: 1 first order, 2 second order, 0 as `first_order` says (the kernels fix it at
// compile time, so a first-order flux loads only the two cells either side).  PART: 0 the
// whole flux; 1 its inviscid part (with the SA row's upwind convection); 2 its viscous
// part alone, the terms the whole flux subtracts, negated (0 - term), so that part 1 plus
// part 2 is the whole flux bitwise (a + (0 - b) == a - b).
template <class T, bool VISC, bool SA, int FO = 0, int PART = 0>
__host__ __device__ void face_flux(const Plan3Dev& p, const T* Q, int a, int fi, int fj, int fk, bool first_order_arg,
                                   T F[NV3_MAX]) {
  constexpr int NV = SA ? 6 : 5;
  const bool first_order = FO == 0 ? first_order_arg : FO == 1;
  const Physics3& P = p.P;
  const double g = P.gamma;
  int idx[4];
#pragma unroll
  for (int o = 0; o < 4; ++o)
    idx[o] = cell_index(p, fi + (a == 0) * (o - 2), fj + (a == 1) * (o - 2), fk + (a == 2) * (o - 2));
  T qmm[NV3_MAX], qm[NV3_MAX], qp[NV3_MAX], qpp[NV3_MAX];
  load_cell_n<NV>(p, Q, idx[1], qm);
  load_cell_n<NV>(p, Q, idx[2], qp);
  if (PART != 2 && !first_order) {
    load_cell_n<NV>(p, Q, idx[0], qmm);
    load_cell_n<NV>(p, Q, idx[3], qpp);
  }
  double s[3];
  face_vector(p, a, fi, fj, fk, s);
  if constexpr (PART == 2) {
#pragma unroll
    for (int v = 0; v < NV; ++v) F[v] = cst<T>(0.0);
  } else {
  T qL[5], qR[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    if (first_order) {
      qL[v] = qm[v];
      qR[v] = qp[v];
    } else if (P.limiter == 4) {
      const double lo = 0.25 * (1.0 - P.kappa), hi = 0.25 * (1.0 + P.kappa);
      T dm = qm[v] - qmm[v], dd = qp[v] - qm[v], dp = qpp[v] - qp[v];
      qL[v] = qm[v] + lo * dm + hi * dd;
      qR[v] = qp[v] - lo * dp - hi * dd;
    } else {
      T dm = qm[v] - qmm[v], dd = qp[v] - qm[v], dp = qpp[v] - qp[v];
      qL[v] = qm[v] + 0.5 * limit(dm, dd, P.limiter);
      qR[v] = qp[v] - 0.5 * limit(dd, dp, P.limiter);
    }
  }
  T Fi[5];
  riemann3(P.flux, qL, qR, s, g, Fi);
  for (int v = 0; v < 5; ++v) F[v] = Fi[v];
  if constexpr (NV > 5) F[5] = cst<T>(0.0);
  if constexpr (SA) {
    T up = val(Fi[0]) > 0.0 ? qm[5] : qp[5];
    F[5] = Fi[0] * up;
  }
  }
  if constexpr (VISC && PART != 1) {
    T grad[3][5];
    if constexpr (PART == 2) face_gradient_stored<T, SA ? 5 : 4>(p, Q, a, fi, fj, fk, grad);
    else face_gradient<T, SA ? 5 : 4>(p, Q, a, fi, fj, fk, grad);
    // face means of the two cells either side
    T extra[3][3];
    T vel[3], Tl = g * qm[4] / qm[0], Th = g * qp[4] / qp[0];
    for (int m = 0; m < 3; ++m) vel[m] = 0.5 * (qm[1 + m] + qp[1 + m]);
    T Tf = 0.5 * (Tl + Th);
    T mu = viscosity3(P, Tf);
    T k = mu / (PR_LAMINAR * (g - 1.0));
    if constexpr (SA) {
      T fa[NV3_MAX];
      for (int v = 0; v < 6; ++v) fa[v] = 0.5 * (qm[v] + qp[v]);
      T mu_f = viscosity3(P, g * fa[4] / fa[0]);
      T mut = eddy_viscosity(P.sa, fa[0], fa[5] * P.mu_inf, mu_f / fa[0]);
      mu = mu + mut;
      k = k + mut / (PR_TURBULENT * (g - 1.0));
      if (P.c_cr1 != 0.0) qcr_extra(grad, mut, P.c_cr1, extra);
    }
    // grad[d][c] = d v_c / d x_d (the stress is symmetric in the pair)
    T div = grad[0][0] + grad[1][1] + grad[2][2];
    T ttd = (2.0 / 3.0) * div;
    T force[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      T tau[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (c == d) {
          tau[d] = mu * (2.0 * grad[c][c] - ttd);
        } else {
          const int lo = c < d ? c : d, hi = c < d ? d : c;
          tau[d] = mu * (grad[hi][lo] + grad[lo][hi]);
        }
        if (SA && P.c_cr1 != 0.0) tau[d] = tau[d] + extra[c][d];
      }
      force[c] = tau[0] * s[0] + tau[1] * s[1] + tau[2] * s[2];
    }
    T energy = (vel[0] * force[0] + vel[1] * force[1] + vel[2] * force[2]) +
               k * (grad[0][3] * s[0] + grad[1][3] * s[1] + grad[2][3] * s[2]);
    for (int c = 0; c < 3; ++c) F[1 + c] = F[1 + c] - force[c];
    F[4] = F[4] - energy;
    if constexpr (SA) {
      T fa[NV3_MAX];
      for (int v = 0; v < 6; ++v) fa[v] = 0.5 * (qm[v] + qp[v]);
      T mu_f = viscosity3(P, g * fa[4] / fa[0]);
      T coef = diffusion_coefficient(P.sa, fa[0], fa[5] * P.mu_inf, mu_f);
      T gn = grad[0][4] * s[0] + grad[1][4] * s[1] + grad[2][4] * s[2];
      F[5] = F[5] - coef * gn;
    }
  }
}

// The SA row's source at block cell c, times the volume: the production and destruction
// with |curl V| and the c_b2 gradient term, both from Green-Gauss gradients of the face
// means of (u, v, w, nu~) (src/jaxrans/numerics/turbulence.py).
template <class T>
__host__ __device__ T sa_cell_source(const Plan3Dev& p, const T* __restrict__ Q, int c) {
  const int i = c / (p.NJ * p.NK), j = (c / p.NK) % p.NJ, k = c % p.NK;
  T lo_s[3][5], hi_s[3][5];   // face means of (u, v, w, nu~) for the cell's Green-Gauss gradients
  for (int a = 0; a < 3; ++a) {
    int lo[3] = {i, j, k}, hi[3] = {i, j, k};
    lo[a] -= 1;
    hi[a] += 1;
    T qc[NV3_MAX], ql[NV3_MAX], qh[NV3_MAX];
    load_cell_n<6>(p, Q, c, qc);
    load_cell_n<6>(p, Q, cell_index(p, lo[0], lo[1], lo[2]), ql);
    load_cell_n<6>(p, Q, cell_index(p, hi[0], hi[1], hi[2]), qh);
    for (int m = 0; m < 3; ++m) {
      lo_s[a][m] = 0.5 * (ql[1 + m] + qc[1 + m]);
      hi_s[a][m] = 0.5 * (qc[1 + m] + qh[1 + m]);
    }
    lo_s[a][3] = 0.5 * (ql[5] + qc[5]);
    hi_s[a][3] = 0.5 * (qc[5] + qh[5]);
  }
  const Physics3& P = p.P;
  const double vol = p.volume[c];
  // Green-Gauss: (1/V) sum_families (phi_hi S_hi - phi_lo S_lo)[component]
  T gv[3][3], gn[3];
  for (int comp = 0; comp < 3; ++comp) {
    T tv[3], tn = cst<T>(0.0);
    for (int m = 0; m < 3; ++m) tv[m] = cst<T>(0.0);
    for (int a = 0; a < 3; ++a) {
      int f0[3] = {i, j, k}, f1[3] = {i, j, k};
      f1[a] += 1;
      double s0[3], s1[3];
      face_vector(p, a, f0[0], f0[1], f0[2], s0);
      face_vector(p, a, f1[0], f1[1], f1[2], s1);
      for (int m = 0; m < 3; ++m) {
        T d = hi_s[a][m] * s1[comp] - lo_s[a][m] * s0[comp];
        tv[m] = a == 0 ? d : tv[m] + d;
      }
      T dn = hi_s[a][3] * s1[comp] - lo_s[a][3] * s0[comp];
      tn = a == 0 ? dn : tn + dn;
    }
    for (int m = 0; m < 3; ++m) gv[comp][m] = tv[m] / vol;   // gv[direction][component]
    gn[comp] = tn / vol;
  }
  T cx = gv[1][2] - gv[2][1], cy = gv[2][0] - gv[0][2], cz = gv[0][1] - gv[1][0];
  T sq = (cx * cx + cy * cy) + cz * cz;
  T omega = val(sq) > 0.0 ? dsqrt(sq) : cst<T>(0.0);
  T qc[NV3_MAX];
  load_cell(p, Q, c, qc);
  const double g = P.gamma;
  T mu = viscosity3(P, g * qc[4] / qc[0]);
  T Pr, Dd;
  sa_source(P.sa, qc[5] * P.mu_inf, mu / qc[0], omega, p.distance[c], Pr, Dd);
  T src = qc[0] * ((Pr - Dd) / P.mu_inf + P.sa.c_b2 / P.sa.sigma * P.mu_inf * ((gn[0] * gn[0] + gn[1] * gn[1]) + gn[2] * gn[2]));
  return src * vol;
}

// R of block cell c; R = U - U_inf elsewhere (tangent: v).  Each of the cell's six faces
// evaluated here (the fused form; the device runs the two phases below).
template <class T, bool VISC, bool SA>
__host__ __device__ void residual_cell(const Plan3Dev& p, const T* __restrict__ Q, const double* __restrict__ U,
                                       const double* __restrict__ dU, double* __restrict__ R, int first_order, int c) {
  const int n = p.NI * p.NJ * p.NK;
  if (!p.interior[c]) {
    for (int v = 0; v < p.nvar; ++v)
      R[(size_t)v * n + c] = dU ? dU[(size_t)v * n + c] : U[(size_t)v * n + c] - p.P.U_inf[v];
    return;
  }
  const int i = c / (p.NJ * p.NK), j = (c / p.NK) % p.NJ, k = c % p.NK;
  T acc[NV3_MAX];
  for (int v = 0; v < p.nvar; ++v) acc[v] = cst<T>(0.0);
  for (int a = 0; a < 3; ++a) {
    int f0[3] = {i, j, k}, f1[3] = {i, j, k};
    f1[a] += 1;
    T Flo[NV3_MAX], Fhi[NV3_MAX];
    face_flux<T, VISC, SA>(p, Q, a, f0[0], f0[1], f0[2], first_order != 0, Flo);
    face_flux<T, VISC, SA>(p, Q, a, f1[0], f1[1], f1[2], first_order != 0, Fhi);
    for (int v = 0; v < p.nvar; ++v) acc[v] = a == 0 ? Fhi[v] - Flo[v] : acc[v] + (Fhi[v] - Flo[v]);
  }
  if constexpr (SA) acc[5] = acc[5] - sa_cell_source(p, Q, c);
  for (int v = 0; v < p.nvar; ++v) R[(size_t)v * n + c] = tangent_or_value(acc[v]);
}

// Phase 1 of the two-phase residual: the flux through face `flat` -- its value, or for
// Dual its tangent -- stored at Fb[v * nf + flat], for a face with a block cell on
// either side (no cell reads the others).  Every face is evaluated once instead of once
// from each side, with the same arithmetic, so phase 2's sums are residual_cell's.
// (PART 2: the viscous part added to the stored inviscid part; the mass row has none)
template <class T, bool VISC, bool SA, int FO = 0, int PART = 0>
__host__ __device__ void store_face_flux(const Plan3Dev& p, const T* __restrict__ Q, int first_order, int flat,
                                         double* __restrict__ Fb, size_t nf) {
  constexpr int NV = SA ? 6 : 5;
  int a, i, j, k;
  face_of(p, flat, a, i, j, k);
  int h[3] = {i, j, k}, l[3] = {i, j, k};
  l[a] -= 1;
  const int dims[3] = {p.NI, p.NJ, p.NK};
  const bool hi_in = h[a] < dims[a] && p.interior[(h[0] * p.NJ + h[1]) * p.NK + h[2]];
  const bool lo_in = l[a] >= 0 && p.interior[(l[0] * p.NJ + l[1]) * p.NK + l[2]];
  if (!hi_in && !lo_in) return;
  T F[NV3_MAX];
  face_flux<T, VISC, SA, FO, PART>(p, Q, a, i, j, k, first_order != 0, F);
  if constexpr (PART == 2) {
#pragma unroll
    for (int v = 1; v < NV; ++v) Fb[(size_t)v * nf + flat] = Fb[(size_t)v * nf + flat] + tangent_or_value(F[v]);
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) Fb[(size_t)v * nf + flat] = tangent_or_value(F[v]);
  }
}

// Phase 2: R of cell c from the stored face fluxes (residual_cell's sums and SA source)
template <class T, bool SA>
__host__ __device__ void residual_cell_from_faces(const Plan3Dev& p, const T* __restrict__ Q,
                                                  const double* __restrict__ Fb, size_t nf,
                                                  const double* __restrict__ U, const double* __restrict__ dU,
                                                  double* __restrict__ R, int c) {
  const int n = p.NI * p.NJ * p.NK;
  if (!p.interior[c]) {
    for (int v = 0; v < p.nvar; ++v)
      R[(size_t)v * n + c] = dU ? dU[(size_t)v * n + c] : U[(size_t)v * n + c] - p.P.U_inf[v];
    return;
  }
  constexpr int NV = SA ? 6 : 5;
  const int i = c / (p.NJ * p.NK), j = (c / p.NK) % p.NJ, k = c % p.NK;
  double acc[NV3_MAX];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int f1[3] = {i, j, k};
    f1[a] += 1;
    const int lo = face_flat(p, a, i, j, k), hi = face_flat(p, a, f1[0], f1[1], f1[2]);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double d = Fb[(size_t)v * nf + hi] - Fb[(size_t)v * nf + lo];
      acc[v] = a == 0 ? d : acc[v] + d;
    }
  }
  if constexpr (SA) acc[5] = acc[5] - tangent_or_value(sa_cell_source(p, Q, c));
#pragma unroll
  for (int v = 0; v < NV; ++v) R[(size_t)v * n + c] = acc[v];
}

}  // namespace jr
