// The 3D residual R2(U) and the exact first-order J.v on a 3D plan (a swept, tapered
// wing's C-H block; the reference's 3D path, src/jaxrans/numerics/residual.py:54-91,
// 273-334, on the canvas of src/jaxrans/mesh/atlas3d.py:119-210).
//
// The ghost fill runs its gather stages as record kernels (one thread per ghost record,
// double-buffered so every read of a stage precedes its writes); then one thread per
// face evaluates its flux once -- MUSCL on the flow rows, HLLC or Roe with a vector
// normal, the 3D diamond face gradient, the viscous flux (with QCR2000), the SA row's
// convection and diffusion -- into a face buffer, and one thread per cell sums F_hi -
// F_lo per family and adds the SA source with |curl V|.  Templated on the scalar: `double` for R(U), `Dual` (value + tangent) for
// the J.v of the first-order residual.  Every canvas index is clamped to the canvas, the
// reference's edge padding.
#include <cstdint>

#include "linesolve3d.cuh"
#include "residual3d.cuh"

namespace jr {

template <class T, int NV>
__global__ void k3_prim(Plan3Dev p, const double* __restrict__ U, const double* __restrict__ dU, T* __restrict__ Q) {
  const int n = p.NI * p.NJ * p.NK;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    prim_cell_n<NV>(p, U, dU, Q, c);
}

// the primitive canvas of U (and dU) into Q
template <class T>
static void prim_canvas(const Plan3Dev& p, const double* U, const double* dU, T* Q, cudaStream_t st) {
  const int blocks = (p.NI * p.NJ * p.NK + 127) / 128;
  if (p.nvar > 5) k3_prim<T, 6><<<blocks, 128, 0, st>>>(p, U, dU, Q);
  else k3_prim<T, 5><<<blocks, 128, 0, st>>>(p, U, dU, Q);
}

template <class T>
__global__ void k3_ghost_values(Plan3Dev p, const T* __restrict__ Q, int r0, int r1, T* __restrict__ buf) {
  for (int r = r0 + blockIdx.x * blockDim.x + threadIdx.x; r < r1; r += gridDim.x * blockDim.x)
    ghost_value(p, Q, r, r0, r1 - r0, buf);
}

template <class T>
__global__ void k3_ghost_store(Plan3Dev p, const T* __restrict__ buf, int r0, int r1, T* __restrict__ Q) {
  for (int r = r0 + blockIdx.x * blockDim.x + threadIdx.x; r < r1; r += gridDim.x * blockDim.x)
    ghost_store(p, buf, r, r0, r1 - r0, Q);
}

// phase 1: every face's flux once (one thread per face of the three families)
// the diamond gradients' geometry of every face (once per plan, viscous cases)
__global__ void k3_face_geometry(Plan3Dev p, double* __restrict__ geo, int nf) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
    int a, i, j, k;
    face_of(p, f, a, i, j, k);
    double g[10];
    face_gradient_geometry(p, a, i, j, k, g);
    for (int q = 0; q < 10; ++q) geo[(size_t)q * nf + f] = g[q];
  }
}

// every node's mean of its eight cells' gradient variables, for the evaluation's canvas Q
template <class T, int NPHI>
__global__ void k3_node_phi(Plan3Dev p, const T* __restrict__ Q) {
  const int nn = node_count(p);
  T* nb = static_cast<T*>(p.node_buf);
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += gridDim.x * blockDim.x) {
    const int I = e / ((p.NJ + 1) * (p.NK + 1)), J = (e / (p.NK + 1)) % (p.NJ + 1), K = e % (p.NK + 1);
#pragma unroll
    for (int m = 0; m < NPHI; ++m) nb[(size_t)m * nn + e] = node_phi_m(p, Q, I, J, K, m);
  }
}

void launch_face_geometry3(const Plan3Dev& p, double* geo, cudaStream_t st) {
  const int nf = face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  counted3();
  k3_face_geometry<<<(nf + 127) / 128, 128, 0, st>>>(p, geo, nf);
}

// (FO 1: the first-order flux, 2: second order; PART 0: the whole flux, 1: its inviscid
// part, 2: its viscous part added to the stored inviscid part)
template <class T, bool VISC, bool SA, int FO, int PART>
__global__ void __launch_bounds__(128) k3_face_flux(Plan3Dev p, const T* __restrict__ Q, int nf) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x)
    store_face_flux<T, VISC, SA, FO, PART>(p, Q, FO == 1, f, p.face_buf, (size_t)nf);
}

// A viscous flux in two launches (inviscid, then viscous added): each holds half the
// live values of the whole, so neither spills the way the fused face did.  The viscous
// launch reads its diamond gradient's geometry from the plan (k3_face_geometry) and the
// node values from this evaluation's node pass (k3_node_phi: each node once, not once
// for each of the twelve faces round it).
template <class T, bool VISC, bool SA, int FO>
static void face_parts(const Plan3Dev& p, const T* A, int nf, cudaStream_t st) {
  const int fblocks = (nf + 127) / 128;
  if constexpr (VISC) {
    counted3(2);
    const int nn = node_count(p);
    k3_node_phi<T, SA ? 5 : 4><<<(nn + 127) / 128, 128, 0, st>>>(p, A);
    k3_face_flux<T, VISC, SA, FO, 1><<<fblocks, 128, 0, st>>>(p, A, nf);
    k3_face_flux<T, VISC, SA, FO, 2><<<fblocks, 128, 0, st>>>(p, A, nf);
  } else {
    k3_face_flux<T, VISC, SA, FO, 0><<<fblocks, 128, 0, st>>>(p, A, nf);
  }
}

template <class T, bool VISC, bool SA>
static void face_phase(const Plan3Dev& p, const T* A, bool first_order, int nf, cudaStream_t st) {
  if (first_order) face_parts<T, VISC, SA, 1>(p, A, nf, st);
  else face_parts<T, VISC, SA, 2>(p, A, nf, st);
}

// phase 2: each cell's sum of its faces' fluxes (and the SA source)
template <class T, bool SA>
__global__ void __launch_bounds__(128) k3_cell_sum(Plan3Dev p, const T* __restrict__ Q, const double* __restrict__ U,
                                                   const double* __restrict__ dU, double* __restrict__ R, int nf) {
  const int n = p.NI * p.NJ * p.NK;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    residual_cell_from_faces<T, SA>(p, Q, p.face_buf, (size_t)nf, U, dU, R, c);
}

// ---- launchers
// the ghost stages on the canvas A in place, each in two passes through p.ghost_buf
template <class T>
static void fill3(const Plan3Dev& p, T* A, cudaStream_t st) {
  T* buf = static_cast<T*>(p.ghost_buf);
  for (int s = 0; s < p.n_stages; ++s) {
    const int r0 = p.stage_off[s], r1 = p.stage_off[s + 1];
    const int blocks = (r1 - r0 + 127) / 128;
    if (blocks > 0) {
      counted3(2);
      k3_ghost_values<T><<<blocks, 128, 0, st>>>(p, A, r0, r1, buf);
      k3_ghost_store<T><<<blocks, 128, 0, st>>>(p, buf, r0, r1, A);
    }
  }
}

template <class T>
static void residual3_t(const Plan3Dev& p, const double* U, const double* dU, double* R, T* A, bool first_order,
                        cudaStream_t st) {
  const int n = p.NI * p.NJ * p.NK;
  const int blocks = (n + 127) / 128;
  counted3(2);   // the primitive canvas and, below, the residual
  prim_canvas<T>(p, U, dU, A, st);
  fill3(p, A, st);
  const bool visc = p.P.mu_inf > 0.0, sa = p.nvar > 5;
  const int nf = face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  counted3();   // the face phase (the cell phase is counted with the primitive canvas)
  if (sa)
    face_phase<T, true, true>(p, A, first_order, nf, st);
  else if (visc)
    face_phase<T, true, false>(p, A, first_order, nf, st);
  else
    face_phase<T, false, false>(p, A, first_order, nf, st);
  if (sa)
    k3_cell_sum<T, true><<<blocks, 128, 0, st>>>(p, A, U, dU, R, nf);
  else
    k3_cell_sum<T, false><<<blocks, 128, 0, st>>>(p, A, U, dU, R, nf);
}

__global__ void k3_wall_loads(Plan3Dev p, const double* __restrict__ Q, double* __restrict__ loads) {
  for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < p.n_walls; w += gridDim.x * blockDim.x)
    wall_load(p, Q, w, loads + (size_t)7 * w);
}

// the loads on every wall face (7 each) at U: the primitive canvas ghost-filled first
void launch_wall_loads3(const Plan3Dev& p, const double* U, double* loads, void* A, cudaStream_t st) {
  const int n = p.NI * p.NJ * p.NK;
  counted3(p.n_walls > 0 ? 2 : 1);
  prim_canvas<double>(p, U, nullptr, (double*)A, st);
  fill3(p, (double*)A, st);
  if (p.n_walls > 0) k3_wall_loads<<<(p.n_walls + 127) / 128, 128, 0, st>>>(p, (const double*)A, loads);
}

void launch_residual3(const Plan3Dev& p, const double* U, double* R, void* A, bool first_order, cudaStream_t st) {
  residual3_t<double>(p, U, nullptr, R, (double*)A, first_order, st);
}

void launch_jvp3(const Plan3Dev& p, const double* U, const double* v, double* Jv, void* A, cudaStream_t st) {
  residual3_t<Dual>(p, U, v, Jv, (Dual*)A, true, st);
}

}  // namespace jr
