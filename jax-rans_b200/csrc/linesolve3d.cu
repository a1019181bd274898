// The 3D wave speeds and line preconditioner kernels: one thread per canvas face, one
// thread per chain (the bodies are in linesolve3d.cuh, host-and-device code).
#include "linesolve3d.cuh"

namespace jr {

__global__ void k3_wave_speeds(Plan3Dev p, const double* __restrict__ U, double* __restrict__ lam) {
  const int n0 = face_count(p, 0), n1 = face_count(p, 1), n2 = face_count(p, 2);
  const int total = n0 + n1 + n2;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x) {
    int a, i, j, k;
    face_of(p, f, a, i, j, k);
    lam[f] = wave_speed(p, U, a, i, j, k);
  }
}

__global__ void k3_copy_rows(int n, const double* __restrict__ r, double* __restrict__ z) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) z[e] = r[e];
}

template <class TF>
__global__ void __launch_bounds__(64) k3_chain_factor(Plan3Dev p, const double* __restrict__ U, double cfl,
                                                      TF* __restrict__ F) {
  for (int ch = blockIdx.x * blockDim.x + threadIdx.x; ch < p.n_chains; ch += gridDim.x * blockDim.x) {
    chain_factor_flow(p, U, cfl, ch, F);
    if (p.nvar > 5) chain_factor_sa(p, U, cfl, ch, F);
  }
}

template <class TF>
__global__ void __launch_bounds__(128) k3_chain_apply(Plan3Dev p, const TF* __restrict__ F,
                                                      const double* __restrict__ r, double* __restrict__ z) {
  for (int ch = blockIdx.x * blockDim.x + threadIdx.x; ch < p.n_chains; ch += gridDim.x * blockDim.x) {
    chain_apply_flow(p, ch, F, r, z);
    if (p.nvar > 5) chain_apply_sa(p, ch, F, r, z);
  }
}

void launch_wave_speeds3(const Plan3Dev& p, const double* U, double* lam, cudaStream_t st) {
  const int total = face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  counted3();
  k3_wave_speeds<<<(total + 127) / 128, 128, 0, st>>>(p, U, lam);
}

// the line_j factor at (U, cfl) into F: n_chains * chain_L * FACTOR3 words, FP32 where
// p.line_fp32 (the mixed form), else FP64
void launch_line_factor3(const Plan3Dev& p, const double* U, double cfl, void* F, cudaStream_t st) {
  if (p.n_chains == 0) return;
  counted3();
  if (p.line_fp32)
    k3_chain_factor<float><<<(p.n_chains + 63) / 64, 64, 0, st>>>(p, U, cfl, static_cast<float*>(F));
  else
    k3_chain_factor<double><<<(p.n_chains + 63) / 64, 64, 0, st>>>(p, U, cfl, static_cast<double*>(F));
}

// z = M^-1 r from the factor F: r copied where no chain runs (ghosts and the canvas gaps)
void launch_line_apply3(const Plan3Dev& p, const void* F, const double* r, double* z, cudaStream_t st) {
  const int n = p.nvar * p.NI * p.NJ * p.NK;
  counted3(p.n_chains > 0 ? 2 : 1);
  k3_copy_rows<<<(n + 255) / 256, 256, 0, st>>>(n, r, z);
  if (p.n_chains == 0) return;
  if (p.line_fp32)
    k3_chain_apply<float><<<(p.n_chains + 127) / 128, 128, 0, st>>>(p, static_cast<const float*>(F), r, z);
  else
    k3_chain_apply<double><<<(p.n_chains + 127) / 128, 128, 0, st>>>(p, static_cast<const double*>(F), r, z);
}

void launch_precondition3(const Plan3Dev& p, const double* U, double cfl, const double* r, double* z, void* F,
                          cudaStream_t st) {
  launch_line_factor3(p, U, cfl, F, st);
  launch_line_apply3(p, F, r, z, st);
}

}  // namespace jr
