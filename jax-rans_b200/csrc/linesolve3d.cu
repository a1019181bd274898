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

__global__ void __launch_bounds__(64) k3_chain_solve(Plan3Dev p, const double* __restrict__ U, double cfl,
                                                     const double* __restrict__ r, double* __restrict__ z,
                                                     double* __restrict__ scratch) {
  const int L = p.chain_L;
  for (int ch = blockIdx.x * blockDim.x + threadIdx.x; ch < p.n_chains; ch += gridDim.x * blockDim.x) {
    double* Cs = scratch + (size_t)ch * L * 30;
    double* Ds = Cs + (size_t)L * 25;
    chain_flow(p, U, cfl, ch, r, z, Cs, Ds);
    if (p.nvar > 5) chain_sa(p, U, cfl, ch, r, z, Cs, Ds);
  }
}

void launch_wave_speeds3(const Plan3Dev& p, const double* U, double* lam, cudaStream_t st) {
  const int total = face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  counted3();
  k3_wave_speeds<<<(total + 127) / 128, 128, 0, st>>>(p, U, lam);
}

// scratch: n_chains * chain_L * 30 doubles
void launch_precondition3(const Plan3Dev& p, const double* U, double cfl, const double* r, double* z, double* scratch,
                          cudaStream_t st) {
  const int n = p.nvar * p.NI * p.NJ * p.NK;
  counted3(p.n_chains > 0 ? 2 : 1);
  k3_copy_rows<<<(n + 255) / 256, 256, 0, st>>>(n, r, z);
  if (p.n_chains > 0) k3_chain_solve<<<(p.n_chains + 63) / 64, 64, 0, st>>>(p, U, cfl, r, z, scratch);
}

}  // namespace jr
