// The 3D Newton step on the device: newton3d.cuh's driver over kernel-backed vector
// operations (the residual, J.v, wave speeds and line solve of residual3d.cu and
// linesolve3d.cu; dot products by a fixed-order two-stage reduction, so a step is
// bitwise reproducible).  The driver synchronises for the scalars it needs: each CGS2
// pass's dots come back together (k3_mdot_partial), three reads per Arnoldi step.
#include <cstdio>

#include "linesolve3d.cuh"
#include "newton3d.cuh"
#include "newton3d_ops.cuh"

namespace jr {

constexpr int RED3_BLOCKS = 296, RED3_THREADS = 256;

__global__ void k3_vdt(Plan3Dev p, const double* __restrict__ U, double cfl, double* __restrict__ vdt) {
  const int n = p.NI * p.NJ * p.NK;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    vdt[c] = lambda_sum(p, U, c) / cfl;
}

__global__ void k3_vdt_add(size_t N, size_t n, const double* __restrict__ vdt, const double* __restrict__ z,
                           double* __restrict__ w) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x)
    w[e] = vdt[e % n] * z[e] + w[e];
}

__global__ void k3_axpy(size_t N, double al, const double* __restrict__ x, double* __restrict__ y) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x)
    y[e] = y[e] + al * x[e];
}

__global__ void k3_scale(size_t N, double al, const double* x, double* y) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x)
    y[e] = al * x[e];
}

// per block, fixed-order sums of (a_e b_e) and, for the density norm, of w R0^2 and w
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[RED3_THREADS];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = RED3_THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + o];
    __syncthreads();
  }
  const double out = s[0];
  __syncthreads();
  return out;
}

__global__ void k3_dot_partial(size_t N, const double* __restrict__ a, const double* __restrict__ b,
                               double* __restrict__ partial) {
  double acc = 0.0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x)
    acc = acc + a[e] * b[e];
  const double t = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// the dots of basis vectors 0..count-1 with w in one launch: block (x, i) makes exactly
// the partial sum k3_dot_partial makes for V_i . w
__global__ void k3_mdot_partial(size_t N, const double* __restrict__ V, const double* __restrict__ w,
                                double* __restrict__ partial) {
  const double* a = V + (size_t)blockIdx.y * N;
  double acc = 0.0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x)
    acc = acc + a[e] * w[e];
  const double t = block_sum(acc);
  if (threadIdx.x == 0) partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
}

struct Coeffs3 {
  double c[MAX_RESTART3 + 1];
};

// y += c_0 V_0 + c_1 V_1 + ... + c_{count-1} V_{count-1}, term by term in that order (the
// arithmetic of count axpys, in one pass)
__global__ void k3_maxpy(size_t N, int count, Coeffs3 cf, const double* __restrict__ V, double* __restrict__ y) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < N; e += (size_t)gridDim.x * blockDim.x) {
    double acc = y[e];
    for (int i = 0; i < count; ++i) acc = acc + cf.c[i] * V[(size_t)i * N + e];
    y[e] = acc;
  }
}

__global__ void k3_norm_partial(Plan3Dev p, const double* __restrict__ R, double* __restrict__ partial) {
  const int n = p.NI * p.NJ * p.NK;
  double a = 0.0, w = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    if (p.interior[c]) {
      a = a + p.volume[c] * R[c] * R[c];
      w = w + p.volume[c];
    }
  const double ta = block_sum(a), tw = block_sum(w);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = ta;
    partial[gridDim.x + blockIdx.x] = tw;
  }
}

// the largest relative change a cell's density, pressure or nu~ would see
__global__ void k3_worst_partial(Plan3Dev p, const double* __restrict__ U, const double* __restrict__ D,
                                 double* __restrict__ partial) {
  const int n = p.NI * p.NJ * p.NK;
  const double g = p.P.gamma;
  double worst = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double q[NV3_MAX];
    prim_at(p, U, c, q);
    double de = D[(size_t)4 * n + c];
    for (int k = 0; k < 3; ++k) de = de - q[1 + k] * D[(size_t)(1 + k) * n + c];
    const double vv = (q[1] * q[1] + q[2] * q[2]) + q[3] * q[3];
    const double dp = (g - 1.0) * (de + 0.5 * vv * D[c]);
    worst = fmax(worst, fabs(D[c]) / q[0]);
    worst = fmax(worst, fabs(dp) / q[4]);
    if (p.nvar > 5) {
      const double nh = U[(size_t)5 * n + c] / q[0];
      const double dnh = (D[(size_t)5 * n + c] - nh * D[c]) / q[0];
      worst = fmax(worst, fabs(dnh) / fmax(fabs(nh), 1.0));
    }
  }
  __shared__ double s[RED3_THREADS];
  s[threadIdx.x] = worst;
  __syncthreads();
  for (int o = RED3_THREADS / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// flag 1 where U + D is not physical or D not finite
__global__ void k3_physical(Plan3Dev p, const double* __restrict__ U, const double* __restrict__ D, int* flag) {
  const int n = p.NI * p.NJ * p.NK;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double u[NV3_MAX], q[NV3_MAX];
    bool finite = true;
    for (int v = 0; v < p.nvar; ++v) {
      const double d = D[(size_t)v * n + c];
      finite = finite && isfinite(d);
      u[v] = U[(size_t)v * n + c] + d;
    }
    to_prim3(u, q, p.nvar, p.P.gamma);
    const bool ok = finite && q[0] > 1e-10 && q[4] > 1e-10 && isfinite(q[0]) && isfinite(q[4]);
    if (!ok) atomicOr(flag, 1);
  }
}

static int grid_of(size_t N) {
  const size_t b = (N + 255) / 256;
  return (int)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

// ---- the operations
double DeviceOps3::host_sum(int count, int halves) {
  std::vector<double> h((size_t)count * halves);
  cudaMemcpyAsync(h.data(), partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  double s0 = 0.0, s1 = 0.0;
  for (int b = 0; b < count; ++b) s0 = s0 + h[b];
  if (halves > 1) {
    for (int b = 0; b < count; ++b) s1 = s1 + h[count + b];
    last_second = s1;
  }
  return s0;
}

void DeviceOps3::prepare(const double* U, double cfl) {
  counted3();
  k3_vdt<<<grid_of(n), 128, 0, st>>>(p, U, cfl, vdt);
  if (line) launch_line_factor3(p, U, cfl, factor, st);
}

void DeviceOps3::residual(const double* U, int out) { launch_residual3(p, U, v(out), A, false, st); }

void DeviceOps3::matvec(const double* U, double, int src, int out) {
  launch_jvp3(p, U, v(src), v(out), A, st);
  counted3();
  k3_vdt_add<<<grid_of(N), 256, 0, st>>>(N, n, vdt, v(src), v(out));
}

// the factor of this step's (U, cfl), made in prepare
void DeviceOps3::precondition(const double*, double, int src, int dst) {
  launch_line_apply3(p, factor, v(src), v(dst), st);
}

void DeviceOps3::mdot(int count, int w, double* h) {
  counted3();
  k3_mdot_partial<<<dim3(RED3_BLOCKS, count), RED3_THREADS, 0, st>>>(N, v(V(0)), v(w), partial);
  std::vector<double> part((size_t)count * RED3_BLOCKS);
  cudaMemcpyAsync(part.data(), partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  for (int i = 0; i < count; ++i) {
    double s = 0.0;
    for (int b = 0; b < RED3_BLOCKS; ++b) s = s + part[(size_t)i * RED3_BLOCKS + b];
    h[i] = s;
  }
}

void DeviceOps3::maxpy(int count, const double* coef, int y) {
  Coeffs3 cf{};
  for (int i = 0; i < count; ++i) cf.c[i] = coef[i];
  counted3();
  k3_maxpy<<<grid_of(N), 256, 0, st>>>(N, count, cf, v(V(0)), v(y));
}

double DeviceOps3::dot(int a, int b) {
  counted3();
  k3_dot_partial<<<RED3_BLOCKS, RED3_THREADS, 0, st>>>(N, v(a), v(b), partial);
  return host_sum(RED3_BLOCKS, 1);
}

void DeviceOps3::axpy(double al, int x, int y) {
  counted3();
  k3_axpy<<<grid_of(N), 256, 0, st>>>(N, al, v(x), v(y));
}
void DeviceOps3::scale(double al, int x, int y) {
  counted3();
  k3_scale<<<grid_of(N), 256, 0, st>>>(N, al, v(x), v(y));
}
void DeviceOps3::copy(int x, int y) { cudaMemcpyAsync(v(y), v(x), N * sizeof(double), cudaMemcpyDeviceToDevice, st); }
void DeviceOps3::zero(int y) { cudaMemsetAsync(v(y), 0, N * sizeof(double), st); }

double DeviceOps3::density_norm(int r) {
  counted3();
  k3_norm_partial<<<RED3_BLOCKS, RED3_THREADS, 0, st>>>(p, v(r), partial);
  const double a = host_sum(RED3_BLOCKS, 2);
  return sqrt(a / last_second);
}

double DeviceOps3::worst_ratio(const double* U, int du) {
  counted3();
  k3_worst_partial<<<RED3_BLOCKS, RED3_THREADS, 0, st>>>(p, U, v(du), partial);
  std::vector<double> h(RED3_BLOCKS);
  cudaMemcpyAsync(h.data(), partial, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  double w = 0.0;
  for (double x : h) w = fmax(w, x);
  return w;
}

bool DeviceOps3::physical_after(const double* U, int du) {
  cudaMemsetAsync(flag, 0, sizeof(int), st);
  counted3();
  k3_physical<<<grid_of(n), 128, 0, st>>>(p, U, v(du), flag);
  int h = 0;
  cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  return h == 0;
}

void DeviceOps3::add_to_state(double* U, int du) {
  counted3();
  k3_axpy<<<grid_of(N), 256, 0, st>>>(N, 1.0, v(du), U);
}

size_t DeviceOps3::work_doubles(size_t N, size_t n, int m) {
  return (size_t)(BASE + m + 1) * N + n + (size_t)(m + 1) * RED3_BLOCKS;
}

void DeviceOps3::bind(double* work, int* flag_word, int m) {
  vecs = work;
  vdt = work + (size_t)(BASE + m + 1) * N;
  partial = vdt + n;
  flag = flag_word;
}

double newton_step3_device(DeviceOps3& ops, double* U, double& cfl, double& res_prev, const Newton3Config& c) {
  return newton_step3(ops, U, cfl, res_prev, c);
}

}  // namespace jr
