// The device's vector operations for the 3D Newton driver (newton3d.cuh): vectors of
// the canvas length N = nvar * cells in one workspace, basis vector i at V(i).
#pragma once
#include <vector>

#include "device3d.cuh"
#include "newton3d.cuh"

namespace jr {

struct DeviceOps3 {
  enum { R_ = 0, Z_, W_, T_, RES_, B_, DU_, ACT_, BASE };
  Plan3Dev p;
  size_t N = 0, n = 0;
  void* A = nullptr;                 // the primitive canvas of the residual / J.v (Dual-sized)
  void* factor = nullptr;            // the line factor (computed in prepare when line)
  bool line = false;
  double* vecs = nullptr;
  double* vdt = nullptr;
  double* partial = nullptr;
  int* flag = nullptr;
  double last_second = 0.0;
  cudaStream_t st = nullptr;

  int V(int i) const { return BASE + i; }
  double* v(int id) const { return vecs + (size_t)id * N; }
  double host_sum(int count, int halves);
  void prepare(const double* U, double cfl);
  void residual(const double* U, int out);
  void matvec(const double* U, double cfl, int src, int out);
  void precondition(const double* U, double cfl, int src, int dst);
  double dot(int a, int b);
  void mdot(int count, int w, double* h);                 // h[i] = V(i) . w, i < count
  void maxpy(int count, const double* coef, int y);       // y += sum_i coef[i] V(i), in order
  double nrm2(int a) { return sqrt(dot(a, a)); }
  void axpy(double al, int x, int y);
  void scale(double al, int x, int y);
  void copy(int x, int y);
  void zero(int y);
  double density_norm(int r);
  double worst_ratio(const double* U, int du);
  bool physical_after(const double* U, int du);
  void add_to_state(double* U, int du);
  static size_t work_doubles(size_t N, size_t n, int m);
  void bind(double* work, int* flag_word, int m);
};

double newton_step3_device(DeviceOps3& ops, double* U, double& cfl, double& res_prev, const Newton3Config& c);

}  // namespace jr
