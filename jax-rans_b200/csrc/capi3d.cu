// The C ABI of the 3D path: a plan of one 3D case (device copies of its canvas tables
// and ghost records, two work buffers, a stream), its residual and its J.v.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/jaxrans_b200.h"
#include "newton3d_ops.cuh"
#include "plan3d_desc.cuh"

namespace jr {
int report_error(int code, const std::string& msg);
}  // namespace jr

using namespace jr;

long long& jr::launches3() {
  static long long n = 0;
  return n;
}

struct jr_plan3d {
  Plan3Dev dev{};
  std::vector<void*> allocs;
  void* A = nullptr;   // primitive canvases (Dual-sized: the J.v needs value and tangent)
  void* factor = nullptr;      // the line factor: n_chains * chain_L * FACTOR3 words (FP32 in the mixed form)
  size_t n_canvas = 0;
  Newton3Config cfg{};
  double* loads = nullptr;     // 7 per wall face
  std::vector<double> wall_mid;
  double* work = nullptr;      // the Newton step's vectors
  int* flag = nullptr;
  cudaStream_t st = nullptr;
};

static int check3(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return report_error(JR_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
  return JR_OK;
}

template <class T> static int copy3(jr_plan3d* p, const T** dst, const T* src, size_t n) {
  *dst = nullptr;
  if (n == 0 || src == nullptr) return JR_OK;
  void* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(T)) != cudaSuccess) return report_error(JR_ENOMEM, "cudaMalloc failed");
  p->allocs.push_back(d);
  if (cudaMemcpy(d, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return report_error(JR_ECUDA, "cudaMemcpy to the device failed");
  *dst = static_cast<const T*>(d);
  return JR_OK;
}

#define TRY3(x)              \
  do {                       \
    int rc_ = (x);           \
    if (rc_ != JR_OK) {      \
      jr_plan3d_destroy(p);  \
      return rc_;            \
    }                        \
  } while (0)

extern "C" {

int jr_plan3d_destroy(jr_plan3d* plan) {
  if (!plan) return JR_OK;
  for (void* a : plan->allocs) cudaFree(a);
  if (plan->st) cudaStreamDestroy(plan->st);
  delete plan;
  return JR_OK;
}

int jr_plan3d_create(const jr_plan3d_desc* d, jr_plan3d** out) {
  if (!d || !out) return report_error(JR_EINVAL, "null argument");
  *out = nullptr;
  if (d->NI < 5 || d->NJ < 5 || d->NK < 5) return report_error(JR_EINVAL, "a 3D canvas needs at least 5 cells a side");
  if (d->nvar != 5 && d->nvar != 6) return report_error(JR_EINVAL, "nvar must be 5 or 6");
  if (d->nvar == 6 && !(d->mu_inf > 0.0)) return report_error(JR_EINVAL, "the SA model needs a viscous flow");
  if (d->nvar == 6 && !d->distance) return report_error(JR_EINVAL, "the SA model needs the wall distance");
  if (d->n_stages < 1 || d->n_stages > MAX_STAGES3) return report_error(JR_EINVAL, "1 to 12 ghost stages");
  if (!d->interior || !d->volume || !d->centres || !d->faces[0] || !d->faces[1] || !d->faces[2] ||
      !d->stage_records)
    return report_error(JR_EINVAL, "null table");
  if (d->flux < 0 || d->flux > 1 || d->limiter < 0 || d->limiter > 4)
    return report_error(JR_EINVAL, "unknown flux or limiter code");
  const size_t n = (size_t)d->NI * d->NJ * d->NK;
  if (n > (size_t)(1u << 30)) return report_error(JR_EINVAL, "canvas too large");
  // the records: every index inside the canvas, every kind known
  size_t n_rec = 0;
  for (int s = 0; s < d->n_stages; ++s) {
    if (d->stage_records[s] < 0) return report_error(JR_EINVAL, "negative record count");
    n_rec += (size_t)d->stage_records[s];
  }
  if (n_rec > 0 && (!d->ghost || !d->source || !d->kind || !d->normal))
    return report_error(JR_EINVAL, "null ghost records");
  for (size_t r = 0; r < n_rec; ++r) {
    if (d->ghost[r] < 0 || (size_t)d->ghost[r] >= n || d->source[r] < 0 || (size_t)d->source[r] >= n)
      return report_error(JR_EINVAL, "a ghost record outside the canvas");
    if (d->kind[r] < 0 || d->kind[r] > 4) return report_error(JR_EINVAL, "unknown ghost record kind");
  }
  // the neighbour map and the chains: every cell and face inside the canvas
  if (!d->neighbours) return report_error(JR_EINVAL, "null neighbour map");
  for (size_t c = 0; c < n; ++c)
    if (d->neighbours[c] < 0 || (size_t)d->neighbours[c] >= n) return report_error(JR_EINVAL, "a neighbour outside the canvas");
  const size_t n_faces = (size_t)(d->NI + 1) * d->NJ * d->NK + (size_t)d->NI * (d->NJ + 1) * d->NK +
                         (size_t)d->NI * d->NJ * (d->NK + 1);
  if (d->n_chains < 0 || d->chain_L < 0 || (d->n_chains > 0 && (d->chain_L < 1 || !d->chain_cells ||
                                                                 !d->chain_up_face || !d->chain_up_sign)))
    return report_error(JR_EINVAL, "bad chains");
  const size_t n_links = (size_t)d->n_chains * d->chain_L;
  for (size_t e = 0; e < n_links; ++e) {
    if (d->chain_cells[e] < -1 || d->chain_cells[e] >= (int64_t)n) return report_error(JR_EINVAL, "a chain cell outside the canvas");
    if (d->chain_up_face[e] < 0 || (size_t)d->chain_up_face[e] >= n_faces)
      return report_error(JR_EINVAL, "a chain face outside the canvas");
    if (d->chain_up_sign[e] < -1 || d->chain_up_sign[e] > 1) return report_error(JR_EINVAL, "a chain sign not in {-1, 0, 1}");
  }
  jr_plan3d* p = new jr_plan3d();
  p->n_canvas = n;
  Plan3Dev& dv = p->dev;
  dv.NI = d->NI;
  dv.NJ = d->NJ;
  dv.NK = d->NK;
  dv.nvar = d->nvar;
  TRY3(copy3(p, &dv.interior, d->interior, n));
  TRY3(copy3(p, &dv.volume, d->volume, n));
  for (int a = 0; a < 3; ++a) {
    const size_t nf = (size_t)(d->NI + (a == 0)) * (d->NJ + (a == 1)) * (d->NK + (a == 2));
    TRY3(copy3(p, &dv.faces[a], d->faces[a], 3 * nf));
  }
  TRY3(copy3(p, &dv.centres, d->centres, 3 * (size_t)(d->NI + 2) * (d->NJ + 2) * (d->NK + 2)));
  TRY3(copy3(p, &dv.distance, d->nvar == 6 ? d->distance : nullptr, n));
  dv.n_stages = d->n_stages;
  dv.stage_off[0] = 0;
  for (int s = 0; s < d->n_stages; ++s) dv.stage_off[s + 1] = dv.stage_off[s] + d->stage_records[s];
  TRY3(copy3(p, &dv.g_ghost, d->ghost, n_rec));
  TRY3(copy3(p, &dv.g_source, d->source, n_rec));
  TRY3(copy3(p, &dv.g_kind, d->kind, n_rec));
  TRY3(copy3(p, &dv.g_normal, d->normal, 3 * n_rec));
  TRY3(copy3(p, &dv.neighbours, d->neighbours, n));
  dv.n_chains = d->n_chains;
  dv.chain_L = d->chain_L;
  TRY3(copy3(p, &dv.ch_cells, d->chain_cells, n_links));
  TRY3(copy3(p, &dv.ch_face, d->chain_up_face, n_links));
  TRY3(copy3(p, &dv.ch_sign, d->chain_up_sign, n_links));
  if (d->n_walls < 0 || (d->n_walls > 0 && (!d->wall_cell || !d->wall_family || !d->wall_face || !d->wall_into ||
                                            !d->wall_mid))) {
    jr_plan3d_destroy(p);
    return report_error(JR_EINVAL, "bad wall tables");
  }
  for (int w = 0; w < d->n_walls; ++w) {
    const int a = d->wall_family[w];
    const size_t nf = a >= 0 && a < 3 ? (size_t)(d->NI + (a == 0)) * (d->NJ + (a == 1)) * (d->NK + (a == 2)) : 0;
    if (a < 0 || a > 2 || d->wall_face[w] < 0 || (size_t)d->wall_face[w] >= nf || d->wall_cell[w] < 0 ||
        (size_t)d->wall_cell[w] >= n) {
      jr_plan3d_destroy(p);
      return report_error(JR_EINVAL, "a wall face outside the canvas");
    }
  }
  dv.n_walls = d->n_walls;
  TRY3(copy3(p, &dv.w_cell, d->wall_cell, (size_t)d->n_walls));
  TRY3(copy3(p, &dv.w_family, d->wall_family, (size_t)d->n_walls));
  TRY3(copy3(p, &dv.w_face, d->wall_face, (size_t)d->n_walls));
  TRY3(copy3(p, &dv.w_into, d->wall_into, (size_t)d->n_walls));
  p->wall_mid.assign(d->wall_mid, d->wall_mid + 3 * (size_t)d->n_walls);
  if (d->n_walls > 0) {
    void* l = nullptr;
    if (cudaMalloc(&l, (size_t)d->n_walls * 7 * sizeof(double)) != cudaSuccess) {
      jr_plan3d_destroy(p);
      return report_error(JR_ENOMEM, "cudaMalloc failed");
    }
    p->allocs.push_back(l);
    p->loads = static_cast<double*>(l);
  }
  physics3_from_desc(dv.P, d);
  if (d->line_precision != 0 && d->line_precision != 1) {
    jr_plan3d_destroy(p);
    return report_error(JR_EINVAL, "line_precision must be 0 (FP64) or 1 (FP32)");
  }
  dv.line_fp32 = d->line_precision;
  dv.line_coupled = d->preconditioner == 2;
  if (n_links > 0) {
    void* sc = nullptr;
    if (cudaMalloc(&sc, n_links * FACTOR3 * (dv.line_fp32 ? sizeof(float) : sizeof(double))) != cudaSuccess) {
      jr_plan3d_destroy(p);
      return report_error(JR_ENOMEM, "cudaMalloc failed");
    }
    p->allocs.push_back(sc);
    p->factor = sc;
  }
  {
    size_t most = 1;
    for (int s = 0; s < d->n_stages; ++s) most = (size_t)d->stage_records[s] > most ? (size_t)d->stage_records[s] : most;
    void* gb = nullptr;
    if (cudaMalloc(&gb, most * d->nvar * sizeof(Dual)) != cudaSuccess) {
      jr_plan3d_destroy(p);
      return report_error(JR_ENOMEM, "cudaMalloc failed");
    }
    p->allocs.push_back(gb);
    dv.ghost_buf = gb;
  }
  {
    const size_t nf = (size_t)(d->NI + 1) * d->NJ * d->NK + (size_t)d->NI * (d->NJ + 1) * d->NK +
                      (size_t)d->NI * d->NJ * (d->NK + 1);
    void* fb = nullptr;
    if (cudaMalloc(&fb, nf * d->nvar * sizeof(double)) != cudaSuccess) {
      jr_plan3d_destroy(p);
      return report_error(JR_ENOMEM, "cudaMalloc failed");
    }
    p->allocs.push_back(fb);
    dv.face_buf = static_cast<double*>(fb);
  }
  if (d->mu_inf > 0.0) {   // viscous: the faces' gradient geometry and the node values
    const size_t nf = (size_t)(d->NI + 1) * d->NJ * d->NK + (size_t)d->NI * (d->NJ + 1) * d->NK +
                      (size_t)d->NI * d->NJ * (d->NK + 1);
    const size_t nn = (size_t)(d->NI + 1) * (d->NJ + 1) * (d->NK + 1);
    void *geo = nullptr, *nb = nullptr;
    if (cudaMalloc(&geo, nf * 10 * sizeof(double)) != cudaSuccess ||
        (p->allocs.push_back(geo), cudaMalloc(&nb, nn * 5 * sizeof(Dual))) != cudaSuccess) {
      jr_plan3d_destroy(p);
      return report_error(JR_ENOMEM, "cudaMalloc failed");
    }
    p->allocs.push_back(nb);
    dv.face_geo = static_cast<const double*>(geo);
    dv.node_buf = nb;
  }
  const size_t work = (size_t)d->nvar * n * sizeof(Dual);
  if (cudaMalloc(&p->A, work) != cudaSuccess) {
    jr_plan3d_destroy(p);
    return report_error(JR_ENOMEM, "cudaMalloc failed");
  }
  p->allocs.push_back(p->A);
  // the Newton step's configuration and vectors
  if (d->krylov_subspace < 1 || d->krylov_subspace > MAX_RESTART3 || d->krylov_restarts < 1 || d->preconditioner < 0 ||
      d->preconditioner > 2) {
    jr_plan3d_destroy(p);
    return report_error(JR_EINVAL, "krylov_subspace 1..64, krylov_restarts >= 1, preconditioner 0, 1 or 2");
  }
  p->cfg = Newton3Config{d->krylov_subspace, d->krylov_restarts, d->preconditioner, d->krylov_tol, d->krylov_success,
                         d->max_relative_update, d->cfl_min, d->cfl_max, d->cfl_growth, d->cfl_cutback};
  {
    const size_t words = DeviceOps3::work_doubles((size_t)d->nvar * n, n, d->krylov_subspace);
    void *w = nullptr, *f = nullptr;
    if (cudaMalloc(&w, words * sizeof(double)) != cudaSuccess || (p->allocs.push_back(w), cudaMalloc(&f, sizeof(int))) != cudaSuccess) {
      jr_plan3d_destroy(p);
      return report_error(JR_ENOMEM, "cudaMalloc failed");
    }
    p->allocs.push_back(f);
    p->work = static_cast<double*>(w);
    p->flag = static_cast<int*>(f);
  }
  if (cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking) != cudaSuccess) {
    jr_plan3d_destroy(p);
    return report_error(JR_ECUDA, "stream");
  }
  if (dv.face_geo != nullptr) {
    launch_face_geometry3(dv, const_cast<double*>(dv.face_geo), p->st);
    cudaStreamSynchronize(p->st);
  }
  int rc = check3("jr_plan3d_create");
  if (rc) {
    jr_plan3d_destroy(p);
    return rc;
  }
  *out = p;
  return JR_OK;
}

int jr_residual3d(jr_plan3d* plan, const double* U, double* R, int32_t first_order) {
  if (!plan || !U || !R) return report_error(JR_EINVAL, "null argument");
  launch_residual3(plan->dev, U, R, plan->A, first_order != 0, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_residual3d");
  return check3("jr_residual3d");
}

int jr_jvp3d(jr_plan3d* plan, const double* U, const double* v, double* Jv) {
  if (!plan || !U || !v || !Jv) return report_error(JR_EINVAL, "null argument");
  launch_jvp3(plan->dev, U, v, Jv, plan->A, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_jvp3d");
  return check3("jr_jvp3d");
}

int jr_wave_speeds3d(jr_plan3d* plan, const double* U, double* lam) {
  if (!plan || !U || !lam) return report_error(JR_EINVAL, "null argument");
  launch_wave_speeds3(plan->dev, U, lam, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_wave_speeds3d");
  return check3("jr_wave_speeds3d");
}

int jr_precondition3d(jr_plan3d* plan, const double* U, double cfl, const double* r, double* z) {
  if (!plan || !U || !r || !z) return report_error(JR_EINVAL, "null argument");
  if (!(cfl > 0.0)) return report_error(JR_EINVAL, "cfl must be positive");
  launch_precondition3(plan->dev, U, cfl, r, z, plan->factor, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_precondition3d");
  return check3("jr_precondition3d");
}

int jr_newton_steps3d(jr_plan3d* plan, double* U, int32_t n_steps, double* cfl, double* residual_norm,
                      double* history) {
  if (!plan || !U || !cfl || !residual_norm || n_steps < 0) return report_error(JR_EINVAL, "bad argument");
  if (!(*cfl > 0.0)) return report_error(JR_EINVAL, "cfl must be positive");
  DeviceOps3 ops;
  ops.p = plan->dev;
  ops.n = plan->n_canvas;
  ops.N = (size_t)plan->dev.nvar * plan->n_canvas;
  ops.A = plan->A;
  ops.factor = plan->factor;
  ops.line = plan->cfg.preconditioner >= 1;
  ops.st = plan->st;
  ops.bind(plan->work, plan->flag, plan->cfg.restart);
  double c = *cfl, r = *residual_norm;
  for (int s = 0; s < n_steps; ++s) {
    const double norm = newton_step3_device(ops, U, c, r, plan->cfg);
    if (history) history[s] = norm;
    int rc = check3("jr_newton_steps3d");
    if (rc) return rc;
  }
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_newton_steps3d");
  *cfl = c;
  *residual_norm = r;
  return check3("jr_newton_steps3d");
}

int jr_forces3d(jr_plan3d* plan, const double* U, double area, double length, const double* centre, double* out) {
  if (!plan || !U || !centre || !out) return report_error(JR_EINVAL, "null argument");
  if (!(area > 0.0) || !(length > 0.0)) return report_error(JR_EINVAL, "area and length must be positive");
  const int nw = plan->dev.n_walls;
  std::vector<double> loads((size_t)nw * 7);
  if (nw > 0) {
    launch_wall_loads3(plan->dev, U, plan->loads, plan->A, plan->st);
    cudaMemcpyAsync(loads.data(), plan->loads, loads.size() * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  }
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_forces3d");
  int rc = check3("jr_forces3d");
  if (rc) return rc;
  force_coefficients3(plan->dev.P, nw, loads.data(), plan->wall_mid.data(), area, length, centre, out);
  return JR_OK;
}

int jr_wall_loads3d(jr_plan3d* plan, const double* U, double* out) {
  if (!plan || !U || (!out && plan->dev.n_walls > 0)) return report_error(JR_EINVAL, "null argument");
  const int nw = plan->dev.n_walls;
  if (nw > 0) {
    launch_wall_loads3(plan->dev, U, plan->loads, plan->A, plan->st);
    cudaMemcpyAsync(out, plan->loads, (size_t)nw * 7 * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  }
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return check3("jr_wall_loads3d");
  return check3("jr_wall_loads3d");
}

int jr_time_kernels3d(jr_plan3d* plan, const double* U, int32_t reps, double* ms) {
  if (!plan || !U || !ms || reps < 1) return report_error(JR_EINVAL, "bad argument");
  const size_t N = (size_t)plan->dev.nvar * plan->n_canvas;
  double *v = nullptr, *out = nullptr;
  if (cudaMalloc(&v, N * sizeof(double)) != cudaSuccess || cudaMalloc(&out, N * sizeof(double)) != cudaSuccess) {
    cudaFree(v);
    return report_error(JR_ENOMEM, "cudaMalloc failed");
  }
  cudaMemcpyAsync(v, U, N * sizeof(double), cudaMemcpyDeviceToDevice, plan->st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto timed = [&](int k, auto&& launch) {
    launch();
    cudaEventRecord(e0, plan->st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, plan->st);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    ms[k] = (double)t / reps;
  };
  const double cfl = 25.0;
  timed(0, [&] { launch_residual3(plan->dev, U, out, plan->A, false, plan->st); });
  timed(1, [&] { launch_jvp3(plan->dev, U, v, out, plan->A, plan->st); });
  timed(2, [&] { launch_precondition3(plan->dev, U, cfl, v, out, plan->factor, plan->st); });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(plan->st);
  cudaFree(v);
  cudaFree(out);
  return check3("jr_time_kernels3d");
}

int jr_launches3d(int64_t* out) {
  if (!out) return report_error(JR_EINVAL, "null argument");
  *out = launches3();
  return JR_OK;
}

int jr_wall_distance3d(const double* points, int64_t n_points, const double* faces, int32_t n_faces, double* out) {
  if (n_points < 0 || n_faces < 0) return report_error(JR_EINVAL, "negative size");
  if ((n_points > 0 && (!points || !out)) || (n_faces > 0 && !faces)) return report_error(JR_EINVAL, "null argument");
  if (n_points == 0) return JR_OK;
  double* spheres = nullptr;
  if (n_faces > 0 && cudaMalloc(&spheres, (size_t)n_faces * 4 * sizeof(double)) != cudaSuccess)
    return report_error(JR_ENOMEM, "cudaMalloc failed");
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(spheres);
    return check3("jr_wall_distance3d");
  }
  launch_wall_distance3(points, n_points, faces, n_faces, spheres, out, st);
  int rc = check3("jr_wall_distance3d");
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == JR_OK) rc = check3("jr_wall_distance3d");
  cudaStreamDestroy(st);
  cudaFree(spheres);
  return rc;
}

}  // extern "C"
