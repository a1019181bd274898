// The C ABI: plans (device copies of a case's static tables, work buffers, solver
// state, a stream), the per-call entry points, and the Newton step as one CUDA graph.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/jaxrans_b200.h"
#include "device.cuh"

namespace jr {
// residual.cu
void launch_residual(const Canvas&, const Physics&, int visc, bool second, const double* U, const double* qg,
                     double* R, double* partial, cudaStream_t);
void launch_jvp(const Canvas&, const Physics&, int visc, const double* U, const double* qg, const double* V,
                const double* dqg, const double* vdt, double* w, const int* active, cudaStream_t);
void launch_ghosts(const Canvas&, const Physics&, bool dual, const double* U, const double* V, double* qg,
                   double* dqg, const int* active, cudaStream_t);
void launch_faces(const Canvas&, const Physics&, int visc, const double* U, double* lam, double* mflux,
                  double* dflux, cudaStream_t);
void launch_cells(const Canvas&, const Physics&, int visc, const double* U, const double* lam, const double* mflux,
                  const double* dflux, const Scalars*, double* vdt, double* dflow, double* dsa, cudaStream_t);
dim3 tile_grid(const Canvas&);
void configure_kernels();
// linesolve.cu
void launch_chain_factor(const Canvas&, const Physics&, bool sa, bool fp32, const double* U, const double* lam,
                         const double* mflux, const double* dflux, const double* dflow, const double* dsa, void* fflow,
                         void* fsa, void* scratch, cudaStream_t);
void configure_line_kernels(const Canvas&);
void launch_chain_apply(const Canvas&, bool sa, bool fp32, const void* fflow, const void* fsa, const double* r,
                        const double* scale, const int* skip, void* vout, bool vout_fp32, double* z, cudaStream_t);
// krylov.cu
void launch_gmres_init(Scalars*, const double* R, double* b, double* x, double* action, double* r, int n,
                       const double* tile_partial, int n_tiles, double volume_sum, double* history, Reduce,
                       cudaStream_t);
void launch_cycle_start(Scalars*, Config, cudaStream_t);
void launch_arnoldi_orth(Scalars*, const void* V, bool fp32, size_t ldv, int j, int m, double* w, int n, Reduce,
                         cudaStream_t);
void launch_lstsq(Scalars*, int m, cudaStream_t);
void launch_combine(const Scalars*, const void* V, bool fp32, size_t ldv, int m, const double* w, double* tmp,
                    double* action, int n, cudaStream_t);
void launch_cycle_end(Scalars*, double* x, const double* z, const double* b, const double* action, double* r, int n,
                      Reduce, cudaStream_t);
void launch_newton_update(Scalars*, const Canvas&, const Physics&, Config, double* U, const double* dU,
                          const double* action, const double* R, Reduce, cudaStream_t);
int reduce_blocks(int n);
// forces.cu
void launch_forces(const Canvas&, const Physics&, const double* U, const double* qg, double length, double cx0,
                   double cy0, double* out, cudaStream_t);

// V_j = scale * src, z = V_j: the Arnoldi step without a preconditioner
template <class TV>
__global__ void k_scale_copy(const double* src, const double* scale_ptr, const int* skip, TV* vout, double* z, int n) {
  if (skip != nullptr && *skip == 0) return;
  const double s = scale_ptr != nullptr ? *scale_ptr : 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x = s * src[i];
    if (vout != nullptr) {
      TV xv = TV(x);
      vout[i] = xv;
      x = double(xv);
    }
    z[i] = x;
  }
}
}  // namespace jr

using namespace jr;

static thread_local std::string g_error;

struct jr_plan {
  Canvas cv{};
  Physics P{};
  Config cfg{};
  int visc = 0;
  bool mixed = false;
  int m = 10;
  int n_vec = 0;     // nvar * NI * NJ
  int n_faces = 0;
  int n_tiles = 0;
  cudaStream_t st = nullptr;             // the stream work is issued on
  cudaStream_t owned_stream = nullptr;   // the plan's own stream
  std::vector<void*> allocs;
  double *U = nullptr, *qg = nullptr, *dqg = nullptr, *R = nullptr, *b = nullptr, *x = nullptr, *action = nullptr;
  double *r = nullptr, *w = nullptr, *z = nullptr, *tmp = nullptr, *zero = nullptr, *vdt = nullptr;
  double *dflow = nullptr, *dsa = nullptr, *lam = nullptr, *mflux = nullptr, *dflux = nullptr;
  double *tile_partial = nullptr, *history = nullptr, *force_out = nullptr;
  void *V = nullptr, *fflow = nullptr, *fsa = nullptr, *scratch = nullptr;
  Scalars* sc = nullptr;
  Reduce red{};
  int hist_cap = 0;
  cudaGraphExec_t graph = nullptr;
  double force_length = 1.0, cx0 = 0.25, cy0 = 0.0;
};

static int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

static int cuda_check(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(JR_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
  return JR_OK;
}

template <class T> static int dev_copy(jr_plan* p, T** dst, const T* src, size_t n) {
  *dst = nullptr;
  if (n == 0) return JR_OK;
  if (cudaMalloc((void**)dst, n * sizeof(T)) != cudaSuccess) return fail(JR_ENOMEM, "cudaMalloc failed");
  p->allocs.push_back(*dst);
  if (src != nullptr && cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(JR_ECUDA, "cudaMemcpy to the device failed");
  if (src == nullptr) cudaMemset(*dst, 0, n * sizeof(T));
  return JR_OK;
}

static int dev_alloc(jr_plan* p, void** dst, size_t bytes) {
  if (cudaMalloc(dst, bytes) != cudaSuccess) return fail(JR_ENOMEM, "cudaMalloc failed");
  p->allocs.push_back(*dst);
  cudaMemset(*dst, 0, bytes);
  return JR_OK;
}

#define TRY(x)                \
  do {                        \
    int _rc = (x);            \
    if (_rc != JR_OK) {       \
      jr_plan_destroy(plan);  \
      return _rc;             \
    }                         \
  } while (0)

// The launch sequence of one Newton step on the plan's state (captured as a graph).
static void enqueue_step(jr_plan* p) {
  const Canvas& c = p->cv;
  const int n = p->n_vec, N = c.NI * c.NJ, m = p->m;
  const bool sa = c.nvar == 5;
  const size_t ldv = (size_t)n;
  cudaStream_t st = p->st;
  launch_ghosts(c, p->P, false, p->U, nullptr, p->qg, nullptr, nullptr, st);
  launch_residual(c, p->P, p->visc, true, p->U, p->qg, p->R, p->tile_partial, st);
  launch_gmres_init(p->sc, p->R, p->b, p->x, p->action, p->r, n, p->tile_partial, p->n_tiles, c.volume_sum,
                    p->history, p->red, st);
  launch_faces(c, p->P, p->visc, p->U, p->lam, p->mflux, p->dflux, st);
  launch_cells(c, p->P, p->visc, p->U, p->lam, p->mflux, p->dflux, p->sc, p->vdt, p->dflow, p->dsa, st);
  if (p->cfg.preconditioner == 1)
    launch_chain_factor(c, p->P, sa, p->mixed, p->U, p->lam, p->mflux, p->dflux, p->dflow, p->dsa, p->fflow, p->fsa,
                        p->scratch, st);
  const size_t vbytes = p->mixed ? sizeof(float) : sizeof(double);
  for (int cyc = 0; cyc < p->cfg.maxiter; ++cyc) {
    launch_cycle_start(p->sc, p->cfg, st);
    for (int j = 0; j < m; ++j) {
      const double* src = j == 0 ? p->r : p->w;
      void* vj = (char*)p->V + (size_t)j * ldv * vbytes;
      if (p->cfg.preconditioner == 1) {
        launch_chain_apply(c, sa, p->mixed, p->fflow, p->fsa, src, &p->sc->inv_nrm, &p->sc->active, vj, p->mixed,
                           p->z, st);
      } else {
        int blocks = std::min((n + 255) / 256, 148 * 4);
        if (p->mixed)
          k_scale_copy<float><<<blocks, 256, 0, st>>>(src, &p->sc->inv_nrm, &p->sc->active, (float*)vj, p->z, n);
        else
          k_scale_copy<double><<<blocks, 256, 0, st>>>(src, &p->sc->inv_nrm, &p->sc->active, (double*)vj, p->z, n);
      }
      launch_ghosts(c, p->P, true, p->U, p->z, p->qg, p->dqg, &p->sc->active, st);
      launch_jvp(c, p->P, p->visc, p->U, p->qg, p->z, p->dqg, p->vdt, p->w, &p->sc->active, st);
      launch_arnoldi_orth(p->sc, p->V, p->mixed, ldv, j, m, p->w, n, p->red, st);
    }
    launch_lstsq(p->sc, m, st);
    launch_combine(p->sc, p->V, p->mixed, ldv, m, p->w, p->tmp, p->action, n, st);
    if (p->cfg.preconditioner == 1) {
      launch_chain_apply(c, sa, p->mixed, p->fflow, p->fsa, p->tmp, nullptr, &p->sc->active, nullptr, false, p->z, st);
    } else {
      int blocks = std::min((n + 255) / 256, 148 * 4);
      k_scale_copy<double><<<blocks, 256, 0, st>>>(p->tmp, nullptr, &p->sc->active, nullptr, p->z, n);
    }
    launch_cycle_end(p->sc, p->x, p->z, p->b, p->action, p->r, n, p->red, st);
  }
  launch_newton_update(p->sc, c, p->P, p->cfg, p->U, p->x, p->action, p->R, p->red, st);
  (void)N;
}

extern "C" {

const char* jr_last_error(void) { return g_error.c_str(); }

int jr_plan_destroy(jr_plan* plan) {
  if (plan == nullptr) return JR_OK;
  if (plan->graph) cudaGraphExecDestroy(plan->graph);
  if (plan->st) cudaStreamSynchronize(plan->st);
  for (void* a : plan->allocs) cudaFree(a);
  if (plan->owned_stream) cudaStreamDestroy(plan->owned_stream);
  delete plan;
  return JR_OK;
}

int jr_plan_create(const jr_plan_desc* d, jr_plan** out) {
  if (d == nullptr || out == nullptr) return fail(JR_EINVAL, "null argument");
  *out = nullptr;
  if (d->NI < 5 || d->NJ < 5 || (d->nvar != 4 && d->nvar != 5))
    return fail(JR_EINVAL, "canvas must be at least 5 x 5 with nvar 4 or 5");
  if (d->krylov_subspace < 1 || d->krylov_subspace > MAX_KRYLOV)
    return fail(JR_EINVAL, "krylov_subspace must lie in [1, 64]");
  if (d->nvar == 5 && d->distance == nullptr) return fail(JR_EINVAL, "the SA model needs the wall distance");
  if (d->far_field == 1 && d->nvar == 4 && false) return fail(JR_EINVAL, "unreachable");
  jr_plan* plan = new jr_plan();
  const int NI = d->NI, NJ = d->NJ, N = NI * NJ, nv = d->nvar;
  const size_t nfi = (size_t)(NI + 1) * NJ, nfj = (size_t)NI * (NJ + 1);
  plan->n_vec = nv * N;
  plan->n_faces = (int)(nfi + nfj);
  plan->m = d->krylov_subspace;
  plan->mixed = d->precision == 1;
  if (cudaStreamCreateWithFlags(&plan->owned_stream, cudaStreamNonBlocking) == cudaSuccess) plan->st = plan->owned_stream;
  if (plan->st == nullptr) {
    delete plan;
    return fail(JR_ECUDA, "cudaStreamCreate failed");
  }
  Canvas& c = plan->cv;
  c.NI = NI;
  c.NJ = NJ;
  c.nvar = nv;
  TRY(dev_copy(plan, (uint8_t**)&c.interior, d->interior, (size_t)N));
  TRY(dev_copy(plan, (double**)&c.volume, d->volume, (size_t)N));
  TRY(dev_copy(plan, (double**)&c.fi, d->faces_i, 2 * nfi));
  TRY(dev_copy(plan, (double**)&c.fj, d->faces_j, 2 * nfj));
  TRY(dev_copy(plan, (double**)&c.centres, d->centres, (size_t)2 * (NI + 2) * (NJ + 2)));
  if (d->distance) TRY(dev_copy(plan, (double**)&c.distance, d->distance, (size_t)N));
  TRY(dev_copy(plan, (int**)&c.neighbours, d->neighbours, (size_t)N));
  int cells = 0;
  double vsum = 0.0;
  for (int k = 0; k < N; ++k)
    if (d->interior[k]) {
      ++cells;
      vsum += d->volume[k];
    }
  c.n_cells = cells;
  c.volume_sum = vsum;
  for (int s = 0; s < 2; ++s) {
    int n = d->n_ghost[s];
    c.n_ghost[s] = n;
    for (int k = 0; k < n; ++k)
      if (d->ghost[s][k] < 0 || d->ghost[s][k] >= N || d->source[s][k] < 0 || d->source[s][k] >= N ||
          d->kind[s][k] < 0 || d->kind[s][k] > 6) {
        jr_plan_destroy(plan);
        return fail(JR_EINVAL, "a ghost record out of range");
      }
    TRY(dev_copy(plan, (int**)&c.g_ghost[s], d->ghost[s], (size_t)n));
    TRY(dev_copy(plan, (int**)&c.g_source[s], d->source[s], (size_t)n));
    TRY(dev_copy(plan, (int**)&c.g_kind[s], d->kind[s], (size_t)n));
    TRY(dev_copy(plan, (double**)&c.g_geom[s], d->geom[s], (size_t)4 * n));
  }
  {
    // stage 2 reads stage-1 ghosts at the corners: which stage-1 record fills each source
    std::vector<int> rec_of(N, -1), src_rec(d->n_ghost[1], -1);
    for (int k = 0; k < d->n_ghost[0]; ++k) rec_of[d->ghost[0][k]] = k;
    for (int k = 0; k < d->n_ghost[1]; ++k)
      if (!d->interior[d->source[1][k]]) src_rec[k] = rec_of[d->source[1][k]];
    TRY(dev_copy(plan, (int**)&c.g_src_rec, src_rec.data(), src_rec.size()));
  }
  c.n_walls = d->n_walls;
  TRY(dev_copy(plan, (int**)&c.w_cell, d->wall_cell, (size_t)d->n_walls));
  TRY(dev_copy(plan, (int**)&c.w_family, d->wall_family, (size_t)d->n_walls));
  TRY(dev_copy(plan, (int**)&c.w_face, d->wall_face, (size_t)d->n_walls));
  TRY(dev_copy(plan, (double**)&c.w_into, d->wall_into, (size_t)d->n_walls));
  TRY(dev_copy(plan, (double**)&c.w_mid, d->wall_mid, (size_t)2 * d->n_walls));
  const int nc = d->n_chains, L = d->chain_L;
  c.n_chains = nc;
  c.L = L;
  std::vector<int> on_chain(N, 0);
  for (size_t k = 0; k < (size_t)nc * L; ++k) {
    int cell = d->chain_cells[k];
    if (cell >= N) {
      jr_plan_destroy(plan);
      return fail(JR_EINVAL, "a chain cell out of range");
    }
    if (cell >= 0) on_chain[cell] = 1;
  }
  std::vector<int> off;
  for (int k = 0; k < N; ++k)
    if (!on_chain[k]) off.push_back(k);
  c.n_offchain = (int)off.size();
  TRY(dev_copy(plan, (int**)&c.offchain, off.data(), off.size()));
  TRY(dev_copy(plan, (int**)&c.ch_cells, d->chain_cells, (size_t)nc * L));
  TRY(dev_copy(plan, (int**)&c.ch_len, d->chain_len, (size_t)nc));
  TRY(dev_copy(plan, (int**)&c.ch_up_face, d->chain_up_face, (size_t)nc * L));
  TRY(dev_copy(plan, (int**)&c.ch_up_sign, d->chain_up_sign, (size_t)nc * L));
  TRY(dev_copy(plan, (int**)&c.ch_down_face, d->chain_down_face, (size_t)nc * L));
  TRY(dev_copy(plan, (int**)&c.ch_down_sign, d->chain_down_sign, (size_t)nc * L));
  if (L > 1024) {
    jr_plan_destroy(plan);
    return fail(JR_EINVAL, "line chains longer than 1024 cells are not supported");
  }
  std::vector<int> fbase(nc);
  size_t fbase_total = 0;
  for (int k = 0; k < nc; ++k) {
    fbase[k] = (int)fbase_total;
    fbase_total += (size_t)d->chain_len[k] + 16;
  }
  TRY(dev_copy(plan, (int**)&c.ch_fbase, fbase.data(), (size_t)nc));

  Physics& P = plan->P;
  P.gamma = d->gamma;
  P.mu_inf = d->mu_inf;
  P.sutherland = d->sutherland;
  P.c_cr1 = d->c_cr1;
  P.kappa = d->kappa;
  P.flux = d->flux;
  P.limiter = d->limiter;
  P.nvar = nv;
  P.far_field = d->far_field;
  for (int k = 0; k < 5; ++k) P.q_inf[k] = k < nv ? d->q_inf[k] : 0.0;
  {
    double g = d->gamma, rho = P.q_inf[0], u = P.q_inf[1], v = P.q_inf[2], p = P.q_inf[3];
    P.U_inf[0] = rho;
    P.U_inf[1] = rho * u;
    P.U_inf[2] = rho * v;
    P.U_inf[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
    P.U_inf[4] = rho * P.q_inf[4];
  }
  P.quarter_chord[0] = d->quarter_chord[0];
  P.quarter_chord[1] = d->quarter_chord[1];
  SAConst& s = P.sa;
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
  plan->visc = d->mu_inf > 0.0 ? (nv == 5 ? 2 : 1) : 0;
  if (nv == 5 && plan->visc != 2) {
    jr_plan_destroy(plan);
    return fail(JR_EINVAL, "the SA model needs a viscous flow");
  }

  Config& cf = plan->cfg;
  cf.cfl_max = d->cfl_max;
  cf.cfl_growth = d->cfl_growth;
  cf.cfl_cutback = d->cfl_cutback;
  cf.cfl_min = d->cfl_min;
  cf.krylov_tol = d->krylov_tol;
  cf.krylov_success = d->krylov_success;
  cf.max_relative_update = d->max_relative_update;
  cf.restart = d->krylov_subspace;
  cf.maxiter = d->krylov_restarts;
  cf.preconditioner = d->preconditioner;
  plan->force_length = d->force_length;
  plan->cx0 = d->moment_centre[0];
  plan->cy0 = d->moment_centre[1];

  const size_t vec = (size_t)plan->n_vec;
  double** vecs[] = {&plan->U, &plan->qg, &plan->dqg, &plan->R, &plan->b, &plan->x, &plan->action,
                     &plan->r, &plan->w, &plan->z, &plan->tmp};
  for (double** v : vecs) TRY(dev_copy<double>(plan, v, nullptr, vec));
  TRY(dev_copy<double>(plan, &plan->zero, nullptr, (size_t)N));
  TRY(dev_copy<double>(plan, &plan->vdt, nullptr, (size_t)N));
  TRY(dev_copy<double>(plan, &plan->dflow, nullptr, (size_t)N));
  TRY(dev_copy<double>(plan, &plan->dsa, nullptr, (size_t)N));
  TRY(dev_copy<double>(plan, &plan->lam, nullptr, nfi + nfj));
  TRY(dev_copy<double>(plan, &plan->mflux, nullptr, nfi + nfj));
  TRY(dev_copy<double>(plan, &plan->dflux, nullptr, nfi + nfj));
  dim3 tg = tile_grid(c);
  plan->n_tiles = (int)(tg.x * tg.y);
  TRY(dev_copy<double>(plan, &plan->tile_partial, nullptr, (size_t)plan->n_tiles));
  plan->hist_cap = 4096;
  TRY(dev_copy<double>(plan, &plan->history, nullptr, (size_t)plan->hist_cap));
  TRY(dev_copy<double>(plan, &plan->force_out, nullptr, 8));
  const size_t tb = plan->mixed ? sizeof(float) : sizeof(double);
  TRY(dev_alloc(plan, &plan->V, (size_t)(plan->m + 1) * vec * tb));
  // cyclic-reduction factor: per chain at most 80 (flow) and 5 (SA) entries per row of
  // (length + 16) rows; the level systems in scratch at most 104 per row
  TRY(dev_alloc(plan, &plan->fflow, fbase_total * 80 * tb));
  TRY(dev_alloc(plan, &plan->fsa, fbase_total * 5 * tb));
  TRY(dev_alloc(plan, &plan->scratch, fbase_total * 104 * tb));
  TRY(dev_alloc(plan, (void**)&plan->sc, sizeof(Scalars)));
  int rb = reduce_blocks(plan->n_vec);
  plan->red.blocks = rb;
  TRY(dev_alloc(plan, (void**)&plan->red.partial, (size_t)rb * (MAX_KRYLOV + 1) * sizeof(double)));
  TRY(dev_alloc(plan, (void**)&plan->red.ticket, sizeof(unsigned)));
  configure_kernels();
  configure_line_kernels(c);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    int rc = cuda_check("plan create");
    jr_plan_destroy(plan);
    return rc ? rc : fail(JR_ECUDA, "plan create");
  }
  // the freestream state, CFL and |R| = inf
  std::vector<double> U0((size_t)plan->n_vec);
  for (int v = 0; v < nv; ++v)
    for (int k = 0; k < N; ++k) U0[(size_t)v * N + k] = P.U_inf[v];
  int rc = jr_state_set(plan, U0.data(), d->cfl, INFINITY);
  if (rc) {
    jr_plan_destroy(plan);
    return rc;
  }
  *out = plan;
  return JR_OK;
}

int jr_plan_sizes(const jr_plan* plan, int64_t* n_canvas, int64_t* n_faces) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (n_canvas) *n_canvas = (int64_t)plan->cv.NI * plan->cv.NJ;
  if (n_faces) *n_faces = plan->n_faces;
  return JR_OK;
}

void* jr_plan_stream(jr_plan* plan) { return plan ? (void*)plan->st : nullptr; }

int jr_plan_set_stream(jr_plan* plan, void* stream) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_plan_set_stream");
  if (plan->owned_stream && plan->st != plan->owned_stream) {
    // a caller's stream was in use: nothing to release
  }
  plan->st = stream != nullptr ? (cudaStream_t)stream : plan->owned_stream;
  return JR_OK;
}

int jr_synchronize(jr_plan* plan) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("synchronize");
  return JR_OK;
}

int jr_residual(jr_plan* plan, const double* U, double* R, int first_order) {
  if (!plan || !U || !R) return fail(JR_EINVAL, "null argument");
  launch_ghosts(plan->cv, plan->P, false, U, nullptr, plan->qg, nullptr, nullptr, plan->st);
  launch_residual(plan->cv, plan->P, plan->visc, first_order == 0, U, plan->qg, R, plan->tile_partial, plan->st);
  return cuda_check("jr_residual");
}

int jr_jvp(jr_plan* plan, const double* U, const double* v, double* Jv) {
  if (!plan || !U || !v || !Jv) return fail(JR_EINVAL, "null argument");
  launch_ghosts(plan->cv, plan->P, false, U, nullptr, plan->qg, nullptr, nullptr, plan->st);
  launch_ghosts(plan->cv, plan->P, true, U, v, plan->qg, plan->dqg, nullptr, plan->st);
  launch_jvp(plan->cv, plan->P, plan->visc, U, plan->qg, v, plan->dqg, plan->zero, Jv, nullptr, plan->st);
  return cuda_check("jr_jvp");
}

int jr_wave_speeds(jr_plan* plan, const double* U, double* lam) {
  if (!plan || !U || !lam) return fail(JR_EINVAL, "null argument");
  launch_faces(plan->cv, plan->P, plan->visc, U, lam, plan->mflux, plan->dflux, plan->st);
  return cuda_check("jr_wave_speeds");
}

int jr_precond_factor(jr_plan* plan, const double* U, double cfl) {
  if (!plan || !U) return fail(JR_EINVAL, "null argument");
  if (!(cfl > 0.0)) return fail(JR_EINVAL, "cfl must be positive");
  cudaMemcpyAsync(&plan->sc->cfl, &cfl, sizeof(double), cudaMemcpyHostToDevice, plan->st);
  cudaStreamSynchronize(plan->st);
  launch_faces(plan->cv, plan->P, plan->visc, U, plan->lam, plan->mflux, plan->dflux, plan->st);
  launch_cells(plan->cv, plan->P, plan->visc, U, plan->lam, plan->mflux, plan->dflux, plan->sc, plan->vdt,
               plan->dflow, plan->dsa, plan->st);
  launch_chain_factor(plan->cv, plan->P, plan->cv.nvar == 5, plan->mixed, U, plan->lam, plan->mflux, plan->dflux,
                      plan->dflow, plan->dsa, plan->fflow, plan->fsa, plan->scratch, plan->st);
  return cuda_check("jr_precond_factor");
}

int jr_precond_apply(jr_plan* plan, const double* r, double* z) {
  if (!plan || !r || !z) return fail(JR_EINVAL, "null argument");
  launch_chain_apply(plan->cv, plan->cv.nvar == 5, plan->mixed, plan->fflow, plan->fsa, r, nullptr, nullptr, nullptr,
                     false, z, plan->st);
  return cuda_check("jr_precond_apply");
}

int jr_state_set(jr_plan* plan, const double* U_host, double cfl, double residual_norm) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (U_host)
    cudaMemcpyAsync(plan->U, U_host, (size_t)plan->n_vec * sizeof(double), cudaMemcpyHostToDevice, plan->st);
  Scalars s{};
  s.cfl = cfl;
  s.res_prev = residual_norm;
  cudaMemcpyAsync(plan->sc, &s, sizeof(Scalars), cudaMemcpyHostToDevice, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_state_set");
  return cuda_check("jr_state_set");
}

int jr_state_get(jr_plan* plan, double* U_host, double* cfl, double* residual_norm, int32_t* status) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (U_host)
    cudaMemcpyAsync(U_host, plan->U, (size_t)plan->n_vec * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  Scalars s;
  cudaMemcpyAsync(&s, plan->sc, sizeof(Scalars), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_state_get");
  if (cfl) *cfl = s.cfl;
  if (residual_norm) *residual_norm = s.res_prev;
  if (status) *status = s.status;
  return cuda_check("jr_state_get");
}

double* jr_state_device(jr_plan* plan) { return plan ? plan->U : nullptr; }

int jr_state_set_device(jr_plan* plan, const double* U_device, double cfl, double residual_norm) {
  if (!plan || !U_device) return fail(JR_EINVAL, "null argument");
  cudaMemcpyAsync(plan->U, U_device, (size_t)plan->n_vec * sizeof(double), cudaMemcpyDeviceToDevice, plan->st);
  Scalars s{};
  s.cfl = cfl;
  s.res_prev = residual_norm;
  static thread_local Scalars staged;
  staged = s;
  cudaMemcpyAsync(plan->sc, &staged, sizeof(Scalars), cudaMemcpyHostToDevice, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_state_set_device");
  return cuda_check("jr_state_set_device");
}

static int ensure_graph(jr_plan* plan);

int jr_graph_kernels(jr_plan* plan, int64_t* kernels_per_step) {
  if (!plan || !kernels_per_step) return fail(JR_EINVAL, "null argument");
  cudaGraph_t g;
  if (cudaStreamBeginCapture(plan->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return cuda_check("begin capture");
  enqueue_step(plan);
  if (cudaStreamEndCapture(plan->st, &g) != cudaSuccess) return cuda_check("end capture");
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  std::vector<cudaGraphNode_t> nodes(n);
  cudaGraphGetNodes(g, nodes.data(), &n);
  int64_t kernels = 0;
  for (auto node : nodes) {
    cudaGraphNodeType t;
    cudaGraphNodeGetType(node, &t);
    if (t == cudaGraphNodeTypeKernel) ++kernels;
  }
  cudaGraphDestroy(g);
  *kernels_per_step = kernels;
  return cuda_check("jr_graph_kernels");
}

static int ensure_graph(jr_plan* plan) {
  if (plan->graph) return JR_OK;
  cudaGraph_t g;
  if (cudaStreamBeginCapture(plan->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return cuda_check("begin capture");
  enqueue_step(plan);
  if (cudaStreamEndCapture(plan->st, &g) != cudaSuccess) return cuda_check("end capture");
  if (cudaGraphInstantiate(&plan->graph, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_check("graph instantiate");
  }
  cudaGraphDestroy(g);
  return cuda_check("graph");
}

int jr_newton_steps_async(jr_plan* plan, int32_t n_steps, double* history_device) {
  if (!plan || n_steps < 0) return fail(JR_EINVAL, "bad argument");
  if (n_steps > plan->hist_cap) return fail(JR_EINVAL, "at most 4096 steps per call");
  int rc = ensure_graph(plan);
  if (rc) return rc;
  // the history position restarts at 0 for this call
  cudaMemsetAsync(&plan->sc->hpos, 0, sizeof(int), plan->st);
  for (int k = 0; k < n_steps; ++k)
    if (cudaGraphLaunch(plan->graph, plan->st) != cudaSuccess) return cuda_check("graph launch");
  if (history_device && n_steps > 0)
    cudaMemcpyAsync(history_device, plan->history, (size_t)n_steps * sizeof(double), cudaMemcpyDeviceToDevice,
                    plan->st);
  return cuda_check("jr_newton_steps");
}

int jr_newton_steps(jr_plan* plan, int32_t n_steps, double* history) {
  int rc = jr_newton_steps_async(plan, n_steps, nullptr);
  if (rc) return rc;
  if (history && n_steps > 0)
    cudaMemcpyAsync(history, plan->history, (size_t)n_steps * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_newton_steps");
  return cuda_check("jr_newton_steps");
}

int jr_time_kernels(jr_plan* plan, int32_t reps, double* ms) {
  if (!plan || !ms || reps < 1) return fail(JR_EINVAL, "bad argument");
  jr_plan* p = plan;
  const Canvas& c = p->cv;
  const bool sa = c.nvar == 5;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // a consistent state for every kernel: base ghosts, wave speeds, the factor, an
  // active Krylov cycle with z = the residual
  launch_ghosts(c, p->P, false, p->U, nullptr, p->qg, nullptr, nullptr, p->st);
  launch_residual(c, p->P, p->visc, true, p->U, p->qg, p->R, p->tile_partial, p->st);
  launch_faces(c, p->P, p->visc, p->U, p->lam, p->mflux, p->dflux, p->st);
  launch_cells(c, p->P, p->visc, p->U, p->lam, p->mflux, p->dflux, p->sc, p->vdt, p->dflow, p->dsa, p->st);
  launch_chain_factor(c, p->P, sa, p->mixed, p->U, p->lam, p->mflux, p->dflux, p->dflow, p->dsa, p->fflow, p->fsa,
                      p->scratch, p->st);
  cudaMemcpyAsync(p->z, p->R, (size_t)p->n_vec * sizeof(double), cudaMemcpyDeviceToDevice, p->st);
  int one = 1;
  cudaMemcpyAsync(&p->sc->active, &one, sizeof(int), cudaMemcpyHostToDevice, p->st);
  cudaStreamSynchronize(p->st);
  auto timed = [&](int k, auto&& launch) {
    launch();
    cudaEventRecord(e0, p->st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, p->st);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    ms[k] = (double)t / reps;
  };
  timed(0, [&] { launch_residual(c, p->P, p->visc, true, p->U, p->qg, p->R, p->tile_partial, p->st); });
  timed(1, [&] { launch_jvp(c, p->P, p->visc, p->U, p->qg, p->z, p->dqg, p->vdt, p->w, nullptr, p->st); });
  timed(2, [&] { launch_ghosts(c, p->P, true, p->U, p->z, p->qg, p->dqg, nullptr, p->st); });
  timed(3, [&] {
    launch_chain_apply(c, sa, p->mixed, p->fflow, p->fsa, p->R, nullptr, nullptr, nullptr, false, p->tmp, p->st);
  });
  timed(4, [&] {
    launch_chain_factor(c, p->P, sa, p->mixed, p->U, p->lam, p->mflux, p->dflux, p->dflow, p->dsa, p->fflow, p->fsa,
                        p->scratch, p->st);
  });
  timed(5, [&] { launch_arnoldi_orth(p->sc, p->V, p->mixed, (size_t)p->n_vec, p->m - 1, p->m, p->w, p->n_vec,
                                     p->red, p->st); });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cuda_check("jr_time_kernels");
}

int jr_forces(jr_plan* plan, const double* U, double* out) {
  if (!plan || !out) return fail(JR_EINVAL, "null argument");
  const double* u = U ? U : plan->U;
  launch_ghosts(plan->cv, plan->P, false, u, nullptr, plan->qg, nullptr, nullptr, plan->st);
  launch_forces(plan->cv, plan->P, u, plan->qg, plan->force_length, plan->cx0, plan->cy0, plan->force_out, plan->st);
  cudaMemcpyAsync(out, plan->force_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_forces");
  return cuda_check("jr_forces");
}

}  // extern "C"
