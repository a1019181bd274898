// The C ABI: plans (a batch of cases: device copies of each case's static tables, work
// buffers and solver state, one stream), the per-call entry points, and the Newton step
// of every case of the batch as one CUDA graph.  A single case is a batch of one.
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/jaxrans_b200.h"
#include "device.cuh"

namespace jr {
static_assert(JR_STATUS_NONFINITE == ST_NONFINITE && JR_STATUS_REJECTED == ST_REJECTED &&
                  JR_STATUS_GMRES_BREAKDOWN == ST_GMRES_BREAKDOWN && JR_STATUS_WAIT_LIMIT == ST_STAGE_FAILED,
              "the status bits of the C ABI are the device's");
// residual.cu
void launch_residual(const CaseDev*, const BatchDims&, int visc, bool second, int out_id, cudaStream_t);
void launch_jvp(const CaseDev*, const BatchDims&, int visc, bool fp32, int tangent_id, int vdt_id, int out_id,
                int check_active, int own_ghosts, cudaStream_t);
void launch_ghosts(const CaseDev*, const BatchDims&, int tangent_id, int check_active, cudaStream_t);
void launch_linearize(const CaseDev*, const BatchDims&, int visc, bool fp32, cudaStream_t);
int jac_coefficients(int visc);
int jac_cell_coefficients(int visc);
void launch_faces(const CaseDev*, const BatchDims&, int visc, cudaStream_t);
void launch_cells(const CaseDev*, const BatchDims&, int visc, cudaStream_t);
dim3 tile_grid(const Canvas&);
void configure_kernels();
// linesolve.cu
void launch_chain_factor(const CaseDev*, const BatchDims&, bool sa, bool fp32, cudaStream_t);
void launch_chain_apply(const CaseDev*, const BatchDims&, bool sa, bool fp32, int src_id, int scale_on, int vout_j,
                        int out_id, int check_active, cudaStream_t);
int chain_grid_blocks(int n_chains, int n_offchain);
bool apply_threads_valid(int threads, int max_L);
bool apply_stage_fits(int max_L, bool fp32, int stage);
int wait_limit_check(int tries, int* status, cudaStream_t st);
void configure_line_kernels(int max_L);
void launch_chain_couple(const CaseDev*, const BatchDims&, bool fp32, int out_id, int check_active, cudaStream_t);
// krylov.cu
void launch_gmres_init(const CaseDev*, const BatchDims&, cudaStream_t);
void launch_cycle_start(const CaseDev*, const BatchDims&, cudaStream_t);
void launch_cycle_gate(const CaseDev*, const BatchDims&, cudaGraphConditionalHandle, unsigned long long*,
                       cudaStream_t);
void launch_arnoldi_orth(const CaseDev*, const BatchDims&, bool fp32, int j, cudaStream_t);
void launch_lstsq(const CaseDev*, const BatchDims&, cudaStream_t);
void launch_combine(const CaseDev*, const BatchDims&, bool fp32, cudaStream_t);
void launch_cycle_end(const CaseDev*, const BatchDims&, cudaStream_t);
void launch_scale_copy(const CaseDev*, const BatchDims&, bool fp32, int src_id, int scale_on, int vout_j, int out_id,
                       int check_active, cudaStream_t);
void launch_newton_update(const CaseDev*, const BatchDims&, cudaStream_t);
int reduce_blocks(int n);
// forces.cu
void launch_forces(const CaseDev*, const BatchDims&, cudaStream_t);
void launch_monitor(CaseDev* cases, int n_live, int n_slots, int step0, int block_iters, cudaStream_t st);
void launch_norm(const CaseDev* cases, int n_cases, int variable, double* out, cudaStream_t st);
}  // namespace jr

using namespace jr;

static thread_local std::string g_error;

constexpr int MAX_CHAIN = 1024;   // longest line chain (one CTA of the line solve)
constexpr int HIST_STEPS = 4096;  // Newton steps per jr_newton_steps call

struct jr_plan {
  int n_cases = 0;
  int nvar = 4, visc = 0, m = 10;
  bool mixed = false;
  Config cfg{};                          // the settings every case shares (restart, restarts, preconditioner)
  BatchDims dims{};
  std::vector<CaseDev> host;             // the resident case table (host copy)
  CaseDev* cases = nullptr;              // ... on the device: the graph's table
  CaseDev* adhoc = nullptr;              // the table of a call on caller buffers
  std::vector<size_t> vec_off, can_off, face_off, wall_off;   // offsets of each case in batch-long arrays
  size_t total_vec = 0, total_can = 0, total_faces = 0, total_walls = 0;
  double* wall_out = nullptr;            // 5 per wall face, every case
  cudaStream_t st = nullptr;             // the stream work is issued on
  cudaStream_t owned_stream = nullptr;   // the plan's own stream
  std::vector<void*> allocs;
  double* U = nullptr;                   // every case's state, back to back
  double* history = nullptr;             // [step][case]
  double* force_out = nullptr;           // 8 per case
  double* norm_out = nullptr;            // 1 per case (jr_norm)
  Scalars* sc = nullptr;                 // one per case
  Monitor* mon = nullptr;                // one per case: the exit test on the device
  cudaGraphExec_t graph = nullptr;
  int device = 0;                        // the device current when the plan was made
  // the step graph runs over the enabled cases only: their descriptors packed in slot
  // order (`live`) and the launch extents over them; rebuilt, with the graph, whenever
  // a case is enabled, disabled or changed
  CaseDev* live = nullptr;
  BatchDims live_dims{};
  cudaStream_t body_st = nullptr;        // captures the bodies of the conditional cycles
  unsigned long long* cycles = nullptr;  // Krylov cycle bodies run (device counter)
  int64_t steps_run = 0;                 // Newton steps launched
  int64_t kernels_outside = 0;           // kernels of a step outside the cycle bodies
  int64_t kernels_per_cycle = 0;         // kernels of one cycle body
  int64_t launched = 0;                  // kernels launched by steps of earlier graphs
  int64_t steps_since = 0;               // steps of the current graph
  unsigned long long cycles_base = 0;    // the cycle counter when the current graph was made
  int n_live = 0;
  bool live_dirty = true;
  bool live_vortex = false;              // an enabled case uses the point-vortex far field
  std::vector<std::vector<int>> chain_len;   // each case's chain lengths (host copy)
  int ls_factor_threads = 128, ls_apply_threads = 128;   // the line-solve schedule in use
  int ls_apply_stage = 0;                                // s >= 1: the solve stages its factor
  const double* factor_U = nullptr;      // the state of the last jr_precond_factor (the coupled form's)
};

static int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

namespace jr {
// shared with the 3D entry points (capi3d.cu)
int report_error(int code, const std::string& msg) { return fail(code, msg); }

}  // namespace jr

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
  *dst = nullptr;
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(dst, bytes) != cudaSuccess) return fail(JR_ENOMEM, "cudaMalloc failed");
  p->allocs.push_back(*dst);
  cudaMemset(*dst, 0, bytes);
  return JR_OK;
}

#define TRY(x)               \
  do {                       \
    int _rc = (x);           \
    if (_rc != JR_OK) return _rc; \
  } while (0)

// A table of a case: allocated and filled for a new case, or overwritten in place when a
// slot takes a new case of the same shape (`reload`).
template <class T> static int put(jr_plan* p, T** dst, const T* src, size_t n, bool reload) {
  if (!reload) return dev_copy(p, dst, src, n);
  if (n == 0) return JR_OK;
  if (*dst == nullptr) return fail(JR_EMISMATCH, "the slot has no such table");
  if (cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(JR_ECUDA, "cudaMemcpy to the device failed");
  return JR_OK;
}

// Static tables, physics and solver settings of one case (the work buffers come later).
static int build_case(jr_plan* plan, const jr_plan_desc* d, CaseDev& cd, size_t& factor_rows,
                      bool reload = false) {
  if (d->NI < 5 || d->NJ < 5 || (d->nvar != 4 && d->nvar != 5))
    return fail(JR_EINVAL, "canvas must be at least 5 x 5 with nvar 4 or 5");
  if (d->krylov_subspace < 1 || d->krylov_subspace > MAX_KRYLOV)
    return fail(JR_EINVAL, "krylov_subspace must lie in [1, 64]");
  if (d->nvar == 5 && d->distance == nullptr) return fail(JR_EINVAL, "the SA model needs the wall distance");
  const int NI = d->NI, NJ = d->NJ, N = NI * NJ, nv = d->nvar;
  const size_t nfi = (size_t)(NI + 1) * NJ, nfj = (size_t)NI * (NJ + 1);
  Canvas& c = cd.c;
  c.NI = NI;
  c.NJ = NJ;
  c.nvar = nv;
  TRY(put(plan, (uint8_t**)&c.interior, d->interior, (size_t)N, reload));
  TRY(put(plan, (double**)&c.volume, d->volume, (size_t)N, reload));
  TRY(put(plan, (double**)&c.fi, d->faces_i, 2 * nfi, reload));
  TRY(put(plan, (double**)&c.fj, d->faces_j, 2 * nfj, reload));
  TRY(put(plan, (double**)&c.centres, d->centres, (size_t)2 * (NI + 2) * (NJ + 2), reload));
  if (d->distance) TRY(put(plan, (double**)&c.distance, d->distance, (size_t)N, reload));
  TRY(put(plan, (int**)&c.neighbours, d->neighbours, (size_t)N, reload));
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
          d->kind[s][k] < 0 || d->kind[s][k] > 6)
        return fail(JR_EINVAL, "a ghost record out of range");
    TRY(put(plan, (int**)&c.g_ghost[s], d->ghost[s], (size_t)n, reload));
    TRY(put(plan, (int**)&c.g_source[s], d->source[s], (size_t)n, reload));
    TRY(put(plan, (int**)&c.g_kind[s], d->kind[s], (size_t)n, reload));
    TRY(put(plan, (double**)&c.g_geom[s], d->geom[s], (size_t)4 * n, reload));
  }
  {
    // stage 2 reads stage-1 ghosts at the corners: which stage-1 record fills each source
    std::vector<int> rec_of(N, -1), src_rec(d->n_ghost[1], -1);
    for (int k = 0; k < d->n_ghost[0]; ++k) rec_of[d->ghost[0][k]] = k;
    for (int k = 0; k < d->n_ghost[1]; ++k)
      if (!d->interior[d->source[1][k]]) src_rec[k] = rec_of[d->source[1][k]];
    TRY(put(plan, (int**)&c.g_src_rec, src_rec.data(), src_rec.size(), reload));
    // which record fills each canvas cell (stage 2 after stage 1, as the fill order)
    std::vector<int> ghost_rec(N, -1);
    for (int k = 0; k < d->n_ghost[0]; ++k) ghost_rec[d->ghost[0][k]] = k;
    for (int k = 0; k < d->n_ghost[1]; ++k) ghost_rec[d->ghost[1][k]] = d->n_ghost[0] + k;
    TRY(put(plan, (int**)&c.ghost_rec, ghost_rec.data(), ghost_rec.size(), reload));
  }
  c.n_walls = d->n_walls;
  TRY(put(plan, (int**)&c.w_cell, d->wall_cell, (size_t)d->n_walls, reload));
  TRY(put(plan, (int**)&c.w_family, d->wall_family, (size_t)d->n_walls, reload));
  TRY(put(plan, (int**)&c.w_face, d->wall_face, (size_t)d->n_walls, reload));
  TRY(put(plan, (double**)&c.w_into, d->wall_into, (size_t)d->n_walls, reload));
  TRY(put(plan, (double**)&c.w_mid, d->wall_mid, (size_t)2 * d->n_walls, reload));
  const int nc = d->n_chains, L = d->chain_L;
  if (L > MAX_CHAIN) return fail(JR_EINVAL, "line chains longer than 1024 cells are not supported");
  c.n_chains = nc;
  c.L = L;
  std::vector<int> on_chain(N, 0);
  for (size_t k = 0; k < (size_t)nc * L; ++k) {
    int cell = d->chain_cells[k];
    if (cell >= N) return fail(JR_EINVAL, "a chain cell out of range");
    if (cell >= 0) on_chain[cell] = 1;
  }
  std::vector<int> off;
  for (int k = 0; k < N; ++k)
    if (!on_chain[k]) off.push_back(k);
  c.n_offchain = (int)off.size();
  TRY(put(plan, (int**)&c.offchain, off.data(), off.size(), reload));
  TRY(put(plan, (int**)&c.ch_cells, d->chain_cells, (size_t)nc * L, reload));
  TRY(put(plan, (int**)&c.ch_len, d->chain_len, (size_t)nc, reload));
  TRY(put(plan, (int**)&c.ch_up_face, d->chain_up_face, (size_t)nc * L, reload));
  TRY(put(plan, (int**)&c.ch_up_sign, d->chain_up_sign, (size_t)nc * L, reload));
  TRY(put(plan, (int**)&c.ch_down_face, d->chain_down_face, (size_t)nc * L, reload));
  TRY(put(plan, (int**)&c.ch_down_sign, d->chain_down_sign, (size_t)nc * L, reload));
  std::vector<int> fbase(nc);
  size_t fbase_total = 0;
  for (int k = 0; k < nc; ++k) {
    fbase[k] = (int)fbase_total;
    fbase_total += (size_t)d->chain_len[k] + 16;
  }
  factor_rows = fbase_total;
  TRY(put(plan, (int**)&c.ch_fbase, fbase.data(), (size_t)nc, reload));

  Physics& P = cd.P;
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
  sa_constants(P.sa);
  cd.visc = d->mu_inf > 0.0 ? (nv == 5 ? 2 : 1) : 0;
  if (nv == 5 && cd.visc != 2) return fail(JR_EINVAL, "the SA model needs a viscous flow");

  Config& cf = cd.cfg;
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
  cd.force_length = d->force_length;
  cd.moment_centre[0] = d->moment_centre[0];
  cd.moment_centre[1] = d->moment_centre[1];
  cd.n_vec = nv * N;
  cd.m = d->krylov_subspace;
  cd.mixed = d->precision == 1;
  dim3 tg = tile_grid(c);
  cd.tiles_x = (int)tg.x;
  cd.tiles_y = (int)tg.y;
  cd.n_tiles = (int)(tg.x * tg.y);
  if (!reload) cd.enabled = 1;
  return JR_OK;
}

// The line solve reads its chains' factor once per Arnoldi step, and inside the step the
// linearisation and the Krylov basis evict it from L2 between reads.  Where the whole flow
// factor fits the device's persisting-L2 maximum (one case or a small batch), the Krylov
// cycles' capture stream gets an access-policy window over it, so its lines persist (the
// context's persisting size -- a limit of this process's context, gone with it -- is raised
// to cover it, never lowered); larger factors are left
// to the normal policy, which measured as well or better for them.  A cache policy only:
// results are bitwise the same.
static void keep_factor_in_l2(cudaStream_t st, void* factor, size_t bytes) {
  int dev = 0, max_persist = 0, max_window = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev);
  cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev);
  if (bytes == 0 || bytes > (size_t)max_persist || bytes > (size_t)max_window) return;
  size_t now = 0;
  if (cudaDeviceGetLimit(&now, cudaLimitPersistingL2CacheSize) == cudaSuccess && now < bytes)
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, bytes);
  cudaStreamAttrValue a{};
  a.accessPolicyWindow.base_ptr = factor;
  a.accessPolicyWindow.num_bytes = bytes;
  a.accessPolicyWindow.hitRatio = 1.0f;
  a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &a);
  cudaGetLastError();   // a device without persisting L2 refuses quietly: the normal policy stays
}

// Work buffers: each kind is one allocation holding every case's part back to back.
static int build_buffers(jr_plan* p, const std::vector<size_t>& factor_rows) {
  const int nc = p->n_cases;
  std::vector<size_t> tile_off(nc), fb_off(nc), part_off(nc), jac_off(nc);
  size_t tiles = 0, fb = 0, part = 0, jac = 0;
  const int n_coef = jac_coefficients(p->visc), n_cell_coef = jac_cell_coefficients(p->visc);
  p->vec_off.assign(nc, 0);
  p->can_off.assign(nc, 0);
  p->face_off.assign(nc, 0);
  p->wall_off.assign(nc, 0);
  for (int k = 0; k < nc; ++k) {
    const Canvas& c = p->host[k].c;
    const size_t N = (size_t)c.NI * c.NJ, nf = (size_t)(c.NI + 1) * c.NJ + (size_t)c.NI * (c.NJ + 1);
    p->vec_off[k] = p->total_vec;
    p->can_off[k] = p->total_can;
    p->face_off[k] = p->total_faces;
    p->wall_off[k] = p->total_walls;
    p->total_walls += (size_t)c.n_walls;
    tile_off[k] = tiles;
    fb_off[k] = fb;
    part_off[k] = part;
    p->total_vec += (size_t)c.nvar * N;
    p->total_can += N;
    p->total_faces += nf;
    tiles += (size_t)p->host[k].n_tiles;
    p->host[k].jstride = (int)((nf + 31) / 32 * 32);
    jac_off[k] = jac;
    // the face coefficients (FP32 in the mixed form: half as many doubles' room), then the
    // cell coefficients and the ghost maps in FP64
    const size_t face_words = (size_t)n_coef * p->host[k].jstride;
    jac += (p->mixed ? face_words / 2 : face_words) + (size_t)n_cell_coef * N +
           (size_t)(c.n_ghost[0] + c.n_ghost[1]) * c.nvar * c.nvar;
    fb += factor_rows[k];
    part += (size_t)reduce_blocks(p->host[k].n_vec) * (MAX_KRYLOV + 1);
  }
  const size_t tb = p->mixed ? sizeof(float) : sizeof(double);
  const int NVEC = 11;
  double* vec[NVEC];
  for (int v = 0; v < NVEC; ++v) TRY(dev_alloc(p, (void**)&vec[v], p->total_vec * sizeof(double)));
  double *vdt, *dflow, *dsa, *lam, *mflux, *dflux, *tile_partial, *partial, *lin;
  unsigned* ticket;
  void *V, *fflow, *fsa, *scratch;
  TRY(dev_alloc(p, (void**)&vdt, p->total_can * sizeof(double)));
  TRY(dev_alloc(p, (void**)&dflow, p->total_can * sizeof(double)));
  TRY(dev_alloc(p, (void**)&dsa, p->total_can * sizeof(double)));
  TRY(dev_alloc(p, (void**)&lam, p->total_faces * sizeof(double)));
  TRY(dev_alloc(p, (void**)&mflux, p->total_faces * sizeof(double)));
  TRY(dev_alloc(p, (void**)&dflux, p->total_faces * sizeof(double)));
  TRY(dev_alloc(p, (void**)&tile_partial, tiles * sizeof(double)));
  TRY(dev_alloc(p, (void**)&lin, jac * sizeof(double)));
  TRY(dev_alloc(p, (void**)&partial, part * sizeof(double)));
  TRY(dev_alloc(p, (void**)&ticket, (size_t)nc * sizeof(unsigned)));
  TRY(dev_alloc(p, &V, (size_t)(p->m + 1) * p->total_vec * tb));
  // cyclic-reduction factor: per chain at most 80 (flow) and 5 (SA) entries per row of
  // (length + 16) rows; the level systems in scratch at most 104 per row
  TRY(dev_alloc(p, &fflow, fb * 80 * tb));
  TRY(dev_alloc(p, &fsa, fb * 5 * tb));
  TRY(dev_alloc(p, &scratch, fb * 104 * tb));
  TRY(dev_alloc(p, (void**)&p->sc, (size_t)nc * sizeof(Scalars)));
  TRY(dev_alloc(p, (void**)&p->mon, (size_t)nc * sizeof(Monitor)));
  TRY(dev_alloc(p, (void**)&p->history, (size_t)HIST_STEPS * nc * sizeof(double)));
  TRY(dev_alloc(p, (void**)&p->force_out, (size_t)8 * nc * sizeof(double)));
  TRY(dev_alloc(p, (void**)&p->norm_out, (size_t)nc * sizeof(double)));
  TRY(dev_alloc(p, (void**)&p->wall_out, std::max<size_t>(1, p->total_walls) * 5 * sizeof(double)));
  p->U = vec[0];
  for (int k = 0; k < nc; ++k) {
    CaseDev& cd = p->host[k];
    const size_t vo = p->vec_off[k], co = p->can_off[k], fo = p->face_off[k];
    double** mine[NVEC] = {&cd.U, &cd.qg, &cd.dqg, &cd.R, &cd.b, &cd.x, &cd.action, &cd.r, &cd.w, &cd.z, &cd.tmp};
    for (int v = 0; v < NVEC; ++v) *mine[v] = vec[v] + vo;
    cd.vdt = vdt + co;
    cd.dflow = dflow + co;
    cd.dsa = dsa + co;
    cd.lam = lam + fo;
    cd.mflux = mflux + fo;
    cd.dflux = dflux + fo;
    cd.tile_partial = tile_partial + tile_off[k];
    cd.jac = lin + jac_off[k];
    {
      const size_t face_words = (size_t)n_coef * cd.jstride;   // jstride is a multiple of 32
      double* rest = lin + jac_off[k] + (p->mixed ? face_words / 2 : face_words);
      cd.jcell = n_cell_coef > 0 ? rest : nullptr;
      cd.gmap = rest + (size_t)n_cell_coef * cd.c.NI * cd.c.NJ;
    }
    cd.partial = partial + part_off[k];
    cd.ticket = ticket + k;
    cd.V = (char*)V + (size_t)(p->m + 1) * vo * tb;
    cd.fflow = (char*)fflow + fb_off[k] * 80 * tb;
    cd.fsa = (char*)fsa + fb_off[k] * 5 * tb;
    cd.scratch = (char*)scratch + fb_off[k] * 104 * tb;
    cd.sc = p->sc + k;
    cd.mon = p->mon + k;
    cd.slot = k;
    cd.history = p->history;
    cd.force_out = p->force_out + 8 * k;
    cd.wall_out = p->wall_out + 5 * p->wall_off[k];
  }
  TRY(dev_alloc(p, (void**)&p->cases, (size_t)nc * sizeof(CaseDev)));
  TRY(dev_alloc(p, (void**)&p->adhoc, (size_t)nc * sizeof(CaseDev)));
  TRY(dev_alloc(p, (void**)&p->live, (size_t)nc * sizeof(CaseDev)));
  TRY(dev_alloc(p, (void**)&p->cycles, sizeof(unsigned long long)));
  if (cudaStreamCreateWithFlags(&p->body_st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(JR_ECUDA, "cudaStreamCreate failed");
  keep_factor_in_l2(p->body_st, fflow, fb * 80 * tb);
  if (cudaMemcpy(p->cases, p->host.data(), (size_t)nc * sizeof(CaseDev), cudaMemcpyHostToDevice) != cudaSuccess)
    return cuda_check("case table");
  return JR_OK;
}

static BatchDims dims_of(const std::vector<CaseDev>& cases, int n_slots) {
  BatchDims d{};
  d.n_cases = (int)cases.size();
  d.n_slots = n_slots;
  for (const CaseDev& cd : cases) {
    const Canvas& c = cd.c;
    d.tiles_x = std::max(d.tiles_x, cd.tiles_x);
    d.tiles_y = std::max(d.tiles_y, cd.tiles_y);
    d.ghost_records = std::max(d.ghost_records, c.n_ghost[0] + c.n_ghost[1]);
    d.faces = std::max(d.faces, (c.NI + 1) * c.NJ + c.NI * (c.NJ + 1));
    d.cells = std::max(d.cells, c.NI * c.NJ);
    d.n_vec = std::max(d.n_vec, cd.n_vec);
    d.chain_blocks = std::max(d.chain_blocks, chain_grid_blocks(c.n_chains, c.n_offchain));
    d.max_L = std::max(d.max_L, c.L);
    d.cgs_blocks = std::max(d.cgs_blocks, cgs_blocks(cd.n_vec));
  }
  d.chain_blocks = std::max(d.chain_blocks, 1);
  d.ls_factor_threads = 128;
  d.ls_apply_threads = 128;
  d.ls_apply_stage = 0;
  return d;
}

static void compute_dims(jr_plan* p) {
  p->dims = dims_of(p->host, p->n_cases);
  p->dims.ls_factor_threads = p->ls_factor_threads;
  p->dims.ls_apply_threads = p->ls_apply_threads;
  p->dims.ls_apply_stage = p->ls_apply_stage;
}

// The table of a call on caller buffers: the resident table with the named buffers of
// every case moved to its part of the caller's batch-long arrays.
struct Adhoc {
  jr_plan* p;
  std::vector<CaseDev> t;
  explicit Adhoc(jr_plan* plan) : p(plan), t(plan->host) {}
  void vec(double* CaseDev::*field, const double* base) {
    for (int k = 0; k < p->n_cases; ++k) t[k].*field = const_cast<double*>(base) + p->vec_off[k];
  }
  void faces(double* CaseDev::*field, double* base) {
    for (int k = 0; k < p->n_cases; ++k) t[k].*field = base + p->face_off[k];
  }
  const CaseDev* upload() {
    // from pageable memory: staged before the call returns, so `t` may go
    cudaMemcpyAsync(p->adhoc, t.data(), t.size() * sizeof(CaseDev), cudaMemcpyHostToDevice, p->st);
    return p->adhoc;
  }
};

static int upload_table(jr_plan* p) {
  p->live_dirty = true;
  cudaMemcpyAsync(p->cases, p->host.data(), p->host.size() * sizeof(CaseDev), cudaMemcpyHostToDevice, p->st);
  if (cudaStreamSynchronize(p->st) != cudaSuccess) return cuda_check("case table");
  return cuda_check("case table");
}

// The kernels of one Krylov cycle after its start: m Arnoldi steps, the least squares,
// the correction and the end-of-cycle residual.
static void enqueue_cycle(jr_plan* p, cudaStream_t st) {
  const CaseDev* t = p->live;
  const BatchDims& d = p->live_dims;
  const bool sa = p->nvar == 5, pre = p->cfg.preconditioner >= 1;
  const bool coupled = sa && p->cfg.preconditioner == 2;   // the 5x5 form: one more SA chain solve
  for (int j = 0; j < p->m; ++j) {
    const int src = j == 0 ? B_RR : B_W;
    if (pre) launch_chain_apply(t, d, sa, p->mixed, src, 1, j, B_Z, 1, st);
    else launch_scale_copy(t, d, p->mixed, src, 1, j, B_Z, 1, st);
    if (coupled) launch_chain_couple(t, d, p->mixed, B_Z, 1, st);
    // the tangent ghosts: the J.v tiles map their halo's ghosts from the source cells'
    // tangents (the linearisation's ghost maps); a case with the point-vortex far field
    // (its circulation a sum over the wall) has its tangent ghosts filled by a launch
    if (p->live_vortex) launch_ghosts(t, d, B_Z, 1, st);
    launch_jvp(t, d, p->visc, p->mixed, B_Z, B_VDT, B_W, 1, 1, st);
    launch_arnoldi_orth(t, d, p->mixed, j, st);
  }
  launch_lstsq(t, d, st);
  launch_combine(t, d, p->mixed, st);
  if (pre) launch_chain_apply(t, d, sa, p->mixed, B_TMP, 0, -1, B_Z, 1, st);
  else launch_scale_copy(t, d, false, B_TMP, 0, -1, B_Z, 1, st);
  if (coupled) launch_chain_couple(t, d, p->mixed, B_Z, 1, st);
  launch_cycle_end(t, d, st);
}

// Nodes of a captured graph: every node the step captures is a kernel, but for the
// conditional nodes of the cycles (whose type this runtime does not report back).
static int64_t graph_nodes(cudaGraph_t g) {
  size_t n = 0;
  cudaGraphGetNodes(g, nullptr, &n);
  return (int64_t)n;
}

// The launch sequence of one Newton step of every enabled case, captured on the plan's
// stream.  Each Krylov cycle is an IF node of the graph: a gate kernel after the cycle's
// start sets its condition to "some case is still active", so a cycle no case needs is
// skipped on the device without launching its kernels.
static int enqueue_step(jr_plan* p) {
  const CaseDev* t = p->live;
  const BatchDims& d = p->live_dims;
  if (d.n_cases == 0) return JR_OK;   // no enabled case: an empty step
  const bool sa = p->nvar == 5, pre = p->cfg.preconditioner >= 1;
  cudaStream_t st = p->st;
  launch_ghosts(t, d, -1, 0, st);
  launch_residual(t, d, p->visc, true, B_R, st);
  launch_linearize(t, d, p->visc, p->mixed, st);
  launch_gmres_init(t, d, st);
  launch_faces(t, d, p->visc, st);
  launch_cells(t, d, p->visc, st);
  if (pre) launch_chain_factor(t, d, sa, p->mixed, st);
  // JR_GRAPH_CONDITIONALS=0 captures every cycle unconditionally (its kernels return at
  // once when no case is active): for profilers that cannot see the kernels of a graph
  // with conditional nodes.  The results are the same either way.
  const char* env = getenv("JR_GRAPH_CONDITIONALS");
  const bool conditional = env == nullptr || strcmp(env, "0") != 0;
  for (int cyc = 0; cyc < p->cfg.maxiter; ++cyc) {
    launch_cycle_start(t, d, st);
    if (!conditional) {
      enqueue_cycle(p, st);
      p->kernels_per_cycle = 0;
      continue;
    }
    cudaStreamCaptureStatus status;
    cudaGraph_t graph;
    const cudaGraphNode_t* deps;
    size_t n_deps;
    if (cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &n_deps) != cudaSuccess ||
        status != cudaStreamCaptureStatusActive)
      return fail(JR_ECUDA, "the step is not being captured");
    cudaGraphConditionalHandle gate;
    if (cudaGraphConditionalHandleCreate(&gate, graph, 0, 0) != cudaSuccess) return cuda_check("conditional handle");
    launch_cycle_gate(t, d, gate, p->cycles, st);
    if (cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &n_deps) != cudaSuccess)
      return cuda_check("capture info");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = gate;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, graph, deps, n_deps, &cp) != cudaSuccess) return cuda_check("conditional node");
    if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess)
      return cuda_check("capture dependencies");
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(p->body_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess)
      return cuda_check("body capture");
    enqueue_cycle(p, p->body_st);
    cudaGraph_t body_out;
    if (cudaStreamEndCapture(p->body_st, &body_out) != cudaSuccess) return cuda_check("body capture end");
    if (cyc == 0) p->kernels_per_cycle = graph_nodes(body);
  }
  launch_newton_update(t, d, st);
  return JR_OK;
}

extern "C" {

const char* jr_last_error(void) { return g_error.c_str(); }

int jr_plan_destroy(jr_plan* plan) {
  if (plan == nullptr) return JR_OK;
  if (plan->graph) cudaGraphExecDestroy(plan->graph);
  if (plan->st) cudaStreamSynchronize(plan->st);
  for (void* a : plan->allocs) cudaFree(a);
  if (plan->owned_stream) cudaStreamDestroy(plan->owned_stream);
  if (plan->body_st) cudaStreamDestroy(plan->body_st);
  delete plan;
  return JR_OK;
}

int jr_batch_create(const jr_plan_desc* descs, int32_t n_cases, jr_plan** out) {
  if (descs == nullptr || out == nullptr || n_cases < 1) return fail(JR_EINVAL, "null argument or no cases");
  *out = nullptr;
  const jr_plan_desc& d0 = descs[0];
  for (int k = 1; k < n_cases; ++k) {
    const jr_plan_desc& d = descs[k];
    if (d.nvar != d0.nvar || (d.mu_inf > 0.0) != (d0.mu_inf > 0.0) || d.precision != d0.precision ||
        d.krylov_subspace != d0.krylov_subspace || d.krylov_restarts != d0.krylov_restarts ||
        d.preconditioner != d0.preconditioner)
      return fail(JR_EINVAL,
                  "the cases of a batch must share the model, the precision and the Krylov and preconditioner "
                  "settings");
  }
  jr_plan* plan = new jr_plan();
  plan->n_cases = n_cases;
  cudaGetDevice(&plan->device);
  plan->host.resize(n_cases);
  if (cudaStreamCreateWithFlags(&plan->owned_stream, cudaStreamNonBlocking) == cudaSuccess)
    plan->st = plan->owned_stream;
  if (plan->st == nullptr) {
    delete plan;
    return fail(JR_ECUDA, "cudaStreamCreate failed");
  }
  std::vector<size_t> rows(n_cases);
  int rc = JR_OK;
  for (int k = 0; k < n_cases && rc == JR_OK; ++k) rc = build_case(plan, &descs[k], plan->host[k], rows[k]);
  for (int k = 0; k < n_cases && rc == JR_OK; ++k)
    plan->chain_len.emplace_back(descs[k].chain_len, descs[k].chain_len + descs[k].n_chains);
  if (rc == JR_OK) {
    plan->nvar = d0.nvar;
    plan->visc = plan->host[0].visc;
    plan->m = d0.krylov_subspace;
    plan->mixed = d0.precision == 1;
    plan->cfg = plan->host[0].cfg;
    rc = build_buffers(plan, rows);
  }
  if (rc != JR_OK) {
    jr_plan_destroy(plan);
    return rc;
  }
  compute_dims(plan);
  configure_kernels();
  configure_line_kernels(MAX_CHAIN);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    rc = cuda_check("plan create");
    jr_plan_destroy(plan);
    return rc ? rc : fail(JR_ECUDA, "plan create");
  }
  // the freestream state of every case, its CFL and |R| = inf
  std::vector<double> U0(plan->total_vec);
  for (int k = 0; k < n_cases; ++k) {
    const CaseDev& cd = plan->host[k];
    const size_t N = (size_t)cd.c.NI * cd.c.NJ;
    for (int v = 0; v < cd.c.nvar; ++v)
      for (size_t i = 0; i < N; ++i) U0[plan->vec_off[k] + v * N + i] = cd.P.U_inf[v];
  }
  rc = jr_state_set(plan, U0.data(), d0.cfl, INFINITY);
  for (int k = 1; k < n_cases && rc == JR_OK; ++k)
    if (descs[k].cfl != d0.cfl) rc = jr_case_state_set(plan, k, nullptr, descs[k].cfl, INFINITY);
  if (rc) {
    jr_plan_destroy(plan);
    return rc;
  }
  *out = plan;
  return JR_OK;
}

int jr_plan_create(const jr_plan_desc* desc, jr_plan** out) { return jr_batch_create(desc, 1, out); }

int jr_plan_cases(const jr_plan* plan) { return plan ? plan->n_cases : 0; }

int jr_plan_sizes(const jr_plan* plan, int64_t* n_canvas, int64_t* n_faces) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (n_canvas) *n_canvas = (int64_t)plan->total_can;
  if (n_faces) *n_faces = (int64_t)plan->total_faces;
  return JR_OK;
}

int jr_case_sizes(const jr_plan* plan, int32_t c, int64_t* n_canvas, int64_t* n_faces, int64_t* canvas_offset,
                  int64_t* face_offset) {
  if (!plan || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad plan or case");
  const Canvas& cv = plan->host[c].c;
  if (n_canvas) *n_canvas = (int64_t)cv.NI * cv.NJ;
  if (n_faces) *n_faces = (int64_t)(cv.NI + 1) * cv.NJ + (int64_t)cv.NI * (cv.NJ + 1);
  if (canvas_offset) *canvas_offset = (int64_t)plan->can_off[c];
  if (face_offset) *face_offset = (int64_t)plan->face_off[c];
  return JR_OK;
}

void* jr_plan_stream(jr_plan* plan) { return plan ? (void*)plan->st : nullptr; }

int jr_plan_set_stream(jr_plan* plan, void* stream) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  cudaStream_t next = stream != nullptr ? (cudaStream_t)stream : plan->owned_stream;
  if (next == plan->st) return JR_OK;
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_plan_set_stream");
  plan->st = next;
  return JR_OK;
}

int jr_synchronize(jr_plan* plan) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("synchronize");
  return JR_OK;
}

int jr_residual(jr_plan* plan, const double* U, double* R, int first_order) {
  if (!plan || !U || !R) return fail(JR_EINVAL, "null argument");
  Adhoc a(plan);
  a.vec(&CaseDev::U, U);
  a.vec(&CaseDev::R, R);
  const CaseDev* t = a.upload();
  launch_ghosts(t, plan->dims, -1, 0, plan->st);
  launch_residual(t, plan->dims, plan->visc, first_order == 0, B_R, plan->st);
  return cuda_check("jr_residual");
}

int jr_jvp(jr_plan* plan, const double* U, const double* v, double* Jv) {
  if (!plan || !U || !v || !Jv) return fail(JR_EINVAL, "null argument");
  Adhoc a(plan);
  a.vec(&CaseDev::U, U);
  a.vec(&CaseDev::z, v);
  a.vec(&CaseDev::w, Jv);
  const CaseDev* t = a.upload();
  // as in the Newton step: the tiles evaluate the tangent ghosts themselves unless a case
  // uses the point-vortex far field
  bool vortex = false;
  for (const CaseDev& cd : plan->host) vortex = vortex || cd.P.far_field == 1;
  launch_ghosts(t, plan->dims, -1, 0, plan->st);
  launch_linearize(t, plan->dims, plan->visc, plan->mixed, plan->st);
  if (vortex) launch_ghosts(t, plan->dims, B_Z, 0, plan->st);
  launch_jvp(t, plan->dims, plan->visc, plan->mixed, B_Z, -1, B_W, 0, 1, plan->st);
  return cuda_check("jr_jvp");
}

int jr_norm(jr_plan* plan, const double* R, int32_t variable, double* out) {
  if (!plan || !R || !out) return fail(JR_EINVAL, "null argument");
  if (variable < 0 || variable >= plan->nvar) return fail(JR_EINVAL, "variable out of range");
  Adhoc a(plan);
  a.vec(&CaseDev::R, R);
  const CaseDev* t = a.upload();
  launch_norm(t, plan->n_cases, variable, plan->norm_out, plan->st);
  cudaMemcpyAsync(out, plan->norm_out, (size_t)plan->n_cases * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_norm");
  return cuda_check("jr_norm");
}

int jr_wave_speeds(jr_plan* plan, const double* U, double* lam) {
  if (!plan || !U || !lam) return fail(JR_EINVAL, "null argument");
  Adhoc a(plan);
  a.vec(&CaseDev::U, U);
  a.faces(&CaseDev::lam, lam);
  launch_faces(a.upload(), plan->dims, plan->visc, plan->st);
  return cuda_check("jr_wave_speeds");
}

int jr_precond_factor(jr_plan* plan, const double* U, double cfl) {
  if (!plan || !U) return fail(JR_EINVAL, "null argument");
  if (!(cfl > 0.0)) return fail(JR_EINVAL, "cfl must be positive");
  for (int k = 0; k < plan->n_cases; ++k)
    cudaMemcpyAsync(&plan->sc[k].cfl, &cfl, sizeof(double), cudaMemcpyHostToDevice, plan->st);
  plan->factor_U = U;
  Adhoc a(plan);
  a.vec(&CaseDev::U, U);
  const CaseDev* t = a.upload();
  launch_faces(t, plan->dims, plan->visc, plan->st);
  launch_cells(t, plan->dims, plan->visc, plan->st);
  launch_chain_factor(t, plan->dims, plan->nvar == 5, plan->mixed, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_precond_factor");
  return cuda_check("jr_precond_factor");
}

int jr_precond_apply(jr_plan* plan, const double* r, double* z) {
  if (!plan || !r || !z) return fail(JR_EINVAL, "null argument");
  Adhoc a(plan);
  a.vec(&CaseDev::r, r);
  a.vec(&CaseDev::z, z);
  if (plan->factor_U) a.vec(&CaseDev::U, plan->factor_U);   // the coupling is taken at the factor's state
  const CaseDev* t = a.upload();
  launch_chain_apply(t, plan->dims, plan->nvar == 5, plan->mixed, B_RR, 0, -1, B_Z, 0, plan->st);
  if (plan->nvar == 5 && plan->cfg.preconditioner == 2) launch_chain_couple(t, plan->dims, plan->mixed, B_Z, 0, plan->st);
  return cuda_check("jr_precond_apply");
}

int jr_case_state_set(jr_plan* plan, int32_t c, const double* U_host, double cfl, double residual_norm) {
  if (!plan || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad plan or case");
  if (U_host)
    cudaMemcpyAsync(plan->host[c].U, U_host, (size_t)plan->host[c].n_vec * sizeof(double), cudaMemcpyHostToDevice,
                    plan->st);
  Scalars s{};
  s.cfl = cfl;
  s.res_prev = residual_norm;
  cudaMemcpyAsync(plan->sc + c, &s, sizeof(Scalars), cudaMemcpyHostToDevice, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_case_state_set");
  return cuda_check("jr_case_state_set");
}

int jr_case_state_get(jr_plan* plan, int32_t c, double* U_host, double* cfl, double* residual_norm, int32_t* status) {
  if (!plan || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad plan or case");
  if (U_host)
    cudaMemcpyAsync(U_host, plan->host[c].U, (size_t)plan->host[c].n_vec * sizeof(double), cudaMemcpyDeviceToHost,
                    plan->st);
  Scalars s;
  cudaMemcpyAsync(&s, plan->sc + c, sizeof(Scalars), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_case_state_get");
  if (cfl) *cfl = s.cfl;
  if (residual_norm) *residual_norm = s.res_prev;
  if (status) *status = s.status;
  return cuda_check("jr_case_state_get");
}

int jr_state_set(jr_plan* plan, const double* U_host, double cfl, double residual_norm) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (U_host) cudaMemcpyAsync(plan->U, U_host, plan->total_vec * sizeof(double), cudaMemcpyHostToDevice, plan->st);
  std::vector<Scalars> s(plan->n_cases);
  for (Scalars& x : s) {
    memset(&x, 0, sizeof(Scalars));
    x.cfl = cfl;
    x.res_prev = residual_norm;
  }
  cudaMemcpyAsync(plan->sc, s.data(), s.size() * sizeof(Scalars), cudaMemcpyHostToDevice, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_state_set");
  return cuda_check("jr_state_set");
}

int jr_state_get(jr_plan* plan, double* U_host, double* cfl, double* residual_norm, int32_t* status) {
  if (!plan) return fail(JR_EINVAL, "null plan");
  if (U_host) cudaMemcpyAsync(U_host, plan->U, plan->total_vec * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  std::vector<Scalars> s(plan->n_cases);
  cudaMemcpyAsync(s.data(), plan->sc, s.size() * sizeof(Scalars), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_state_get");
  for (int k = 0; k < plan->n_cases; ++k) {
    if (cfl) cfl[k] = s[k].cfl;
    if (residual_norm) residual_norm[k] = s[k].res_prev;
    if (status) status[k] = s[k].status;
  }
  return cuda_check("jr_state_get");
}

double* jr_state_device(jr_plan* plan) { return plan ? plan->U : nullptr; }

int jr_state_set_device(jr_plan* plan, const double* U_device, double cfl, double residual_norm) {
  if (!plan || !U_device) return fail(JR_EINVAL, "null argument");
  cudaMemcpyAsync(plan->U, U_device, plan->total_vec * sizeof(double), cudaMemcpyDeviceToDevice, plan->st);
  return jr_state_set(plan, nullptr, cfl, residual_norm);
}

int jr_case_enable(jr_plan* plan, int32_t c, int32_t enabled) {
  if (!plan || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad plan or case");
  plan->host[c].enabled = enabled != 0;
  return upload_table(plan);
}

int jr_case_set_inflow(jr_plan* plan, int32_t c, const double* q_inf) {
  if (!plan || !q_inf || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad argument");
  Physics& P = plan->host[c].P;
  for (int k = 0; k < 5; ++k) P.q_inf[k] = k < plan->nvar ? q_inf[k] : 0.0;
  const double g = P.gamma, rho = P.q_inf[0], u = P.q_inf[1], v = P.q_inf[2], p = P.q_inf[3];
  P.U_inf[0] = rho;
  P.U_inf[1] = rho * u;
  P.U_inf[2] = rho * v;
  P.U_inf[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
  P.U_inf[4] = rho * P.q_inf[4];
  return upload_table(plan);
}

int jr_case_load(jr_plan* plan, int32_t c, const jr_plan_desc* d) {
  if (!plan || !d || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad argument");
  CaseDev& cd = plan->host[c];
  const Canvas& cv = cd.c;
  bool same = d->NI == cv.NI && d->NJ == cv.NJ && d->nvar == cv.nvar && d->n_ghost[0] == cv.n_ghost[0] &&
              d->n_ghost[1] == cv.n_ghost[1] && d->n_walls == cv.n_walls && d->n_chains == cv.n_chains &&
              d->chain_L == cv.L && (d->distance != nullptr) == (cv.distance != nullptr) &&
              (d->mu_inf > 0.0) == (cd.visc > 0) && d->precision == (plan->mixed ? 1 : 0) &&
              d->krylov_subspace == plan->m && d->krylov_restarts == plan->cfg.maxiter &&
              d->preconditioner == plan->cfg.preconditioner;
  for (int k = 0; same && k < d->n_chains; ++k) same = d->chain_len[k] == plan->chain_len[c][k];
  if (same) {
    const int N = d->NI * d->NJ;
    std::vector<char> on(N, 0);
    for (size_t k = 0; k < (size_t)d->n_chains * d->chain_L; ++k) {
      const int cell = d->chain_cells[k];
      if (cell >= N) return fail(JR_EINVAL, "a chain cell out of range");
      if (cell >= 0) on[cell] = 1;
    }
    int off = 0;
    for (int k = 0; k < N; ++k) off += on[k] == 0;
    same = off == cv.n_offchain;
  }
  if (!same)
    return fail(JR_EMISMATCH,
                "jr_case_load: the new case's canvas, tables or solver settings differ from the slot's");
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_case_load");
  size_t rows = 0;
  int rc = build_case(plan, d, cd, rows, true);
  if (rc != JR_OK) {
    cd.enabled = 0;   // half overwritten: keep the slot out of every launch
    upload_table(plan);
    return rc;
  }
  return upload_table(plan);
}

// The packed table of the enabled cases (slot order) and its extents; the step graph
// is dropped so that the next launch captures one over them.
static int refresh_live(jr_plan* p) {
  if (!p->live_dirty) return JR_OK;
  std::vector<CaseDev> on;
  for (const CaseDev& cd : p->host)
    if (cd.enabled) on.push_back(cd);
  p->n_live = (int)on.size();
  p->live_vortex = false;
  for (const CaseDev& cd : on) p->live_vortex = p->live_vortex || cd.P.far_field == 1;
  p->live_dims = dims_of(on, p->n_cases);
  p->live_dims.ls_factor_threads = p->ls_factor_threads;
  p->live_dims.ls_apply_threads = p->ls_apply_threads;
  p->live_dims.ls_apply_stage = p->ls_apply_stage;
  if (!on.empty()) {
    cudaMemcpyAsync(p->live, on.data(), on.size() * sizeof(CaseDev), cudaMemcpyHostToDevice, p->st);
    if (cudaStreamSynchronize(p->st) != cudaSuccess) return cuda_check("live table");
  }
  if (p->graph) {
    cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
  }
  p->live_dirty = false;
  return cuda_check("live table");
}

static int capture_step(jr_plan* plan, cudaGraph_t* g) {
  int rc = refresh_live(plan);
  if (rc) return rc;
  if (cudaStreamBeginCapture(plan->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return cuda_check("begin capture");
  int rc2 = enqueue_step(plan);
  cudaGraph_t made = nullptr;
  cudaError_t e = cudaStreamEndCapture(plan->st, &made);
  if (rc2 != JR_OK) {
    if (made) cudaGraphDestroy(made);
    return rc2;
  }
  if (e != cudaSuccess) return cuda_check("end capture");
  *g = made;
  // every node is a kernel but the cycles' conditional nodes (none without them)
  plan->kernels_outside = graph_nodes(made) - (plan->kernels_per_cycle > 0 ? plan->cfg.maxiter : 0);
  return JR_OK;
}

// Folds the kernels launched by the current graph's steps into `launched`.
static int fold_launches(jr_plan* p) {
  unsigned long long cycles = 0;
  cudaMemcpyAsync(&cycles, p->cycles, sizeof(cycles), cudaMemcpyDeviceToHost, p->st);
  if (cudaStreamSynchronize(p->st) != cudaSuccess) return cuda_check("launch count");
  p->launched += p->steps_since * p->kernels_outside + (int64_t)(cycles - p->cycles_base) * p->kernels_per_cycle;
  p->cycles_base = cycles;
  p->steps_since = 0;
  return JR_OK;
}

int jr_graph_kernels(jr_plan* plan, int64_t* kernels_per_step) {
  if (!plan || !kernels_per_step) return fail(JR_EINVAL, "null argument");
  int rc = fold_launches(plan);
  if (rc) return rc;
  cudaGraph_t g;
  rc = capture_step(plan, &g);
  if (rc) return rc;
  cudaGraphDestroy(g);
  *kernels_per_step = plan->kernels_outside + plan->cfg.maxiter * plan->kernels_per_cycle;
  return cuda_check("jr_graph_kernels");
}

int jr_launch_count(jr_plan* plan, int64_t* kernels) {
  if (!plan || !kernels) return fail(JR_EINVAL, "null argument");
  int rc = fold_launches(plan);
  if (rc) return rc;
  *kernels = plan->launched;
  return JR_OK;
}

static int ensure_graph(jr_plan* plan) {
  if (plan->live_dirty && plan->graph) {
    int rcf = fold_launches(plan);
    if (rcf) return rcf;
  }
  int rc0 = refresh_live(plan);
  if (rc0) return rc0;
  if (plan->graph) return JR_OK;
  cudaGraph_t g;
  int rc = capture_step(plan, &g);
  if (rc) return rc;
  if (cudaGraphInstantiate(&plan->graph, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_check("graph instantiate");
  }
  cudaGraphDestroy(g);
  return cuda_check("graph");
}

int jr_newton_steps_async(jr_plan* plan, int32_t n_steps, double* history_device) {
  if (!plan || n_steps < 0) return fail(JR_EINVAL, "bad argument");
  if (n_steps > HIST_STEPS) return fail(JR_EINVAL, "at most 4096 steps per call");
  int rc = ensure_graph(plan);
  if (rc) return rc;
  // the history position of every case restarts at 0 for this call
  for (int k = 0; k < plan->n_cases; ++k) cudaMemsetAsync(&plan->sc[k].hpos, 0, sizeof(int), plan->st);
  if (plan->n_live > 0) {
    for (int k = 0; k < n_steps; ++k)
      if (cudaGraphLaunch(plan->graph, plan->st) != cudaSuccess) return cuda_check("graph launch");
    plan->steps_since += n_steps;
  }
  if (history_device && n_steps > 0)
    cudaMemcpyAsync(history_device, plan->history, (size_t)n_steps * plan->n_cases * sizeof(double),
                    cudaMemcpyDeviceToDevice, plan->st);
  return cuda_check("jr_newton_steps");
}

int jr_newton_steps(jr_plan* plan, int32_t n_steps, double* history) {
  int rc = jr_newton_steps_async(plan, n_steps, nullptr);
  if (rc) return rc;
  if (history && n_steps > 0)
    cudaMemcpyAsync(history, plan->history, (size_t)n_steps * plan->n_cases * sizeof(double), cudaMemcpyDeviceToHost,
                    plan->st);
  // every case's status word, one strided copy
  std::vector<int> status(plan->n_cases, 0);
  cudaMemcpy2DAsync(status.data(), sizeof(int), &plan->sc[0].status, sizeof(Scalars), sizeof(int), plan->n_cases,
                    cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_newton_steps");
  rc = cuda_check("jr_newton_steps");
  if (rc) return rc;
  for (int k = 0; k < plan->n_cases; ++k)
    if (status[k] & ST_STAGE_FAILED)
      return fail(JR_ETIMEOUT, "a line solve's staged copy did not land within its wait limit");
  return JR_OK;
}

int jr_monitor_set(jr_plan* plan, int32_t c, double tol, double forces_tol, int32_t max_blocks, int32_t release) {
  if (!plan || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad plan or case");
  if (max_blocks < 1 || max_blocks > MONITOR_BLOCKS)
    return fail(JR_EINVAL, "max_blocks must lie in [1, " + std::to_string(MONITOR_BLOCKS) + "]");
  if (!(tol >= 0.0)) return fail(JR_EINVAL, "tol must be >= 0");
  Monitor head{};
  head.tol = tol;
  head.forces_tol = forces_tol > 0.0 ? forces_tol : -1.0;
  head.peak = 0.0;
  head.max_blocks = max_blocks;
  head.blocks = 0;
  head.reason = MON_RUNNING;
  head.release = release != 0;
  cudaMemcpyAsync(plan->mon + c, &head, offsetof(Monitor, coef), cudaMemcpyHostToDevice, plan->st);
  if (!plan->host[c].enabled) {
    plan->host[c].enabled = 1;
    return upload_table(plan);
  }
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_monitor_set");
  return cuda_check("jr_monitor_set");
}

int jr_monitor_blocks(jr_plan* plan, int32_t n_blocks, int32_t block_iters, double* history) {
  if (!plan || n_blocks < 1 || block_iters < 1) return fail(JR_EINVAL, "bad argument");
  if ((int64_t)n_blocks * block_iters > HIST_STEPS) return fail(JR_EINVAL, "at most 4096 steps per call");
  int rc = ensure_graph(plan);
  if (rc) return rc;
  cudaStream_t st = plan->st;
  for (int k = 0; k < plan->n_cases; ++k) cudaMemsetAsync(&plan->sc[k].hpos, 0, sizeof(int), st);
  if (plan->n_live > 0) {
    for (int b = 0; b < n_blocks; ++b) {
      for (int k = 0; k < block_iters; ++k)
        if (cudaGraphLaunch(plan->graph, st) != cudaSuccess) return cuda_check("graph launch");
      plan->steps_since += block_iters;
      launch_ghosts(plan->live, plan->live_dims, -1, 0, st);
      launch_forces(plan->live, plan->live_dims, st);
      launch_monitor(plan->live, plan->n_live, plan->n_cases, b * block_iters, block_iters, st);
      plan->launched += 3;
    }
  }
  if (history)
    cudaMemcpyAsync(history, plan->history, (size_t)n_blocks * block_iters * plan->n_cases * sizeof(double),
                    cudaMemcpyDeviceToHost, st);
  std::vector<int> status(plan->n_cases, 0), reason(plan->n_cases, 0), release(plan->n_cases, 0);
  cudaMemcpy2DAsync(status.data(), sizeof(int), &plan->sc[0].status, sizeof(Scalars), sizeof(int), plan->n_cases,
                    cudaMemcpyDeviceToHost, st);
  cudaMemcpy2DAsync(reason.data(), sizeof(int), &plan->mon[0].reason, sizeof(Monitor), sizeof(int), plan->n_cases,
                    cudaMemcpyDeviceToHost, st);
  cudaMemcpy2DAsync(release.data(), sizeof(int), &plan->mon[0].release, sizeof(Monitor), sizeof(int),
                    plan->n_cases, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_check("jr_monitor_blocks");
  rc = cuda_check("jr_monitor_blocks");
  if (rc) return rc;
  // a stopped case the device took out of the launches: a batch's leaves the host's
  // launch set too; a single case's plan is left enabled, as after jr_newton_steps
  bool changed = false;
  for (int k = 0; k < plan->n_cases; ++k) {
    if (!plan->host[k].enabled || reason[k] == MON_RUNNING || !release[k]) continue;
    if (plan->n_cases > 1) {
      plan->host[k].enabled = 0;
      changed = true;
    } else {
      const int on = 1;
      cudaMemcpyAsync(&plan->live[0].enabled, &on, sizeof(int), cudaMemcpyHostToDevice, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) return cuda_check("jr_monitor_blocks");
    }
  }
  if (changed) {
    rc = upload_table(plan);
    if (rc) return rc;
  }
  for (int k = 0; k < plan->n_cases; ++k)
    if (status[k] & ST_STAGE_FAILED)
      return fail(JR_ETIMEOUT, "a line solve's staged copy did not land within its wait limit");
  return JR_OK;
}

int jr_monitor_get(jr_plan* plan, int32_t c, int32_t* reason, int32_t* blocks, double* peak, double* coefficients) {
  if (!plan || c < 0 || c >= plan->n_cases) return fail(JR_EINVAL, "bad plan or case");
  Monitor head{};
  cudaMemcpyAsync(&head, plan->mon + c, offsetof(Monitor, coef), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_monitor_get");
  const int n = head.blocks < MONITOR_BLOCKS ? head.blocks : MONITOR_BLOCKS;
  if (coefficients && n > 0) {
    const char* coef = reinterpret_cast<const char*>(plan->mon + c) + offsetof(Monitor, coef);
    cudaMemcpyAsync(coefficients, coef, (size_t)n * 3 * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
    if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_monitor_get");
  }
  if (reason) *reason = head.reason;
  if (blocks) *blocks = head.blocks;
  if (peak) *peak = head.peak;
  return cuda_check("jr_monitor_get");
}

int jr_time_kernels(jr_plan* plan, int32_t reps, double* ms) {
  if (!plan || !ms || reps < 1) return fail(JR_EINVAL, "bad argument");
  jr_plan* p = plan;
  const CaseDev* t = p->cases;
  const BatchDims& d = p->dims;
  const bool sa = p->nvar == 5;
  cudaStream_t st = p->st;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // a consistent state for every kernel: base ghosts, wave speeds, the factor, an
  // active Krylov cycle with z = the residual
  launch_ghosts(t, d, -1, 0, st);
  launch_residual(t, d, p->visc, true, B_R, st);
  launch_linearize(t, d, p->visc, p->mixed, st);
  launch_faces(t, d, p->visc, st);
  launch_cells(t, d, p->visc, st);
  launch_chain_factor(t, d, sa, p->mixed, st);
  for (int k = 0; k < p->n_cases; ++k) {
    const CaseDev& cd = p->host[k];
    cudaMemcpyAsync(cd.z, cd.R, (size_t)cd.n_vec * sizeof(double), cudaMemcpyDeviceToDevice, st);
  }
  std::vector<Scalars> s(p->n_cases);
  cudaMemcpyAsync(s.data(), p->sc, s.size() * sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  for (Scalars& x : s) x.active = 1;
  cudaMemcpyAsync(p->sc, s.data(), s.size() * sizeof(Scalars), cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);
  auto timed = [&](int k, auto&& launch) {
    launch();
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms1 = 0.f;
    cudaEventElapsedTime(&ms1, e0, e1);
    ms[k] = (double)ms1 / reps;
  };
  timed(0, [&] { launch_residual(t, d, p->visc, true, B_R, st); });
  timed(1, [&] { launch_jvp(t, d, p->visc, p->mixed, B_Z, B_VDT, B_W, 0, 1, st); });
  timed(2, [&] { launch_ghosts(t, d, B_Z, 0, st); });
  timed(3, [&] { launch_chain_apply(t, d, sa, p->mixed, B_R, 0, -1, B_TMP, 0, st); });
  timed(4, [&] { launch_chain_factor(t, d, sa, p->mixed, st); });
  timed(5, [&] { launch_arnoldi_orth(t, d, p->mixed, p->m - 1, st); });
  timed(6, [&] { launch_linearize(t, d, p->visc, p->mixed, st); });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return cuda_check("jr_time_kernels");
}

// The autotuner: for the line factor and the line solve, time every block size the
// plan's longest chain allows (64, 128, 256 threads per chain), and for the solve each
// form (factor read from global memory level by level, or staged into shared memory
// from level s-1 of the longest chain, s = 1..4, where it fits), at the plan's state,
// and keep the fastest.  Only the schedule
// changes -- each row's arithmetic is the same -- so results do not depend on the
// choice.  The step graph is captured anew.
int jr_autotune(jr_plan* plan, int32_t reps, int32_t* chosen) {
  if (!plan || reps < 1) return fail(JR_EINVAL, "bad argument");
  jr_plan* p = plan;
  const CaseDev* t = p->cases;
  const bool sa = p->nvar == 5;
  cudaStream_t st = p->st;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  launch_faces(t, p->dims, p->visc, st);
  launch_cells(t, p->dims, p->visc, st);
  const int cands[3] = {64, 128, 256};
  float best_f = 1e30f, best_a = 1e30f;
  int pick_f = p->ls_factor_threads, pick_a = p->ls_apply_threads, pick_s = p->ls_apply_stage;
  auto timed = [&](auto&& launch) {
    launch();
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  for (int c : cands) {
    BatchDims d = p->dims;
    d.ls_factor_threads = c;
    d.ls_apply_threads = c;
    float tf = timed([&] { launch_chain_factor(t, d, sa, p->mixed, st); });
    if (tf < best_f) {
      best_f = tf;
      pick_f = c;
    }
    if (!apply_threads_valid(c, p->dims.max_L)) continue;
    for (int s = 0; s <= APPLY_STAGES; ++s) {
      if (!apply_stage_fits(p->dims.max_L, p->mixed, s)) continue;
      d.ls_apply_stage = s;
      float ta = timed([&] { launch_chain_apply(t, d, sa, p->mixed, B_R, 0, -1, B_TMP, 0, st); });
      if (ta < best_a) {
        best_a = ta;
        pick_a = c;
        pick_s = s;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc = cuda_check("jr_autotune");
  if (rc) return rc;
  p->ls_factor_threads = pick_f;
  p->ls_apply_threads = pick_a;
  p->ls_apply_stage = pick_s;
  compute_dims(p);
  p->live_dirty = true;
  if (chosen) {
    chosen[0] = pick_f;
    chosen[1] = pick_a;
    chosen[2] = pick_s;
  }
  return JR_OK;
}

// The bounded device wait checked on its own: a barrier no copy completes, waited on
// for `tries` tries (each up to 1 us), must give up and say so.
int jr_wait_limit_check(int32_t tries, int32_t* status) {
  if (tries < 1 || tries > (1 << 20)) return fail(JR_EINVAL, "tries must be in 1 .. 2^20");
  int s = -1;
  if (wait_limit_check(tries, &s, 0)) return cuda_check("jr_wait_limit_check");
  int rc = cuda_check("jr_wait_limit_check");
  if (rc) return rc;
  if (status) *status = s;
  if (s & ST_STAGE_FAILED) return fail(JR_ETIMEOUT, "the wait ran out (as it must: nothing completes its barrier)");
  return JR_OK;
}

// A line-solve schedule set by the caller: the block sizes of the factor and of the
// solve (64, 128 or 256 threads per chain) and the solve's form (0: factor read from
// global memory; s = 1..4: staged into shared memory from level s-1 of the longest
// chain).  Results do not depend on it.
int jr_line_schedule(jr_plan* plan, int32_t factor_threads, int32_t apply_threads, int32_t apply_stage) {
  if (!plan) return fail(JR_EINVAL, "bad argument");
  auto ok = [](int th) { return th == 64 || th == 128 || th == 256; };
  if (!ok(factor_threads) || !ok(apply_threads))
    return fail(JR_EINVAL, "line-solve blocks must have 64, 128 or 256 threads");
  if (!apply_threads_valid(apply_threads, plan->dims.max_L))
    return fail(JR_EINVAL, "too few line-solve threads for the longest chain (4 x threads >= its even rows)");
  if (apply_stage < 0 || apply_stage > APPLY_STAGES) return fail(JR_EINVAL, "apply_stage must be 0 to 4");
  if (!apply_stage_fits(plan->dims.max_L, plan->mixed, apply_stage))
    return fail(JR_EINVAL, "the staged factor does not fit one block's shared memory");
  plan->ls_factor_threads = factor_threads;
  plan->ls_apply_threads = apply_threads;
  plan->ls_apply_stage = apply_stage;
  compute_dims(plan);
  plan->live_dirty = true;
  return JR_OK;
}

int jr_wall_loads(jr_plan* plan, const double* U, double* out) {
  if (!plan || !out) return fail(JR_EINVAL, "null argument");
  std::vector<double> f((size_t)6 * plan->n_cases);
  int rc = jr_forces(plan, U, f.data());   // the same launch writes the per-face loads
  if (rc) return rc;
  if (plan->total_walls > 0) {
    cudaMemcpyAsync(out, plan->wall_out, plan->total_walls * 5 * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
    if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_wall_loads");
  }
  return cuda_check("jr_wall_loads");
}

int jr_forces(jr_plan* plan, const double* U, double* out) {
  if (!plan || !out) return fail(JR_EINVAL, "null argument");
  Adhoc a(plan);
  if (U) a.vec(&CaseDev::U, U);
  const CaseDev* t = a.upload();
  launch_ghosts(t, plan->dims, -1, 0, plan->st);
  launch_forces(t, plan->dims, plan->st);
  std::vector<double> f((size_t)8 * plan->n_cases);
  cudaMemcpyAsync(f.data(), plan->force_out, f.size() * sizeof(double), cudaMemcpyDeviceToHost, plan->st);
  if (cudaStreamSynchronize(plan->st) != cudaSuccess) return cuda_check("jr_forces");
  for (int k = 0; k < plan->n_cases; ++k)
    for (int i = 0; i < 6; ++i) out[6 * k + i] = f[8 * k + i];
  return cuda_check("jr_forces");
}

}  // extern "C"

// ------------------------------------------------------------------------------------
// The residual without allocation.  Some callers cannot allocate device memory when they
// evaluate a residual: a handler running inside another framework's step (an XLA custom
// call, a serving loop on a caching allocator), where the framework owns the device's
// memory and a cudaMalloc or cudaFree would also synchronise the whole device.
// jr_residual_noalloc serves them: its scratch (the call's case table, the ghost-filled
// primitive canvas and the per-tile partial sums) lives in the file-scope array below,
// which every GPU that loads this library holds until exit, so a call allocates nothing
// and writes no work buffer of the plan; it reads the plan's static tables, U, and
// writes R.
// ------------------------------------------------------------------------------------

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(8) << 20;   // 8 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
// the array's device address on each device; the name g_noalloc_scratch in host code is
// only a host-side stand-in, never a device address.  Looked up once per device and kept
// for the life of the process: a cudaDeviceReset (or anything else that re-creates the
// device's primary context) leaves the kept address stale, so the library must not be
// used across one.  Host threads may race on an entry the first time; the race is benign,
// as every writer stores the same address.
static unsigned char* g_noalloc_ptr[NOALLOC_MAX_DEVICES];

static size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// The call's table in the scratch: the plan's cases with U and R moved to the caller's
// arrays and qg, tile_partial into the scratch.  One thread walks the cases, in case
// order, so the offsets are the plan's own.
__global__ void k_noalloc_table(const CaseDev* __restrict__ src, CaseDev* __restrict__ dst, int n_cases,
                                const double* U, double* R, double* qg, double* tile_partial) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  size_t vec = 0, tiles = 0;
  for (int k = 0; k < n_cases; ++k) {
    CaseDev cd = src[k];
    cd.U = const_cast<double*>(U) + vec;
    cd.R = R + vec;
    cd.qg = qg + vec;
    cd.tile_partial = tile_partial + tiles;
    dst[k] = cd;
    vec += (size_t)cd.n_vec;
    tiles += (size_t)cd.n_tiles;
  }
}

extern "C" int jr_residual_noalloc(jr_plan* plan, const double* U, double* R, int first_order) {
  if (!plan || !U || !R) return fail(JR_EINVAL, "null argument");
  size_t tiles = 0;
  for (const CaseDev& cd : plan->host) tiles += (size_t)cd.n_tiles;
  const size_t table_bytes = round256((size_t)plan->n_cases * sizeof(CaseDev));
  const size_t qg_bytes = round256(plan->total_vec * sizeof(double));
  const size_t need = table_bytes + qg_bytes + tiles * sizeof(double);
  if (need > NOALLOC_SCRATCH_BYTES)
    return fail(JR_EINVAL, "jr_residual_noalloc: the plan needs " + std::to_string(need) +
                               " bytes of scratch, more than the 8 MiB (8388608 bytes) this entry point has; "
                               "use jr_residual");
  if (plan->device < 0 || plan->device >= NOALLOC_MAX_DEVICES)
    return fail(JR_EINVAL, "jr_residual_noalloc: device ordinal beyond 63");
  int current = 0;
  if (cudaGetDevice(&current) != cudaSuccess) return cuda_check("jr_residual_noalloc: cudaGetDevice");
  if (current != plan->device) return fail(JR_EINVAL, "jr_residual_noalloc: make the plan's device current first");
  // set-up, once per device (the first call on it): the array's device address
  unsigned char* base = g_noalloc_ptr[current];
  if (base == nullptr) {
    cudaError_t e = cudaGetSymbolAddress((void**)&base, g_noalloc_scratch);
    if (e != cudaSuccess || base == nullptr)
      return fail(JR_ECUDA, std::string("jr_residual_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[current] = base;
  }
  CaseDev* table = reinterpret_cast<CaseDev*>(base);
  double* qg = reinterpret_cast<double*>(base + table_bytes);
  double* tile_partial = reinterpret_cast<double*>(base + table_bytes + qg_bytes);
  // the array keeps the last call's contents: clearing the ghost canvas makes the result
  // independent of earlier calls (the residual reads a canvas entry of this buffer only
  // where a ghost record has just written it)
  if (cudaMemsetAsync(qg, 0, plan->total_vec * sizeof(double), plan->st) != cudaSuccess)
    return cuda_check("jr_residual_noalloc: clear");
  k_noalloc_table<<<1, 32, 0, plan->st>>>(plan->cases, table, plan->n_cases, U, R, qg, tile_partial);
  launch_ghosts(table, plan->dims, -1, 0, plan->st);
  launch_residual(table, plan->dims, plan->visc, first_order == 0, B_R, plan->st);
  return cuda_check("jr_residual_noalloc");
}
