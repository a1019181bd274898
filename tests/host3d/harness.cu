// Test only: the 3D kernels' per-cell and per-record bodies (jax-rans_b200/csrc/
// residual3d.cuh) run on the host, in the order the device runs them, on a plan given by
// its C-ABI descriptor -- a check of the kernels' indexing and arithmetic without a GPU.
// Nothing of the library calls this; it is built by tests/test_host3d.py.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "../../jax-rans_b200/csrc/plan3d_desc.cuh"
#include "../../jax-rans_b200/csrc/linesolve3d.cuh"
#include "../../jax-rans_b200/csrc/newton3d.cuh"
#include "../../jax-rans_b200/csrc/walldist3d.cuh"

using namespace jr;

// the ghost stages in place as the device runs them: each stage's values first (from the
// canvas before the stage), then the stores
template <class T>
static void fill_ghosts(const Plan3Dev& p, std::vector<T>& A) {
  for (int s = 0; s < p.n_stages; ++s) {
    const int r0 = p.stage_off[s], r1 = p.stage_off[s + 1];
    std::vector<T> buf((size_t)p.nvar * (r1 - r0 > 0 ? r1 - r0 : 1));
    for (int r = r0; r < r1; ++r) ghost_value(p, A.data(), r, r0, r1 - r0, buf.data());
    for (int r = r0; r < r1; ++r) ghost_store(p, buf.data(), r, r0, r1 - r0, A.data());
  }
}

// the ghost stages double-buffered (each stage from a copy of the canvas): the gather
// form's meaning, for checking the in-place passes against it
template <class T>
static void fill_ghosts_copying(const Plan3Dev& p, std::vector<T>& A) {
  std::vector<T> B;
  for (int s = 0; s < p.n_stages; ++s) {
    B = A;
    for (int r = p.stage_off[s]; r < p.stage_off[s + 1]; ++r) ghost_record(p, A.data(), B.data(), r);
    std::swap(A, B);
  }
}

// the residual in the fused form (each cell evaluates its six faces), or in the device's
// two phases (every face once into a buffer, unwritten entries NaN, then the cell sums)
template <class T, bool VISC, bool SA>
static void run(const Plan3Dev& p, const double* U, const double* dU, double* R, int first_order,
                bool two_phase = false) {
  const int n = p.NI * p.NJ * p.NK;
  std::vector<T> A((size_t)p.nvar * n);
  for (int c = 0; c < n; ++c) prim_cell(p, U, dU, A.data(), c);
  fill_ghosts(p, A);
  if (!two_phase) {
    for (int c = 0; c < n; ++c) residual_cell<T, VISC, SA>(p, A.data(), U, dU, R, first_order, c);
    return;
  }
  const int nf = face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  std::vector<double> Fb((size_t)p.nvar * nf, std::nan(""));
  for (int f = 0; f < nf; ++f) store_face_flux<T, VISC, SA>(p, A.data(), first_order, f, Fb.data(), (size_t)nf);
  for (int c = 0; c < n; ++c) residual_cell_from_faces<T, SA>(p, A.data(), Fb.data(), (size_t)nf, U, dU, R, c);
}

static Plan3Dev plan_of(const jr_plan3d_desc* d) {
  Plan3Dev p{};
  p.NI = d->NI;
  p.NJ = d->NJ;
  p.NK = d->NK;
  p.nvar = d->nvar;
  p.interior = d->interior;
  p.volume = d->volume;
  for (int a = 0; a < 3; ++a) p.faces[a] = d->faces[a];
  p.centres = d->centres;
  p.distance = d->distance;
  p.n_stages = d->n_stages < MAX_STAGES3 ? d->n_stages : MAX_STAGES3;
  p.stage_off[0] = 0;
  for (int s = 0; s < p.n_stages; ++s) p.stage_off[s + 1] = p.stage_off[s] + d->stage_records[s];
  p.g_ghost = d->ghost;
  p.g_source = d->source;
  p.g_kind = d->kind;
  p.g_normal = d->normal;
  p.neighbours = d->neighbours;
  p.n_chains = d->n_chains;
  p.line_fp32 = d->line_precision;
  p.line_coupled = d->preconditioner == 2;
  p.chain_L = d->chain_L;
  p.ch_cells = d->chain_cells;
  p.ch_face = d->chain_up_face;
  p.ch_sign = d->chain_up_sign;
  p.n_walls = d->n_walls;
  p.w_cell = d->wall_cell;
  p.w_family = d->wall_family;
  p.w_face = d->wall_face;
  p.w_into = d->wall_into;
  physics3_from_desc(p.P, d);
  return p;
}

static int eval(const jr_plan3d_desc* d, const double* U, const double* dU, double* R, int first_order,
                bool two_phase) {
  if (d->n_stages < 1 || d->n_stages > MAX_STAGES3) return 1;
  const Plan3Dev p = plan_of(d);
  const bool visc = p.P.mu_inf > 0.0, sa = p.nvar > 5;
  if (dU) {
    if (sa) run<Dual, true, true>(p, U, dU, R, 1, two_phase);
    else if (visc) run<Dual, true, false>(p, U, dU, R, 1, two_phase);
    else run<Dual, false, false>(p, U, dU, R, 1, two_phase);
  } else {
    if (sa) run<double, true, true>(p, U, nullptr, R, first_order, two_phase);
    else if (visc) run<double, true, false>(p, U, nullptr, R, first_order, two_phase);
    else run<double, false, false>(p, U, nullptr, R, first_order, two_phase);
  }
  return 0;
}

// the device's two-phase form of jr3_host_eval
extern "C" int jr3_host_eval_faces(const jr_plan3d_desc* d, const double* U, const double* dU, double* R,
                                   int first_order) {
  return eval(d, U, dU, R, first_order, true);
}

extern "C" int jr3_host_eval(const jr_plan3d_desc* d, const double* U, const double* dU, double* R,
                             int first_order) {
  return eval(d, U, dU, R, first_order, false);
}

extern "C" int jr3_host_wave_speeds(const jr_plan3d_desc* d, const double* U, double* lam) {
  const Plan3Dev p = plan_of(d);
  const int total = face_count(p, 0) + face_count(p, 1) + face_count(p, 2);
  for (int f = 0; f < total; ++f) {
    int a, i, j, k;
    face_of(p, f, a, i, j, k);
    lam[f] = wave_speed(p, U, a, i, j, k);
  }
  return 0;
}

// the line factor of every chain, then the apply, in the words the descriptor asks for
template <class TF>
static void line_solve(const Plan3Dev& p, const double* U, double cfl, const double* r, double* z) {
  const size_t n = (size_t)p.nvar * p.NI * p.NJ * p.NK;
  for (size_t e = 0; e < n; ++e) z[e] = r[e];
  std::vector<TF> F((size_t)p.n_chains * p.chain_L * FACTOR3);
  for (int ch = 0; ch < p.n_chains; ++ch) {
    chain_factor_flow(p, U, cfl, ch, F.data());
    if (p.nvar > 5) chain_factor_sa(p, U, cfl, ch, F.data());
  }
  for (int ch = 0; ch < p.n_chains; ++ch) {
    chain_apply_flow(p, ch, F.data(), r, z);
    if (p.nvar > 5) chain_apply_sa(p, ch, F.data(), r, z);
  }
}

static void line_solve_as(const Plan3Dev& p, const double* U, double cfl, const double* r, double* z) {
  if (p.line_fp32) line_solve<float>(p, U, cfl, r, z);
  else line_solve<double>(p, U, cfl, r, z);
}

extern "C" int jr3_host_precondition(const jr_plan3d_desc* d, const double* U, double cfl, const double* r,
                                     double* z) {
  line_solve_as(plan_of(d), U, cfl, r, z);
  return 0;
}

// The Newton step's vector operations as host loops (sums in index order).
struct HostOps {
  enum { R_ = 0, Z_, W_, T_, RES_, B_, DU_, ACT_, BASE };
  const Plan3Dev& p;
  size_t N, n;
  std::vector<std::vector<double>> vec;
  std::vector<double> vdt;
  HostOps(const Plan3Dev& plan, int m) : p(plan) {
    n = (size_t)p.NI * p.NJ * p.NK;
    N = (size_t)p.nvar * n;
    vec.assign(BASE + m + 1, std::vector<double>(N, 0.0));
    vdt.assign(n, 0.0);
  }
  int V(int i) const { return BASE + i; }
  double* d(int id) { return vec[id].data(); }
  void prepare(const double* U, double cfl) {
    for (size_t c = 0; c < n; ++c) vdt[c] = lambda_sum(p, U, (int)c) / cfl;
  }
  void residual(const double* U, int out) {
    const bool visc = p.P.mu_inf > 0.0, sa = p.nvar > 5;
    if (sa) run<double, true, true>(p, U, nullptr, d(out), 0, true);
    else if (visc) run<double, true, false>(p, U, nullptr, d(out), 0, true);
    else run<double, false, false>(p, U, nullptr, d(out), 0, true);
  }
  void matvec(const double* U, double, int src, int out) {
    const bool visc = p.P.mu_inf > 0.0, sa = p.nvar > 5;
    if (sa) run<Dual, true, true>(p, U, d(src), d(out), 1, true);
    else if (visc) run<Dual, true, false>(p, U, d(src), d(out), 1, true);
    else run<Dual, false, false>(p, U, d(src), d(out), 1, true);
    for (size_t e = 0; e < N; ++e) d(out)[e] = vdt[e % n] * d(src)[e] + d(out)[e];
  }
  void precondition(const double* U, double cfl, int src, int dst) { line_solve_as(p, U, cfl, d(src), d(dst)); }
  double dot(int a, int b) {
    double s = 0.0;
    for (size_t e = 0; e < N; ++e) s += d(a)[e] * d(b)[e];
    return s;
  }
  double nrm2(int a) { return std::sqrt(dot(a, a)); }
  void mdot(int count, int w, double* h) {
    for (int i = 0; i < count; ++i) h[i] = dot(V(i), w);
  }
  void maxpy(int count, const double* coef, int y) {
    for (int i = 0; i < count; ++i) axpy(coef[i], V(i), y);
  }
  void axpy(double al, int x, int y) { for (size_t e = 0; e < N; ++e) d(y)[e] = d(y)[e] + al * d(x)[e]; }
  void scale(double al, int x, int y) { for (size_t e = 0; e < N; ++e) d(y)[e] = al * d(x)[e]; }
  void copy(int x, int y) { vec[y] = vec[x]; }
  void zero(int y) { std::fill(vec[y].begin(), vec[y].end(), 0.0); }
  double density_norm(int r) {
    double a = 0.0, w = 0.0;
    for (size_t c = 0; c < n; ++c)
      if (p.interior[c]) {
        a += p.volume[c] * d(r)[c] * d(r)[c];
        w += p.volume[c];
      }
    return std::sqrt(a / w);
  }
  double worst_ratio(const double* U, int du) {
    double worst = 0.0;
    for (size_t c = 0; c < n; ++c) {
      double q[NV3_MAX];
      prim_at(p, U, (int)c, q);
      const double* D = d(du);
      double de = D[4 * n + c];
      for (int k = 0; k < 3; ++k) de = de - q[1 + k] * D[(1 + k) * n + c];
      const double vv = (q[1] * q[1] + q[2] * q[2]) + q[3] * q[3];
      const double dp = (p.P.gamma - 1.0) * (de + 0.5 * vv * D[c]);
      worst = std::fmax(worst, std::fabs(D[c]) / q[0]);
      worst = std::fmax(worst, std::fabs(dp) / q[4]);
      if (p.nvar > 5) {
        const double nh = U[5 * n + c] / q[0];
        const double dnh = (D[5 * n + c] - nh * D[c]) / q[0];
        worst = std::fmax(worst, std::fabs(dnh) / std::fmax(std::fabs(nh), 1.0));
      }
    }
    return worst;
  }
  bool physical_after(const double* U, int du) {
    std::vector<double> cand(N);
    for (size_t e = 0; e < N; ++e) {
      if (!std::isfinite(d(du)[e])) return false;
      cand[e] = U[e] + d(du)[e];
    }
    for (size_t c = 0; c < n; ++c) {
      double q[NV3_MAX];
      prim_at(p, cand.data(), (int)c, q);
      if (!(q[0] > 1e-10) || !(q[4] > 1e-10) || !std::isfinite(q[0]) || !std::isfinite(q[4])) return false;
    }
    return true;
  }
  void add_to_state(double* U, int du) { for (size_t e = 0; e < N; ++e) U[e] = U[e] + d(du)[e]; }
};

extern "C" int jr3_host_newton_steps(const jr_plan3d_desc* d, const double* config, const int* iconfig, double* U,
                                     double* cfl, double* res_prev, int n_steps, double* history) {
  const Plan3Dev p = plan_of(d);
  Newton3Config c{iconfig[0], iconfig[1], iconfig[2], config[0], config[1], config[2], config[3], config[4],
                  config[5], config[6]};
  HostOps ops(p, c.restart);
  for (int s = 0; s < n_steps; ++s) history[s] = newton_step3(ops, U, *cfl, *res_prev, c);
  return 0;
}

// the 7 loads of every wall face (n_walls x 7) from the ghost-filled state
extern "C" int jr3_host_wall_loads(const jr_plan3d_desc* d, const double* U, double* loads) {
  const Plan3Dev p = plan_of(d);
  const int n = p.NI * p.NJ * p.NK;
  std::vector<double> A((size_t)p.nvar * n);
  for (int c = 0; c < n; ++c) prim_cell(p, U, (const double*)nullptr, A.data(), c);
  fill_ghosts(p, A);
  for (int w = 0; w < p.n_walls; ++w) wall_load(p, A.data(), w, loads + (size_t)7 * w);
  return 0;
}

extern "C" int jr3_host_forces(const jr_plan3d_desc* d, const double* U, double area, double length,
                               const double* centre, double* out) {
  std::vector<double> loads((size_t)d->n_walls * 7);
  jr3_host_wall_loads(d, U, loads.data());
  force_coefficients3(plan_of(d).P, d->n_walls, loads.data(), d->wall_mid, area, length, centre, out);
  return 0;
}

// the wall distance of points (n x 3) to faces (m x 4 x 3), faces offered in order as the
// kernel offers them (bounded = 1: skipping by the bounding spheres; 0: every face ranked)
extern "C" int jr3_host_wall_distance(const double* points, long long n, const double* faces, int m, double* out,
                                      int bounded) {
  std::vector<double> spheres((size_t)4 * m);
  for (int f = 0; f < m; ++f) face_sphere(faces + (size_t)12 * f, spheres.data() + (size_t)4 * f);
  for (long long i = 0; i < n; ++i) {
    const V3 p = v3(points + 3 * i);
    Candidates c;
    c.init(m);
    for (int f = 0; f < m; ++f) {
      if (bounded) offer_face(c, p, faces + (size_t)12 * f, spheres.data() + (size_t)4 * f, f);
      else c.offer(face_rank_distance(p, faces + (size_t)12 * f), f);
    }
    out[i] = m > 0 ? candidates_distance(p, c, faces) : INFINITY;
  }
  return 0;
}

// the ghost-filled primitive canvas (nvar x canvas) at U, in place (mode 0) or
// double-buffered (mode 1)
extern "C" int jr3_host_fill(const jr_plan3d_desc* d, const double* U, double* Q, int mode) {
  const Plan3Dev p = plan_of(d);
  const int n = p.NI * p.NJ * p.NK;
  std::vector<double> A((size_t)p.nvar * n);
  for (int c = 0; c < n; ++c) prim_cell(p, U, (const double*)nullptr, A.data(), c);
  if (mode == 0) fill_ghosts(p, A);
  else fill_ghosts_copying(p, A);
  std::copy(A.begin(), A.end(), Q);
  return 0;
}
