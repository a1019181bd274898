// Test only: the 3D kernels' per-cell and per-record bodies (jax-rans_b200/csrc/
// residual3d.cuh) run on the host, in the order the device runs them, on a plan given by
// its C-ABI descriptor -- a check of the kernels' indexing and arithmetic without a GPU.
// Nothing of the library calls this; it is built by tests/test_host3d.py.
#include <utility>
#include <vector>

#include "../../jax-rans_b200/csrc/plan3d_desc.cuh"
#include "../../jax-rans_b200/csrc/linesolve3d.cuh"

using namespace jr;

template <class T, bool VISC, bool SA>
static void run(const Plan3Dev& p, const double* U, const double* dU, double* R, int first_order) {
  const int n = p.NI * p.NJ * p.NK;
  std::vector<T> A((size_t)p.nvar * n), B((size_t)p.nvar * n);
  for (int c = 0; c < n; ++c) prim_cell(p, U, dU, A.data(), c);
  for (int s = 0; s < p.n_stages; ++s) {
    B = A;
    for (int r = p.stage_off[s]; r < p.stage_off[s + 1]; ++r) ghost_record(p, A.data(), B.data(), r);
    std::swap(A, B);
  }
  for (int c = 0; c < n; ++c) residual_cell<T, VISC, SA>(p, A.data(), U, dU, R, first_order, c);
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
  p.chain_L = d->chain_L;
  p.ch_cells = d->chain_cells;
  p.ch_face = d->chain_up_face;
  p.ch_sign = d->chain_up_sign;
  physics3_from_desc(p.P, d);
  return p;
}

extern "C" int jr3_host_eval(const jr_plan3d_desc* d, const double* U, const double* dU, double* R,
                             int first_order) {
  if (d->n_stages < 1 || d->n_stages > MAX_STAGES3) return 1;
  const Plan3Dev p = plan_of(d);
  const bool visc = p.P.mu_inf > 0.0, sa = p.nvar > 5;
  if (dU) {
    if (sa) run<Dual, true, true>(p, U, dU, R, 1);
    else if (visc) run<Dual, true, false>(p, U, dU, R, 1);
    else run<Dual, false, false>(p, U, dU, R, 1);
  } else {
    if (sa) run<double, true, true>(p, U, nullptr, R, first_order);
    else if (visc) run<double, true, false>(p, U, nullptr, R, first_order);
    else run<double, false, false>(p, U, nullptr, R, first_order);
  }
  return 0;
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

extern "C" int jr3_host_precondition(const jr_plan3d_desc* d, const double* U, double cfl, const double* r,
                                     double* z) {
  const Plan3Dev p = plan_of(d);
  const size_t n = (size_t)p.nvar * p.NI * p.NJ * p.NK;
  for (size_t e = 0; e < n; ++e) z[e] = r[e];
  std::vector<double> scratch((size_t)p.chain_L * 30);
  for (int ch = 0; ch < p.n_chains; ++ch) {
    chain_flow(p, U, cfl, ch, r, z, scratch.data(), scratch.data() + (size_t)p.chain_L * 25);
    if (p.nvar > 5) chain_sa(p, U, cfl, ch, r, z, scratch.data(), scratch.data() + (size_t)p.chain_L * 25);
  }
  return 0;
}
