// Test only: the 3D kernels' per-cell and per-record bodies (jax-rans_b200/csrc/
// residual3d.cuh) run on the host, in the order the device runs them, on a plan given by
// its C-ABI descriptor -- a check of the kernels' indexing and arithmetic without a GPU.
// Nothing of the library calls this; it is built by tests/test_host3d.py.
#include <utility>
#include <vector>

#include "../../jax-rans_b200/csrc/plan3d_desc.cuh"
#include "../../jax-rans_b200/csrc/residual3d.cuh"

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

extern "C" int jr3_host_eval(const jr_plan3d_desc* d, const double* U, const double* dU, double* R,
                             int first_order) {
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
  p.n_stages = d->n_stages;
  if (p.n_stages < 1 || p.n_stages > MAX_STAGES3) return 1;
  p.stage_off[0] = 0;
  for (int s = 0; s < d->n_stages; ++s) p.stage_off[s + 1] = p.stage_off[s] + d->stage_records[s];
  p.g_ghost = d->ghost;
  p.g_source = d->source;
  p.g_kind = d->kind;
  p.g_normal = d->normal;
  physics3_from_desc(p.P, d);
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
