// The physics of a 3D plan from its C-ABI descriptor (shared by the plan builder and
// the host check of the 3D kernels' bodies).
#pragma once
#include "../../include/jaxrans_b200.h"
#include "device3d.cuh"

namespace jr {

inline void physics3_from_desc(Physics3& P, const jr_plan3d_desc* d) {
  P.gamma = d->gamma;
  P.mu_inf = d->mu_inf > 0.0 ? d->mu_inf : 0.0;
  P.sutherland = d->sutherland;
  P.kappa = d->kappa;
  P.flux = d->flux;
  P.limiter = d->limiter;
  for (int v = 0; v < NV3_MAX; ++v) P.q_inf[v] = v < d->nvar ? d->q_inf[v] : 0.0;
  const double g = d->gamma, rho = P.q_inf[0], u = P.q_inf[1], v = P.q_inf[2], w = P.q_inf[3], pr = P.q_inf[4];
  P.U_inf[0] = rho;
  P.U_inf[1] = rho * u;
  P.U_inf[2] = rho * v;
  P.U_inf[3] = rho * w;
  P.U_inf[4] = pr / (g - 1.0) + 0.5 * rho * ((u * u + v * v) + w * w);
  P.U_inf[5] = rho * P.q_inf[5];
  sa_constants(P.sa);
}

}  // namespace jr
