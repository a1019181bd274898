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
  P.c_cr1 = d->c_cr1;
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

// cl, cd, cm, cd_friction from the per-face wall loads (7 each) and the faces' midpoints
// (src/jaxrans/post/forces.py:108-161, 3D: lift and drag in the x-z plane)
inline void force_coefficients3(const Physics3& P, int n_walls, const double* loads, const double* mid, double area,
                                double length, const double* centre, double out[4]) {
  const double* q = P.q_inf;
  const double speed = sqrt((q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]);
  const double drag[3] = {q[1] / speed, q[2] / speed, q[3] / speed};
  const double lift[3] = {-drag[2], 0.0, drag[0]};
  const double q_area = 0.5 * q[0] * speed * speed * area;
  double cl = 0.0, cd = 0.0, cm = 0.0, shear[3] = {0.0, 0.0, 0.0};
  for (int w = 0; w < n_walls; ++w) {
    const double* L = loads + (size_t)7 * w;
    double load[3];
    for (int m = 0; m < 3; ++m) {
      load[m] = -L[0] * L[1 + m] + L[4 + m];
      shear[m] = shear[m] + L[4 + m];
    }
    cl = cl + ((lift[0] * load[0] + lift[1] * load[1]) + lift[2] * load[2]);
    cd = cd + ((drag[0] * load[0] + drag[1] * load[1]) + drag[2] * load[2]);
    const double rx = mid[3 * w] - centre[0], rz = mid[3 * w + 2] - centre[2];
    cm = cm + (rz * load[0] - rx * load[2]) / length;
  }
  out[0] = cl / q_area;
  out[1] = cd / q_area;
  out[2] = cm / q_area;
  out[3] = ((drag[0] * shear[0] + drag[1] * shear[1]) + drag[2] * shear[2]) / q_area;
}

}  // namespace jr
