// Phase-point functions in the reference's spherical layout (src/hawaii.h:210-284):
// the kinetic energy (src/hawaii.c:1041-1137) and the potential of one phase point,
// shared by the sampler (hh_sampler.cuh) and the VEGAS integrands (hh_vegas.cuh).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "hh_consts.h"
#include "hh_internal.h"
#include "hh_physics.cuh"
#include "hh_traj.cuh"

namespace hh {

struct SamplerArgs {
  int sys;
  double mu, II;
  double T;
  double Rmin, Rmax, pesmin;
  int pair_state;  // 1 free+metastable, 2 bound, 3 all
  SamplerExtra x;
};

// kinetic energy (src/hawaii.c:1041-1137) and potential for one phase point
__device__ __forceinline__ double kinetic(const SamplerArgs &a, const double *qp) {
  double mu = a.mu;
  double pPhi = qp[1], Theta = qp[2], pTheta = qp[3], R = qp[4], pR = qp[5];
  double sT = sin(Theta);
  double K = pR * pR / (2.0 * mu) + pTheta * pTheta / (2.0 * mu * R * R) +
             pPhi * pPhi / (2.0 * mu * R * R * sT * sT);
  if (a.sys == SYS_CH4CO2) {
    // ROTOR (src/hawaii.c:1090-1110), then the LINEAR_MOLECULE (1119-1127)
    const double *II = a.x.II1;
    double pphi1t = qp[7], theta = qp[8], ptheta1t = qp[9], psi = qp[10], ppsi1t = qp[11];
    double sin_theta = sin(theta), cos_theta = cos(theta), sin_psi = sin(psi), cos_psi = cos(psi);
    double t1 = (pphi1t - ppsi1t * cos_theta) * sin_psi + ptheta1t * sin_theta * cos_psi;
    double t2 = (pphi1t - ppsi1t * cos_theta) * cos_psi - ptheta1t * sin_theta * sin_psi;
    K += t1 * t1 / (2.0 * II[0] * sin_theta * sin_theta) + t2 * t2 / (2.0 * II[1] * sin_theta * sin_theta) +
         ppsi1t * ppsi1t / (2.0 * II[2]);
    double I = a.II, pphi = qp[13], th = qp[14], pth = qp[15];
    double s = sin(th);
    K += pth * pth / (2.0 * I) + pphi * pphi / (2.0 * I * s * s);
  } else if (a.sys != SYS_HEAR) {
    double I = a.II, pphi = qp[7], th = qp[8], pth = qp[9];
    double s = sin(th);
    K += pth * pth / (2.0 * I) + pphi * pphi / (2.0 * I * s * s);
  }
  return K;
}

__device__ __forceinline__ double potential(const SamplerArgs &a, const Co2arTables<double> *tb,
                                            const double *qp) {
  if (a.sys == SYS_HEAR) {
    double V, dV;
    hear_V_dV<double>(qp[4], 1.0 / qp[4], V, dV);
    return V;
  }
  if (a.sys == SYS_CH4CO2) {
    double y[19], M[3][3];
    ch4co2_qp_to_state(qp, a.x.II1, y);
    quat_matrix<double>(y + 6, M);
    return ch4co2_lj<double>(a.x.lj, M, y, y + 10).V;
  }
  double y[12];
  qp_to_state<SYS_CO2AR>(qp, y);
  if (a.sys == SYS_N2AR) {
    // N1 = +L/2 u^, N2 = -L/2 u^ (lab_to_xyz, ai_pes_n2_ar_pip_nn.cpp:103-121)
    const double h = N2AR_L / 2.0;
    double d1 = 0.0, d2 = 0.0;
    for (int c = 0; c < 3; ++c) {
      const double e1 = y[c] - h * y[6 + c], e2 = y[c] + h * y[6 + c];
      d1 += e1 * e1;
      d2 += e2 * e2;
    }
    return n2ar_pes_energy<double>(sqrt(d1), sqrt(d2));
  }
  double R = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
  double x = (y[0] * y[6] + y[1] * y[7] + y[2] * y[8]) / R;
  double V, VR, Vx;
  co2ar_pes<double, false>(tb->pes, tb->fpes, tb->rbound, tb->rlo, R, 1.0 / R, x, V, VR, Vx, true);
  return V;
}

}  // namespace hh
