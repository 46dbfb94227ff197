// CH4-CO2 (ROTOR + LINEAR_MOLECULE) on the device: Cartesian equations of motion
// and the stand-in site-site surface of hh_ch4co2_standin.h.
//
// State y (19): r (CO2 centre minus CH4 centre), p, the unit quaternion (w, x, y, z)
// of the CH4 body -> lab rotation M, the CO2 axis u, the CH4 lab angular momentum
// L and the CO2 angular momentum j, all in the reference's lab frame.  These are
// the reference's Euler-angle equations (rhsMonomer ROTOR / LINEAR_MOLECULE and
// the intermolecular part of rhs, src/hawaii.c:474-616) written without angles:
//   dr/dt = p / mu,              dp/dt = -dV/dr
//   dq/dt = (0, w) q / 2,        w = M diag(1/I) M^T L      (lab angular velocity)
//   dL/dt = sum_s x_s x (-dV/dx_s)   (CH4 sites x_s relative to the CH4 centre)
//   du/dt = (j x u) / I_CO2,     dj/dt = -u x dV/du
// with no coordinate singularity at theta = 0 or pi.
//
// The dipole is not evaluated here: a CH4-CO2 sample is written out as a
// record (r, q, u) and evaluated by the batched kernels of hh_ch4co2_dip.cuh.
#pragma once

#include <cuda_runtime.h>

#include "hh_ch4co2_standin.h"
#include "hh_physics.cuh"

namespace hh {

// A = 4 eps sigma^12 and B = 4 eps sigma^6 of the four site-class pairs
// ([CH4 class C, H][CO2 class C, O]), from hh_ch4co2_lj_pairs on the host
struct Ch4Co2Lj {
  double A[2][2], B[2][2];
};

// body -> lab rotation matrix of a quaternion (normalised here)
template <typename T> __device__ __forceinline__ void quat_matrix(const T *q, T M[3][3]) {
  const T n = inv_sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const T w = q[0] * n, x = q[1] * n, y = q[2] * n, z = q[3] * n;
  M[0][0] = T(1) - T(2) * (y * y + z * z);
  M[0][1] = T(2) * (x * y - w * z);
  M[0][2] = T(2) * (x * z + w * y);
  M[1][0] = T(2) * (x * y + w * z);
  M[1][1] = T(1) - T(2) * (x * x + z * z);
  M[1][2] = T(2) * (y * z - w * x);
  M[2][0] = T(2) * (x * z - w * y);
  M[2][1] = T(2) * (y * z + w * x);
  M[2][2] = T(1) - T(2) * (x * x + y * y);
}

// Site-site surface: V, the gradient Gr = dV/dr, the CH4 torque tau = sum_s x_s x (-dV/dx_s)
// and Gu = dV/du, from the CH4 rotation M (body -> lab), r and the unit CO2 axis u.
template <typename T> struct Ch4Co2Grad {
  T V, Gr[3], tau[3], Gu[3];
};
template <typename T>
__device__ __noinline__ Ch4Co2Grad<T> ch4co2_lj(const Ch4Co2Lj &lj, const T (&M)[3][3], const T *r,
                                                 const T *u) {
  const T a = T(HH_CH4CO2_RCH / 1.7320508075688772);
  const T rco = T(HH_CH4CO2_RCO);
  // H sites a (+-c0 +-c1 +-c2) with c_k the columns of M (body axes in the lab frame)
  T xs[5][3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T c0 = M[i][0] * a, c1 = M[i][1] * a, c2 = M[i][2] * a;
    xs[0][i] = T(0);
    xs[1][i] = c0 + c1 + c2;
    xs[2][i] = c0 - c1 - c2;
    xs[3][i] = -c0 + c1 - c2;
    xs[4][i] = -c0 - c1 + c2;
  }
  Ch4Co2Grad<T> g;
  g.V = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) g.Gr[i] = g.tau[i] = g.Gu[i] = T(0);
#pragma unroll
  for (int t = 0; t < 3; ++t) {
    const T sgn = (t == 0) ? T(0) : (t == 1 ? T(1) : T(-1));
    const T xt[3] = {r[0] + sgn * rco * u[0], r[1] + sgn * rco * u[1], r[2] + sgn * rco * u[2]};
    T Gt[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const T A = T(lj.A[s ? 1 : 0][t ? 1 : 0]), B = T(lj.B[s ? 1 : 0][t ? 1 : 0]);
      const T dx[3] = {xt[0] - xs[s][0], xt[1] - xs[s][1], xt[2] - xs[s][2]};
      const T i2 = T(1) / (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      const T i6 = i2 * i2 * i2;
      g.V += i6 * (A * i6 - B);
      const T f = -(T(12) * A * i6 - T(6) * B) * i6 * i2;  // (dV/dd) / d
      const T gx[3] = {f * dx[0], f * dx[1], f * dx[2]};
#pragma unroll
      for (int i = 0; i < 3; ++i) Gt[i] += gx[i];
      if (s) {  // torque of -dV/dx_s = +gx on the H site
        g.tau[0] += xs[s][1] * gx[2] - xs[s][2] * gx[1];
        g.tau[1] += xs[s][2] * gx[0] - xs[s][0] * gx[2];
        g.tau[2] += xs[s][0] * gx[1] - xs[s][1] * gx[0];
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      g.Gr[i] += Gt[i];
      g.Gu[i] += sgn * rco * Gt[i];
    }
  }
  return g;
}

template <typename PHYS, typename STG, bool COMP, bool SOLO_ = false> struct Ch4Co2Sys {
  static constexpr bool SOLO = SOLO_;  // the solo kernel's instance
  static constexpr int N = 19;
  static constexpr int QP = 16;
  // components a sample reads: r, the quaternion and u
  static constexpr int NQ = 10;
  static constexpr bool RECORDS = true;
  static constexpr bool EST64 = false;
  static constexpr int MOM2 = 13;  // L and j follow the orientation block
  static __device__ __forceinline__ constexpr int qidx(int i) { return i < 3 ? i : i + 3; }
  double inv_mu, inv_II;      // 1 / mu, 1 / I_CO2
  double inv_I1[3];           // 1 / principal moments of CH4
  Ch4Co2Lj lj;
  template <typename YT> __device__ void rhs(const YT *y, STG *f) const {
    const PHYS r[3] = {PHYS(y[0]), PHYS(y[1]), PHYS(y[2])};
    const PHYS qt[4] = {PHYS(y[6]), PHYS(y[7]), PHYS(y[8]), PHYS(y[9])};
    const PHYS u[3] = {PHYS(y[10]), PHYS(y[11]), PHYS(y[12])};
    const PHYS iu = inv_sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const PHYS uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    PHYS M[3][3];
    quat_matrix<PHYS>(qt, M);
    const Ch4Co2Grad<PHYS> g = ch4co2_lj<PHYS>(lj, M, r, uh);
    // lab angular velocity of CH4: M diag(1/I) M^T L
    const PHYS L[3] = {PHYS(y[13]), PHYS(y[14]), PHYS(y[15])};
    PHYS wb[3], w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) wb[k] = (M[0][k] * L[0] + M[1][k] * L[1] + M[2][k] * L[2]) * PHYS(inv_I1[k]);
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = M[i][0] * wb[0] + M[i][1] * wb[1] + M[i][2] * wb[2];
    const STG im = STG(inv_mu), iI = STG(inv_II);
    f[0] = STG(y[3]) * im;
    f[1] = STG(y[4]) * im;
    f[2] = STG(y[5]) * im;
#pragma unroll
    for (int i = 0; i < 3; ++i) f[3 + i] = STG(-g.Gr[i]);
    // dq/dt = (0, w) q / 2 on the quaternion as integrated (its norm is an invariant)
    const STG hw[3] = {STG(0.5) * STG(w[0]), STG(0.5) * STG(w[1]), STG(0.5) * STG(w[2])};
    const STG q0 = STG(y[6]), q1 = STG(y[7]), q2 = STG(y[8]), q3 = STG(y[9]);
    f[6] = -(hw[0] * q1 + hw[1] * q2 + hw[2] * q3);
    f[7] = hw[0] * q0 + hw[1] * q3 - hw[2] * q2;
    f[8] = hw[1] * q0 + hw[2] * q1 - hw[0] * q3;
    f[9] = hw[2] * q0 + hw[0] * q2 - hw[1] * q1;
    const STG u0 = STG(y[10]), u1 = STG(y[11]), u2 = STG(y[12]);
    const STG j0 = STG(y[16]), j1 = STG(y[17]), j2 = STG(y[18]);
    f[10] = (j1 * u2 - j2 * u1) * iI;
    f[11] = (j2 * u0 - j0 * u2) * iI;
    f[12] = (j0 * u1 - j1 * u0) * iI;
#pragma unroll
    for (int i = 0; i < 3; ++i) f[13 + i] = STG(g.tau[i]);
    // dj/dt = -u^ x dV/du
    f[16] = STG(-(uh[1] * g.Gu[2] - uh[2] * g.Gu[1]));
    f[17] = STG(-(uh[2] * g.Gu[0] - uh[0] * g.Gu[2]));
    f[18] = STG(-(uh[0] * g.Gu[1] - uh[1] * g.Gu[0]));
  }
  // samples are written as records; no dipole on this path
  __device__ void dipole(const double *, PHYS d[3]) const { d[0] = d[1] = d[2] = PHYS(0); }
};

// Euler phase point of the reference (PHI pPHI THETA pTHETA R pR | phi1 pphi1 theta1
// ptheta1 psi1 ppsi1 | phi2 pphi2 theta2 ptheta2) -> the 19 Cartesian components
__device__ __forceinline__ void ch4co2_qp_to_state(const double *qp, const double *II1, double *y) {
  const double Phi = qp[0], pPhi = qp[1], Th = qp[2], pTh = qp[3], R = qp[4], pR = qp[5];
  double sT, cT, sP, cP;
  sincos(Th, &sT, &cT);
  sincos(Phi, &sP, &cP);
  // r^ = Sz(PHI)^T Sy_ns(THETA)^T z (src/angles_handler.cpp:396)
  const double rh[3] = {-sT * cP, -sT * sP, cT};
  const double eT[3] = {-cT * cP, -cT * sP, -sT};
  const double eP[3] = {sP, -cP, 0.0};
  const double a = pTh / R, b = pPhi / (R * sT);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    y[i] = R * rh[i];
    y[3 + i] = pR * rh[i] + a * eT[i] + b * eP[i];
  }
  // CH4: S1 = Sz(psi) Sx(theta) Sz(phi) (lab -> body); M = S1^T = Rz(phi) Rx(theta) Rz(psi)
  const double phi = qp[6], pphi = qp[7], th = qp[8], pth = qp[9], psi = qp[10], ppsi = qp[11];
  double sa, ca, sb, cb, sc, cc;
  sincos(0.5 * phi, &sa, &ca);
  sincos(0.5 * th, &sb, &cb);
  sincos(0.5 * psi, &sc, &cc);
  // (ca, 0, 0, sa) (cb, sb, 0, 0) (cc, 0, 0, sc)
  const double t0 = ca * cb, t1 = ca * sb, t2 = sa * sb, t3 = sa * cb;
  y[6] = t0 * cc - t3 * sc;
  y[7] = t1 * cc + t2 * sc;
  y[8] = t2 * cc - t1 * sc;
  y[9] = t0 * sc + t3 * cc;
  double st, ct, sp, cp;
  sincos(th, &st, &ct);
  sincos(psi, &sp, &cp);
  // body angular momentum of the rotor's kinetic energy (src/hawaii.c:1090-1110)
  const double Lb[3] = {((pphi - ppsi * ct) * sp + pth * st * cp) / st,
                        ((pphi - ppsi * ct) * cp - pth * st * sp) / st, ppsi};
  double M[3][3];
  quat_matrix<double>(y + 6, M);
#pragma unroll
  for (int i = 0; i < 3; ++i) y[13 + i] = M[i][0] * Lb[0] + M[i][1] * Lb[1] + M[i][2] * Lb[2];
  (void)II1;
  // CO2: u = Sz(phi2)^T Sy_ns(theta2)^T z, j = u x p_u (src/angles_handler.cpp:408)
  const double ph2 = qp[12], pph2 = qp[13], th2 = qp[14], pth2 = qp[15];
  double s2, c2, sp2, cp2;
  sincos(th2, &s2, &c2);
  sincos(ph2, &sp2, &cp2);
  const double u[3] = {-s2 * cp2, -s2 * sp2, c2};
  const double u_th[3] = {-c2 * cp2, -c2 * sp2, -s2};
  const double u_ph[3] = {s2 * sp2, -s2 * cp2, 0.0};
  double pu[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) pu[i] = pth2 * u_th[i] + pph2 / (s2 * s2) * u_ph[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) y[10 + i] = u[i];
  y[16] = u[1] * pu[2] - u[2] * pu[1];
  y[17] = u[2] * pu[0] - u[0] * pu[2];
  y[18] = u[0] * pu[1] - u[1] * pu[0];
}

}  // namespace hh
