// Device physics for the trajectory hot path: potential-energy gradients and
// induced dipoles of the supported pairs, written in Cartesian vector form.
//
// The reference integrates Hamilton's equations in spherical coordinates
// (src/hawaii.c:474-616) and evaluates its plugins through a lab->molecular
// frame transform with acos/atan2 and 3x3 Euler chains
// (src/angles_handler.cpp:106-193, PES-IDS/ai_pes_co2ar_lib.cpp:11-30,
// PES-IDS/ai_ids_co2ar_lib.cpp:12-37).  Here the state is
//   atom-atom:    y = (r[3], p[3])                     (relative position, momentum)
//   linear-atom:  y = (r[3], p[3], u[3], j[3])         (+ rotor axis, rotor angular momentum)
// and every surface is evaluated from R = |r| and x = cos(theta_mol) = (r/R).u,
// which needs no inverse trigonometry and has no coordinate poles.
//   dr/dt = p/mu,  dp/dt = -dV/dr,  du/dt = (j x u)/I,  dj/dt = -(u x dV/du).
// With V = V(R, x):  dV/dr = V_R r^ + V_x (u - x r^)/R,  u x dV/du = V_x (u x r^).
// The body-frame dipole (d_x, 0, d_z) of the reference, with d_x = sum a_l P_l^1
// and the Condon-Shortley phase, is d_z r^ - (sum a_l P_l'(x)) (u - x r^) in the lab.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_consts.h"

namespace hh {

// Paired FP32 arithmetic of sm_100: one instruction computes both halves of a float2,
// each half rounded as the scalar operation would be.  Kernels bound by instruction
// issue (the sample and M0 kernels) put pairs of independent operations through as one.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }

// ----------------------------------------------------------------------------
// He-Ar (PES-IDS/HeAr.h:33-107): exponential repulsion + damped dispersion
// V = A exp(-g1 R - g2 R^2) - sum_{n=3..8} C_2n f_2n(bR) / R^2n,
// f_2n(x) = 1 - exp(-x) sum_{k<=2n} x^k/k!.
// ----------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void hear_V_dV(T R, T iR, T &V, T &dV) {
  const T A = T(0.2303058634e2), G1 = T(0.163051044e1), G2 = T(0.4680016e-1);
  const T B = T(0.16274792500000e1);
  const T C[6] = {T(0.940835513e1), T(0.165523018e3), T(0.379715796e4),
                  T(0.1165179999e6), T(0.466258000e7), T(0.236861000e9)};
  T x = B * R;
  T ex = exp(-x);
  T rep = A * exp(-G1 * R - G2 * R * R);
  V = rep;
  dV = rep * (-G1 - T(2) * G2 * R);
  // S = sum_{k<=2n} x^k/k!, term = x^2n/(2n)!
  T term = T(1), S = T(1);
#pragma unroll
  for (int m = 1; m <= 4; ++m) {
    term *= x * T(1.0 / double(m));
    S += term;
  }
  T iR2 = iR * iR;
  T iRp = iR2 * iR2;  // R^-4, multiplied up to R^-2n
#pragma unroll
  for (int n = 3; n <= 8; ++n) {
    term *= x * T(1.0 / double(2 * n - 1));
    S += term;
    term *= x * T(1.0 / double(2 * n));
    S += term;
    iRp *= iR2;
    T f = T(1) - ex * S;
    T fp = B * ex * term;
    V -= C[n - 3] * f * iRp;
    dV -= C[n - 3] * (fp * iRp - T(2 * n) * f * iRp * iR);
  }
}

template <typename T>
__device__ __forceinline__ T hear_dip(T R, T iR) {
  T iR2 = iR * iR;
  T iR7 = iR2 * iR2 * iR2 * iR;
  return exp(T(0.47293181) - T(0.40100613) * R - T(0.10292726) * R * R) - T(148.55391) * iR7;
}

// ----------------------------------------------------------------------------
// CO2-Ar surfaces (PES-IDS/ai_pes_co2ar.c, PES-IDS/ai_ids_co2ar.cpp) from the
// generated tables: per R-interval and per l = 0,2,..,10 a radial function
//   c(R) = a0 + a1 t + a2 t^2 + a3 t^3 (t = R - R_lo) + sum_p b_p R^-p + A exp(k R)
// Rows are stored as 10 reals: a0 a1 a2 a3 b4 b5 b6 b7 A k.
// ----------------------------------------------------------------------------
constexpr int CO2AR_NINT = 32;
constexpr int CO2AR_NL = 6;
constexpr int CO2AR_ROW = 10;
constexpr int CO2AR_TABLE = CO2AR_NINT * CO2AR_NL * CO2AR_ROW;

// interval index with the reference's `R < bound` semantics (all bounds are
// exactly representable in FP32 and FP64)
template <typename T>
__device__ __forceinline__ int co2ar_interval(T R, const T *rbound) {
  int i;
  if (R < T(4.5)) i = 0;
  else if (R < T(10)) i = 1 + (int)((R - T(4.5)) * T(4));
  else if (R < T(12)) i = 23 + (int)(R - T(10));
  else if (R < T(20)) i = 25 + (int)((R - T(12)) * T(0.5));
  else if (R < T(25)) i = 29;
  else if (R < T(30)) i = 30;
  else i = 31;
  // exact correction against the bounds (guards any rounding of the arithmetic)
  while (i < CO2AR_NINT - 1 && !(R < rbound[i])) ++i;
  while (i > 0 && !(R >= rbound[i - 1])) --i;
  return i;
}

// interval flags: bit0 inverse powers present, bit1 exponential present
template <typename T>
__device__ __forceinline__ void radial(const T *row, T R, T t, T iR, int flags, T &c, T &dc) {
  c = ((row[3] * t + row[2]) * t + row[1]) * t + row[0];
  dc = (T(3) * row[3] * t + T(2) * row[2]) * t + row[1];
  if (flags & 1) {
    T iR2 = iR * iR;
    T iR4 = iR2 * iR2, iR5 = iR4 * iR, iR6 = iR5 * iR, iR7 = iR6 * iR;
    c += row[4] * iR4 + row[5] * iR5 + row[6] * iR6 + row[7] * iR7;
    dc -= (T(4) * row[4] * iR4 + T(5) * row[5] * iR5 + T(6) * row[6] * iR6 + T(7) * row[7] * iR7) * iR;
  }
  if (flags & 2) {
    T e = row[8] * exp(row[9] * R);
    c += e;
    dc += row[9] * e;
  }
}

template <typename T>
__device__ __forceinline__ T radial_value(const T *row, T R, T t, T iR, int flags) {
  T c = ((row[3] * t + row[2]) * t + row[1]) * t + row[0];
  if (flags & 1) {
    T iR2 = iR * iR;
    T iR4 = iR2 * iR2, iR5 = iR4 * iR, iR6 = iR5 * iR, iR7 = iR6 * iR;
    c += row[4] * iR4 + row[5] * iR5 + row[6] * iR6 + row[7] * iR7;
  }
  if (flags & 2) c += row[8] * exp(row[9] * R);
  return c;
}

// 1/sqrt: hardware estimate refined to ~1 ulp in FP32, CUDA's rsqrt in FP64
__device__ __forceinline__ float inv_sqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double inv_sqrt(double x) { return rsqrt(x); }

// compensated (Kahan-Babuska) accumulation, used by the FP32 M0 integrand
template <typename T> struct Acc {
  T s, c;
  __device__ __forceinline__ Acc() : s(0), c(0) {}
  __device__ __forceinline__ void add(T v, bool comp) {
    if (comp) {
      T t = s + v;
      if (fabs(s) >= fabs(v)) c += (s - t) + v;
      else c += (v - t) + s;
      s = t;
    } else {
      s += v;
    }
  }
  __device__ __forceinline__ T get() const { return s + c; }
};

// Legendre P_l(x), P_l'(x), l = 0..10 (only even l are consumed)
template <typename T>
__device__ __forceinline__ void legendre10(T x, T P[11], T dP[11]) {
  P[0] = T(1);
  P[1] = x;
  dP[0] = T(0);
  dP[1] = T(1);
#pragma unroll
  for (int l = 1; l < 10; ++l) {
    P[l + 1] = (T(2 * l + 1) * x * P[l] - T(l) * P[l - 1]) * T(1.0 / double(l + 1));
    dP[l + 1] = dP[l - 1] + T(2 * l + 1) * P[l];
  }
}

// V (Hartree) and its partial derivatives V_R, V_x at (R, x)
template <typename T, bool COMP>
__device__ __forceinline__ void co2ar_pes(const T *tab, const int *flags, const T *rbound,
                                          const T *rlo, T R, T iR, T x, T &V, T &VR, T &Vx,
                                          bool want_V) {
  int i = co2ar_interval<T>(R, rbound);
  T P[11], dP[11];
  legendre10(x, P, dP);
  T t = R - rlo[i];
  int fl = flags[i];
  Acc<T> aV, aR, ax;
  const T *base = tab + i * CO2AR_NL * CO2AR_ROW;
#pragma unroll
  for (int li = 0; li < CO2AR_NL; ++li) {
    T c, dc;
    radial<T>(base + li * CO2AR_ROW, R, t, iR, fl, c, dc);
    if (want_V) aV.add(P[2 * li] * c, COMP);
    aR.add(P[2 * li] * dc, COMP);
    ax.add(dP[2 * li] * c, COMP);
  }
  const T s = T(1.0 / HH_HTOCM);
  V = aV.get() * s;
  VR = aR.get() * s;
  Vx = ax.get() * s;
}

// V (Hartree) alone at (R, x): the sums of co2ar_pes without the derivatives
template <typename T, bool COMP>
__device__ __forceinline__ T co2ar_pes_value(const T *tab, const int *flags, const T *rbound, const T *rlo, T R,
                                             T iR, T x) {
  int i = co2ar_interval<T>(R, rbound);
  T P[11], dP[11];
  legendre10(x, P, dP);
  T t = R - rlo[i];
  int fl = flags[i];
  Acc<T> aV;
  const T *base = tab + i * CO2AR_NL * CO2AR_ROW;
#pragma unroll
  for (int li = 0; li < CO2AR_NL; ++li) aV.add(P[2 * li] * radial_value<T>(base + li * CO2AR_ROW, R, t, iR, fl), COMP);
  return aV.get() * T(1.0 / HH_HTOCM);
}

// body-frame dipole sums: dz = sum b_l P_l(x), ax = sum a_l P_l'(x)
template <typename T, bool COMP>
__device__ __forceinline__ void co2ar_dip(const T *tabx, const T *tabz, const int *flags,
                                          const T *rbound, const T *rlo, T R, T iR, T x, T &dz,
                                          T &ax) {
  int i = co2ar_interval<T>(R, rbound);
  T P[11], dP[11];
  legendre10(x, P, dP);
  T t = R - rlo[i];
  int fl = flags[i];
  Acc<T> az, aa;
  const T *bx = tabx + i * CO2AR_NL * CO2AR_ROW;
  const T *bz = tabz + i * CO2AR_NL * CO2AR_ROW;
#pragma unroll
  for (int li = 0; li < CO2AR_NL; ++li) {
    T a = radial_value<T>(bx + li * CO2AR_ROW, R, t, iR, fl);
    T b = radial_value<T>(bz + li * CO2AR_ROW, R, t, iR, fl);
    az.add(P[2 * li] * b, COMP);
    aa.add(dP[2 * li] * a, COMP);
  }
  dz = az.get();
  ax = aa.get();
}

}  // namespace hh
