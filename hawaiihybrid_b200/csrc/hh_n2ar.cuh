// N2-Ar PIP-NN surfaces on the device.
//
// PES (PES-IDS/ai_pes_n2_ar_pip_nn.cpp:8-146, PES-IDS/mlp.hpp:178-256): the
// three site distances |N1-N2| (fixed, rigid rotor), d1 = |N1-Ar|, d2 = |N2-Ar|
// map to y = exp(-d/2), switched to 1e4/d^6 on [6, 20] bohr for the N-Ar pairs,
// then to 17 permutationally invariant polynomials (PIPs), a standard scaler, a
// 17-32-1 SiLU network and an inverse scaler (cm^-1).  The kernels need dE/dd1
// and dE/dd2 (the network's backward pass); the sampler and M0 need E.  The
// network is unrolled over the constexpr tables of hh_n2ar_tables.h, so every
// weight is a compile-time constant operand, and the function is called out of
// line (one copy per kernel).
//
// Dipole (PES-IDS/ai_ids_n2_ar_pip_nn.cpp:11-128, PES-IDS/QModel.hpp:144-257):
// five sites N1, N2 = -N1, N1', N2' = -N1' (the effective-quadrupole sites,
// perpendicular to the N2 axis) and Ar; charges from 308 PIPs of y = exp(-d/a0)
// of the 10 site distances through three SiLU sub-networks, minus the charges
// at infinite separation; the dipole is sum q_i x_i, blended between the short-
// (a0 = 2) and long-range (a0 = 6) models on R in [9.5, 12.5] bohr.  The kernels
// evaluate the exact refolding of hh_n2ar_fold.h in FP64 on both precision
// paths: the charges relative to infinity are small differences of O(0.1)
// network outputs, which FP32 resolves only to about 5e-4 of the dipole.
#pragma once

#include <cuda_runtime.h>

#include "hh_consts.h"
#include "hh_n2ar_fold.h"
#include "hh_n2ar_tables.h"

namespace hh {

constexpr double N2AR_L = 2.07856749;                 // src/constants.h:80
constexpr double N2AR_EN_INF = 0.0384490895371528;    // ai_pes_n2_ar_pip_nn.cpp:130, cm^-1

template <typename T> __device__ __forceinline__ T n2ar_silu(T x) { return x / (T(1) + exp(-x)); }

// quintic switch 10r^3 - 15r^4 + 6r^5 on [xi, xf] and its derivative
template <typename T> __device__ __forceinline__ T n2ar_switch(T x, T xi, T xf) {
  if (x < xi) return T(0);
  if (x < xf) {
    const T r = (x - xi) / (xf - xi), r3 = r * r * r, r4 = r3 * r, r5 = r4 * r;
    return T(10) * r3 - T(15) * r4 + T(6) * r5;
  }
  return T(1);
}

// y(d) of an N-Ar pair and dy/dd (ai_pes_n2_ar_pip_nn.cpp:43-101)
template <typename T> __device__ __forceinline__ void n2ar_pair_y(T d, T &y, T &dy) {
  const T xi = T(6), xf = T(20);
  const T e = exp(-d / T(2));
  if (d < xi) {
    y = e;
    dy = -e / T(2);
    return;
  }
  const T d2 = d * d, d6 = d2 * d2 * d2, d7 = d6 * d;
  if (d < xf) {
    const T w = xf - xi, r = (d - xi) / w, r2 = r * r, r3 = r2 * r, r4 = r3 * r, r5 = r4 * r;
    const T s = T(10) * r3 - T(15) * r4 + T(6) * r5;
    const T ds = (T(30) * r2 - T(60) * r3 + T(30) * r4) / w;
    y = (T(1) - s) * e + s * T(1e4) / d6;
    dy = -ds * e - (T(1) - s) * e / T(2) + ds * T(1e4) / d6 - s * T(6e4) / d7;
  } else {
    y = T(1e4) / d6;
    dy = -T(6e4) / d7;
  }
}

// PES network: E (cm^-1, before the en_inf shift) and, with GRAD, dE/dy1 and
// dE/dy2 (mlp.hpp:178-256: forward, then backward through the hidden layer and
// the PIP Jacobian).  y0 = exp(-|N1-N2|/2) is fixed by the rigid rotor.
template <typename T, bool GRAD>
__device__ __forceinline__ T n2ar_pes_net(T y1, T y2, T *gy) {
  constexpr int NP = HH_N2AR_PES_NPIP, NH = HH_N2AR_PES_HIDDEN;
  const T y[3] = {exp(-T(N2AR_L) / T(2)), y1, y2};
  T p[NP], j1[NP], j2[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) p[i] = j1[i] = j2[i] = T(0);
#pragma unroll
  for (int m = 0; m < HH_N2AR_PES_NMONO; ++m) {
    const int pi = hh_n2ar_pes_poly[m];
    T prod = T(1);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (hh_n2ar_pes_var[m][k] >= 0) prod *= y[hh_n2ar_pes_var[m][k]];
    p[pi] += prod;
    if (GRAD) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int vk = hh_n2ar_pes_var[m][k];
        if (vk == 1 || vk == 2) {
          T d = T(1);
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if (i != k && hh_n2ar_pes_var[m][i] >= 0) d *= y[hh_n2ar_pes_var[m][i]];
          if (vk == 1) j1[pi] += d;
          else j2[pi] += d;
        }
      }
    }
  }
  T ptr[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) ptr[i] = (p[i] - T(hh_n2ar_pes_xmean[i])) * T(1.0 / hh_n2ar_pes_xscale[i]);
  T out = T(hh_n2ar_pes_b1[0]);
  T g[NH];
#pragma unroll
  for (int j = 0; j < NH; ++j) {
    T h = T(hh_n2ar_pes_b0[j]);
#pragma unroll
    for (int i = 0; i < NP; ++i) h += ptr[i] * T(hh_n2ar_pes_w0[i][j]);
    const T e = exp(-h), r = T(1) / (T(1) + e);
    out += h * r * T(hh_n2ar_pes_w1[j]);
    if (GRAD) g[j] = r * (T(1) + h * e * r) * T(hh_n2ar_pes_w1[j]);  // SiLU'(h) W1
  }
  if (GRAD) {
    T a1 = T(0), a2 = T(0);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      T a = T(0);
#pragma unroll
      for (int j = 0; j < NH; ++j) a += T(hh_n2ar_pes_w0[i][j]) * g[j];
      a *= T(1.0 / hh_n2ar_pes_xscale[i]);
      a1 += j1[i] * a;
      a2 += j2[i] * a;
    }
    gy[0] = a1 * T(hh_n2ar_pes_y[1]);
    gy[1] = a2 * T(hh_n2ar_pes_y[1]);
  }
  return T(hh_n2ar_pes_y[1]) * out + T(hh_n2ar_pes_y[0]);
}

template <typename T> struct N2arGrad {
  T g1, g2;  // dV/dd1, dV/dd2 in Hartree/bohr
};

// Arithmetic of the PES gradient with the rounding of every operation fixed
// (no contraction left to the compiler), so that the per-lane and the cooperative
// gradient below give bit-identical results.
__device__ __forceinline__ float n2_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double n2_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float n2_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double n2_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float n2_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double n2_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float n2_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double n2_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float n2_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double n2_div(double a, double b) { return __ddiv_rn(a, b); }

// y(d) of an N-Ar pair and dy/dd as n2ar_pair_y, with fixed rounding
template <typename T> __device__ __forceinline__ void n2ar_pair_y_rn(T d, T &y, T &dy) {
  const T e = exp(-n2_mul(d, T(0.5)));
  if (d < T(6)) {
    y = e;
    dy = -n2_mul(e, T(0.5));
    return;
  }
  const T d2 = n2_mul(d, d), d6 = n2_mul(n2_mul(d2, d2), d2), d7 = n2_mul(d6, d);
  const T a6 = n2_div(T(1e4), d6), a7 = n2_div(T(6e4), d7);
  if (d < T(20)) {
    const T w = T(14), r = n2_div(n2_sub(d, T(6)), w);
    const T r2 = n2_mul(r, r), r3 = n2_mul(r2, r), r4 = n2_mul(r3, r), r5 = n2_mul(r4, r);
    const T sw = n2_add(n2_sub(n2_mul(T(10), r3), n2_mul(T(15), r4)), n2_mul(T(6), r5));
    const T ds = n2_div(n2_add(n2_sub(n2_mul(T(30), r2), n2_mul(T(60), r3)), n2_mul(T(30), r4)), w);
    const T om = n2_sub(T(1), sw);
    y = n2_add(n2_mul(om, e), n2_mul(sw, a6));
    dy = n2_sub(n2_add(n2_sub(-n2_mul(ds, e), n2_mul(n2_mul(om, e), T(0.5))), n2_mul(ds, a6)), n2_mul(sw, a7));
  } else {
    y = a6;
    dy = -a7;
  }
}

// network inputs of the gradient: the scaled PIPs ptr_i = (p_i - mean_i) / scale_i
// and the PIP Jacobian dp_i/dy_1, dp_i/dy_2 (the monomial table unrolled)
template <typename T>
__device__ __forceinline__ void n2ar_grad_inputs(const N2arPesNet<T> *net, T d1, T d2, T (&ptr)[N2AR_PES_NP],
                                                 T (&j1)[N2AR_PES_NP], T (&j2)[N2AR_PES_NP], T &dy1, T &dy2) {
  constexpr int NP = N2AR_PES_NP;
  T y1, y2;
  n2ar_pair_y_rn(d1, y1, dy1);
  n2ar_pair_y_rn(d2, y2, dy2);
  const T y[3] = {exp(-T(N2AR_L) / T(2)), y1, y2};
  T p[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) p[i] = j1[i] = j2[i] = T(0);
#pragma unroll
  for (int m = 0; m < HH_N2AR_PES_NMONO; ++m) {
    const int pi = hh_n2ar_pes_poly[m];
    T prod = T(1);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (hh_n2ar_pes_var[m][k] >= 0) prod = n2_mul(prod, y[hh_n2ar_pes_var[m][k]]);
    p[pi] = n2_add(p[pi], prod);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int vk = hh_n2ar_pes_var[m][k];
      if (vk == 1 || vk == 2) {
        T d = T(1);
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (i != k && hh_n2ar_pes_var[m][i] >= 0) d = n2_mul(d, y[hh_n2ar_pes_var[m][i]]);
        if (vk == 1) j1[pi] = n2_add(j1[pi], d);
        else j2[pi] = n2_add(j2[pi], d);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < NP; ++i) ptr[i] = n2_mul(n2_sub(p[i], net->xmean[i]), net->ixscale[i]);
}

// SiLU'(h) W1 of one hidden unit
template <typename T> __device__ __forceinline__ T n2ar_unit_grad(T h, T w1) {
  const T e = exp(-h), r = n2_div(T(1), n2_add(T(1), e));
  return n2_mul(n2_mul(r, n2_add(T(1), n2_mul(n2_mul(h, e), r))), w1);
}

// dV/dd1, dV/dd2 (Hartree/bohr) for d1 = |N1-Ar|, d2 = |N2-Ar|, out of line.  The
// PIPs and their Jacobian are unrolled over the monomial table; the network is a
// runtime loop over the 32 hidden units (forward and backward in one pass) with
// the weights of `net` (shared memory in the kernels), so the code stays small.
// FP32: two hidden units per iteration with the paired FP32 instructions of sm_100,
// each half the scalar loop's fma chain in the same order (h_j over i, a_i over j), so
// the values are bit for bit those of the scalar loop and of n2ar_pes_grad_coop.
template <typename T>
__device__ __noinline__ N2arGrad<T> n2ar_pes_grad(const N2arPesNet<T> *net, T d1, T d2) {
  constexpr int NP = N2AR_PES_NP;
  T ptr[NP], j1[NP], j2[NP], a[NP + 1], dy1, dy2;
  n2ar_grad_inputs(net, d1, d2, ptr, j1, j2, dy1, dy2);
#pragma unroll
  for (int i = 0; i <= NP; ++i) a[i] = T(0);
  if constexpr (sizeof(T) == 4) {
    static_assert(N2AR_PES_NH % 2 == 0 && NP + 1 <= N2AR_PES_ROW, "unit pairs, input pairs within a row");
#pragma unroll 1
    for (int jp = 0; jp < N2AR_PES_NH / 2; ++jp) {
      const float2 *wp = reinterpret_cast<const float2 *>(net->w0p[jp]);
      float2 h = make_float2(net->b0[2 * jp], net->b0[2 * jp + 1]);
#pragma unroll
      for (int i = 0; i < NP; ++i) h = __ffma2_rn(make_float2(ptr[i], ptr[i]), wp[i], h);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int j = 2 * jp + b;
        const T g = n2ar_unit_grad(b == 0 ? h.x : h.y, net->w1[j]);
        const float2 *w = reinterpret_cast<const float2 *>(net->w0t[j]);
#pragma unroll
        for (int i = 0; i < NP; i += 2) {  // w0t[j][NP] is zero: a[NP] is never read
          const float2 r = __ffma2_rn(w[i / 2], make_float2(g, g), make_float2(a[i], a[i + 1]));
          a[i] = r.x;
          a[i + 1] = r.y;
        }
      }
    }
  } else {
#pragma unroll 1
    for (int j = 0; j < N2AR_PES_NH; ++j) {
      const T *w = net->w0t[j];
      T h = net->b0[j];
#pragma unroll
      for (int i = 0; i < NP; ++i) h = n2_fma(ptr[i], w[i], h);
      const T g = n2ar_unit_grad(h, net->w1[j]);
#pragma unroll
      for (int i = 0; i < NP; ++i) a[i] = n2_fma(w[i], g, a[i]);
    }
  }
  T a1 = T(0), a2 = T(0);
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const T ai = n2_mul(a[i], net->ixscale[i]);
    a1 = n2_fma(j1[i], ai, a1);
    a2 = n2_fma(j2[i], ai, a2);
  }
  const T s = n2_mul(net->yscale, T(1.0 / HH_HTOCM));
  return {n2_mul(n2_mul(a1, dy1), s), n2_mul(n2_mul(a2, dy2), s)};
}

// n2ar_pes_grad with the 32 lanes of a warp on one (d1, d2), bit for bit: every
// lane forms the network inputs, lane j evaluates hidden unit j (the same sum over
// the 17 inputs, in the same order), lane i < 17 forms a_i = sum_j W0[i][j] g_j
// over the units in the order of the per-lane loop from values shuffled out of the
// other lanes, and every lane sums j1_i a_i / xscale_i and j2_i a_i / xscale_i over
// i in order from the a_i shuffled out of lanes 0..16.  A trajectory therefore
// takes the same steps in the solo kernel as in the bulk kernel.  All 32 lanes
// call it with the same arguments.
template <typename T>
__device__ __noinline__ N2arGrad<T> n2ar_pes_grad_coop(const N2arPesNet<T> *net, T d1, T d2) {
  static_assert(N2AR_PES_NH == 32 && N2AR_PES_NP <= 32, "one hidden unit per lane");
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int NP = N2AR_PES_NP;
  T ptr[NP], j1[NP], j2[NP], dy1, dy2;
  n2ar_grad_inputs(net, d1, d2, ptr, j1, j2, dy1, dy2);
  const int lane = threadIdx.x & 31;
  const T *wt = net->w0t[lane];
  T h = net->b0[lane];
#pragma unroll
  for (int i = 0; i < NP; ++i) h = n2_fma(ptr[i], wt[i], h);
  const T g = n2ar_unit_grad(h, net->w1[lane]);
  const int ir = lane < NP ? lane : NP - 1;
  T a = T(0);
#pragma unroll
  for (int j = 0; j < N2AR_PES_NH; ++j) a = n2_fma(net->w0t[j][ir], __shfl_sync(FULL, g, j), a);
  T a1 = T(0), a2 = T(0);
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const T ai = n2_mul(__shfl_sync(FULL, a, i), net->ixscale[i]);
    a1 = n2_fma(j1[i], ai, a1);
    a2 = n2_fma(j2[i], ai, a2);
  }
  const T s = n2_mul(net->yscale, T(1.0 / HH_HTOCM));
  return {n2_mul(n2_mul(a1, dy1), s), n2_mul(n2_mul(a2, dy2), s)};
}

// V (Hartree) for d1 = |N1-Ar|, d2 = |N2-Ar| (pes_xyz, ai_pes_n2_ar_pip_nn.cpp:127-132)
template <typename T> __device__ __noinline__ T n2ar_pes_energy(T d1, T d2) {
  T y1, dy1, y2, dy2;
  n2ar_pair_y(d1, y1, dy1);
  n2ar_pair_y(d2, y2, dy2);
  const T e = n2ar_pes_net<T, false>(y1, y2, nullptr);
  return (e - T(N2AR_EN_INF)) * T(1.0 / HH_HTOCM);
}

template <typename T> struct N2arDipBody {
  T dx, dz;  // body-frame dipole: Ar on +z, the N2 axis in the xz plane at angle T
};

// body-frame dipole (FP64) at R (bohr) and c = cos T from the folded charge models
// F (shared memory in the kernels); dipole_bf and dipole_xyz of
// ai_ids_n2_ar_pip_nn.cpp:83-127.  Out of line.
static __device__ __noinline__ N2arDipBody<double> n2ar_dip_body(const N2arDipFold *F, double R,
                                                              double c) {
  const double h = N2AR_L / 2.0;
  const double s = sqrt(fmax(0.0, (1.0 - c) * (1.0 + c)));
  const double base = h * h + R * R, hc = 2.0 * h * c * R, hs = 2.0 * h * s * R;
  // the varying distances N1-Ar, N2-Ar, N1'-Ar, N2'-Ar
  const double dv[4] = {sqrt(base - hc), sqrt(base + hc), sqrt(base + hs), sqrt(base - hs)};
  const double sw = n2ar_switch(R, 9.5, 12.5);
  N2arDipBody<double> out = {0.0, 0.0};
#pragma unroll 1
  for (int m = 0; m < 2; ++m) {
    const double wm = (m == 0) ? 1.0 - sw : sw;
    if (wm == 0.0) continue;
    const double ia0 = (m == 0) ? 0.5 : 1.0 / 6.0;
    double v[4], z[N2AR_NZ];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = exp(-dv[i] * ia0);
    int k = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) z[k++] = v[i];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = i; j < 4; ++j) z[k++] = v[i] * v[j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = i; j < 4; ++j)
#pragma unroll
        for (int l = j; l < 4; ++l) z[k++] = v[i] * v[j] * v[l];
    double dh[N2AR_NH];
#pragma unroll
    for (int j = 0; j < N2AR_NH; ++j) dh[j] = 0.0;
    const double2 *W = reinterpret_cast<const double2 *>(&F->w[m][0][0]);
#pragma unroll 2
    for (int kk = 0; kk < N2AR_NZ; ++kk) {
      const double zk = z[kk];
#pragma unroll
      for (int j = 0; j < N2AR_NH / 2; ++j) {
        const double2 w2 = W[kk * (N2AR_NH / 2) + j];
        dh[2 * j] += zk * w2.x;
        dh[2 * j + 1] += zk * w2.y;
      }
    }
    double A = 0.0, B = 0.0, Q = 0.0;
#pragma unroll
    for (int j = 0; j < N2AR_NH; ++j) {
      const double d = dh[j], u = expm1(-d);
      const double e0 = F->e0[m][j];
      const double sd = 1.0 / (1.0 + (e0 + e0 * u));
      const double ds = sd * (d - F->c1[m][j] * u);
      const double t = ds * F->wo[m][j];
      if (j < 16) A += t;
      else if (j < 32) B += t;
      else Q += t;
    }
    out.dx += wm * (h * s * A + h * c * B);
    out.dz += wm * (h * c * A - h * s * B + R * Q);
  }
  return out;
}

// Mixed-path dipole table.  The body-frame dipole (d_x, d_z) of n2ar_dip_body is a
// smooth function of R and of the angle T in [0, pi] between r^ and u^ (the site
// distances are analytic in T; in x = cos T they are not, at x = +-1).  The mixed
// path replaces the network by a piecewise Chebyshev series of degree 9 in each
// variable on cells of
//   R: 0.5 bohr on [4.5, 12.5] (the switch edges 9.5 and 12.5 are cell edges),
//      1.5 bohr on [12.5, 20], 4 bohr on [20, 60];   T: 12 cells of pi/12,
// built on the device from the FP64 network at the Chebyshev nodes of every cell
// (n2ar_tab_build_kernel) and evaluated in FP32.  The series error is below 1.3e-9
// of the largest |d| at the same R (sampled against the network); FP32 evaluation
// adds about 1e-7.  Outside [4.5, 60) bohr the mixed path evaluates the network.
constexpr int N2T_DEG = 10;                 // Chebyshev coefficients per variable
constexpr int N2T_NR = 16 + 5 + 10;         // R cells
constexpr int N2T_NT = 12;                  // T cells
constexpr int N2T_CELLS = N2T_NR * N2T_NT;
constexpr int N2T_CELL_F4 = N2T_DEG * N2T_DEG / 2;  // float4 per cell: [i_R][j_T] (d_x, d_z) pairs
constexpr double N2T_RLO = 4.5, N2T_RHI = 60.0;

// lower edge and width of R cell i
__host__ __device__ inline void n2t_rcell(int i, double &lo, double &w) {
  if (i < 16) {
    w = 0.5;
    lo = 4.5 + 0.5 * i;
  } else if (i < 21) {
    w = 1.5;
    lo = 12.5 + 1.5 * (i - 16);
  } else {
    w = 4.0;
    lo = 20.0 + 4.0 * (i - 21);
  }
}

// R cell of R in [4.5, 60) and the cell coordinate x in [-1, 1]
__device__ __forceinline__ int n2t_rindex(float R, float &x) {
  int i;
  float lo, s;
  if (R < 12.5f) {
    i = min(max(int((R - 4.5f) * 2.0f), 0), 15);
    lo = 4.5f + 0.5f * float(i);
    s = 4.0f;
  } else if (R < 20.0f) {
    i = min(int((R - 12.5f) * (1.0f / 1.5f)), 4);
    lo = 12.5f + 1.5f * float(i);
    s = 2.0f / 1.5f;
    i += 16;
  } else {
    i = min(int((R - 20.0f) * 0.25f), 9);
    lo = 20.0f + 4.0f * float(i);
    s = 0.5f;
    i += 21;
  }
  x = (R - lo) * s - 1.0f;
  return i;
}

// one block per cell: the network at the 10 x 10 Chebyshev nodes, then the
// coefficients c_ij = (2 - d_i0)(2 - d_j0)/100 sum_ab f(x_a, y_b) T_i(x_a) T_j(y_b)
static __global__ void __launch_bounds__(128) n2ar_tab_build_kernel(const N2arDipFold *F, float4 *tab) {
  constexpr int D = N2T_DEG;
  __shared__ double v[2][D][D];
  const int cell = blockIdx.x, ir = cell / N2T_NT, it = cell - ir * N2T_NT;
  double lo, w;
  n2t_rcell(ir, lo, w);
  const int t = threadIdx.x;
  if (t < D * D) {
    const int a = t / D, b = t - a * D;
    const double xa = cospi((a + 0.5) / D), xb = cospi((b + 0.5) / D);
    const double R = lo + 0.5 * w * (xa + 1.0);
    const double T = (it + 0.5 * (xb + 1.0)) * (HH_PI / N2T_NT);
    const N2arDipBody<double> d = n2ar_dip_body(F, R, cos(T));
    v[0][a][b] = d.dx;
    v[1][a][b] = d.dz;
  }
  __syncthreads();
  if (t < D * D) {
    const int i = t / D, j = t - i * D;
    double sx = 0.0, sz = 0.0;
    for (int a = 0; a < D; ++a) {
      const double ca = cospi(i * (a + 0.5) / D);
      for (int b = 0; b < D; ++b) {
        const double wab = ca * cospi(j * (b + 0.5) / D);
        sx += v[0][a][b] * wab;
        sz += v[1][a][b] * wab;
      }
    }
    const double f = (i ? 2.0 : 1.0) * (j ? 2.0 : 1.0) / double(D * D);
    reinterpret_cast<float2 *>(tab)[(size_t)cell * D * D + i * D + j] =
        make_float2(float(sx * f), float(sz * f));
  }
}

// body-frame dipole from the table (FP32), R in [4.5, 60), T in [0, pi]
__device__ __forceinline__ void n2ar_dip_tab(const float4 *tab, float R, float T, float &dx, float &dz) {
  constexpr int D = N2T_DEG;
  float xr;
  const int ir = n2t_rindex(R, xr);
  const float tc = T * float(N2T_NT / HH_PI);
  const int it = min(max(int(tc), 0), N2T_NT - 1);
  const float xt = 2.0f * (tc - float(it)) - 1.0f;
  float Tt[D];
  Tt[0] = 1.0f;
  Tt[1] = xt;
#pragma unroll
  for (int j = 2; j < D; ++j) Tt[j] = 2.0f * xt * Tt[j - 1] - Tt[j - 2];
  const float4 *c = tab + (size_t)(ir * N2T_NT + it) * N2T_CELL_F4;
  float ax = 0.0f, az = 0.0f, r0 = 1.0f, r1 = xr;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    float ri;
    if (i == 0) ri = 1.0f;
    else if (i == 1) ri = xr;
    else {
      ri = 2.0f * xr * r1 - r0;
      r0 = r1;
      r1 = ri;
    }
    float sx = 0.0f, sz = 0.0f;
#pragma unroll
    for (int q = 0; q < D / 2; ++q) {
      const float4 v = __ldg(&c[i * (D / 2) + q]);
      sx += v.x * Tt[2 * q] + v.z * Tt[2 * q + 1];
      sz += v.y * Tt[2 * q] + v.w * Tt[2 * q + 1];
    }
    ax += ri * sx;
    az += ri * sz;
  }
  dx = ax;
  dz = az;
}

// body-frame dipole of the mixed path at R, x = cos T, s = sin T >= 0: the table
// inside its range, the FP64 network outside
__device__ __forceinline__ N2arDipBody<double> n2ar_dip_body_mixed(const float4 *tab, const N2arDipFold *F,
                                                                   double R, double x, double s) {
  if (R >= N2T_RLO && R < N2T_RHI) {
    float dx, dz;
    n2ar_dip_tab(tab, float(R), atan2f(float(s), float(x)), dx, dz);
    return {double(dx), double(dz)};
  }
  return n2ar_dip_body(F, R, x);
}

}  // namespace hh
