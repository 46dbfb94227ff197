// Zeroth spectral moment by plain Monte Carlo over phase space, all
// temperatures in one launch.
//
// The reference integrates jac * |mu(q)|^2 * exp(-H/kT) over phase space with
// VEGAS (src/hep_hawaii.cpp:148-201) and scales by ZeroCoeff / pf_analytic
// (src/driver.c:3425-3431).  With R uniform on [Rmin, Rmax], isotropic angles
// and momenta drawn from exp(-K/kT) (the p_generator distribution), the
// momentum integral cancels pf_analytic except for its configurational part:
//   M0(T) = ZeroCoeff * 4 pi (Rmax - Rmin) * < R^2 |mu|^2 exp(-V/kT) 1[filter] >
// where the free+metastable filter keeps H = K + V >= 0 (bound: H <= 0).
// Only K enters, and K = kT * kappa with kappa half a chi^2 variable of 3
// (atom-atom) or 5 (linear-atom) degrees of freedom; it is drawn with
// Box-Muller sums, so one phase-space sample serves every temperature.
//
// Random numbers: Philox4x32-10, counter (i_lo, i_hi, block, 0), key = seed,
// uniforms ((w >> 8) + 0.5) * 2^-24, which are exact in FP32 and FP64, so the
// FP32 and FP64 integrands see the same sample.
//
// Sums: per thread FP64 compensated sums of w and plain sums of w^2 per
// temperature, a fixed-order block reduction, then one fixed-order pass over
// the block partials.
//
// Second moment (calculate_M2, src/hawaii.c:1524-1617; VEGAS integrand_M2,
// src/hep_hawaii.cpp:228-330): the integrand is |dmu/dt|^2 = qdot^T D D^T qdot with
// D = dmu/dq and qdot = dH/dp.  At fixed q and kinetic energy K the momentum
// direction is uniform in the mass-weighted metric, so E[qdot qdot^T | K] =
// (2K/nu) M^-1 and
//   M2(T) = SecondCoeff * 4 pi (Rmax - Rmin) * < R^2 (2K/nu) G(q) exp(-V/kT) 1[filter] >,
//   G(q) = tr(D^T M^-1 D) = |grad_r mu|^2 / mu_red + sum_{b=1,2} |dmu/dphi_b|^2 / I,
// with nu = 3 (atom-atom) or 5 (linear-atom) and phi_b rotations of u^ about two
// axes normal to it.  G is formed by central differences with h = 1e-3 (bohr,
// radian), as the reference forms D, from the FP64 lab-frame dipole of the
// trajectory kernels at 10 displaced configurations.  The same samples, K included,
// as M0.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_consts.h"
#include "hh_physics.cuh"
#include "hh_traj.cuh"

namespace hh {

constexpr int M0_MAXT = 16;  // temperatures per launch chunk (even: the mixed path pairs them)
static_assert(M0_MAXT % 2 == 0, "temperature pairs");

// 2^x by the ex2.approx instruction (PTX ISA: maximum relative error about 2^-22)
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct M0Args {
  int sys;
  int moment;                // 0: M0, 2: M2
  double inv_mu, inv_II;     // M2: 1 / reduced mass, 1 / moment of inertia (a.u.)
  double Rmin, Rmax;
  int pair_state;
  int nT;
  double invkT[M0_MAXT];   // Hartree^-1
  float kT[M0_MAXT];       // mixed path: kT (Hartree) and log2(e) / kT, FP32
  float l2e_kT[M0_MAXT];
  uint64_t n_samples, offset, seed;
};

__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                              uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

template <typename T> __device__ __forceinline__ T u24(uint32_t w) {
  return (T(w >> 8) + T(0.5)) * T(1.0 / 16777216.0);
}

// G(q) of the second moment at distance R and x = cos(angle between r^ and u^), in
// the frame r^ = z, u^ = (s, 0, x): central differences of the lab dipole over the
// three Cartesian displacements of r and (linear molecules) the rotations of u^
// about y and about u^ x y
template <class Sys>
__device__ double m2_geometry(const Sys &sys, double R, double x, double inv_mu, double inv_II, bool rotor) {
  const double h = 1.0e-3;
  const double s = sqrt(fmax(0.0, (1.0 - x) * (1.0 + x)));
  double q[6] = {0.0, 0.0, R, s, 0.0, x};
  double dp[3], dm[3], gt = 0.0, gr = 0.0;
  for (int a = 0; a < 3; ++a) {
    const double q0 = q[a];
    q[a] = q0 + h;
    sys.dipole(q, dp);
    q[a] = q0 - h;
    sys.dipole(q, dm);
    q[a] = q0;
    for (int c = 0; c < 3; ++c) gt += (dp[c] - dm[c]) * (dp[c] - dm[c]);
  }
  if (rotor) {
    double sh, ch;
    sincos(h, &sh, &ch);
    // about y: u^ -> u^ cos h +- (x, 0, -s) sin h
    q[3] = s * ch + x * sh;
    q[5] = x * ch - s * sh;
    sys.dipole(q, dp);
    q[3] = s * ch - x * sh;
    q[5] = x * ch + s * sh;
    sys.dipole(q, dm);
    for (int c = 0; c < 3; ++c) gr += (dp[c] - dm[c]) * (dp[c] - dm[c]);
    // about u^ x y: u^ -> u^ cos h +- y sin h
    q[3] = s * ch;
    q[5] = x * ch;
    q[4] = sh;
    sys.dipole(q, dp);
    q[4] = -sh;
    sys.dipole(q, dm);
    for (int c = 0; c < 3; ++c) gr += (dp[c] - dm[c]) * (dp[c] - dm[c]);
  }
  return (gt * inv_mu + gr * inv_II) / (4.0 * h * h);
}

// the launch's temperatures T[0 .. nT-1] (K) into a
inline void m0_set_temperatures(M0Args &a, const double *T, int nT) {
  a.nT = nT;
  for (int t = 0; t < M0_MAXT; ++t) {
    const double ikT = t < nT ? HH_HKT / T[t] : 0.0;
    a.invkT[t] = ikT;
    a.kT[t] = t < nT ? float(T[t] / HH_HKT) : 0.f;
    a.l2e_kT[t] = float(ikT * HH_LOG2E);
  }
}

template <int SYS, typename PHYS, bool COMP, int MOMENT = 0>
__global__ void __launch_bounds__(256) m0_kernel(M0Args a, const Co2arTablesGlobal *gtab,
                                                 const void *dipnet, double *partials) {
  static_assert(MOMENT == 0 || sizeof(PHYS) == 8, "the second moment is evaluated in FP64");
  extern __shared__ unsigned char smem_raw[];
  Co2arTables<PHYS> *tb = reinterpret_cast<Co2arTables<PHYS> *>(smem_raw);
  N2arDipFold *fold = reinterpret_cast<N2arDipFold *>(smem_raw);
  if (SYS == SYS_CO2AR) load_tables<PHYS>(tb, gtab);
  if (SYS == SYS_N2AR) load_words(fold, dipnet, sizeof(N2arDipFold));
  __syncthreads();
  // per-thread sums of w (compensated) and w^2: FP64 on the FP64 path; on the mixed path
  // FP32 with compensation (a thread sums a few hundred samples per launch, the block
  // and launch reductions are FP64)
  using AT = typename std::conditional<sizeof(PHYS) == 4 && MOMENT == 0, float, double>::type;
  AT s[M0_MAXT], c[M0_MAXT], q[M0_MAXT];
  PHYS ikT[M0_MAXT];
#pragma unroll
  for (int t = 0; t < M0_MAXT; ++t) {
    s[t] = c[t] = q[t] = AT(0);
    ikT[t] = PHYS(a.invkT[t]);
  }
  // mixed path: the temperatures in pairs (paired FP32, fma2): the sums, kT and
  // log2(e) / kT of temperatures (2j, 2j + 1)
  constexpr bool PAIRED = sizeof(PHYS) == 4 && MOMENT == 0;
  float2 s2[M0_MAXT / 2], c2[M0_MAXT / 2], q2[M0_MAXT / 2];
  if constexpr (PAIRED) {
#pragma unroll
    for (int j = 0; j < M0_MAXT / 2; ++j) s2[j] = c2[j] = q2[j] = make_float2(0.f, 0.f);
  }
  const PHYS Rmin = PHYS(a.Rmin), dR = PHYS(a.Rmax - a.Rmin);
  const PHYS twopi = PHYS(2.0 * HH_PI);
  const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.n_samples; i += stride) {
    uint64_t id = a.offset + i;
    uint32_t w[12];
    philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), 0u, 0u, k0, k1, w);
    philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), 1u, 0u, k0, k1, w + 4);
    philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), 2u, 0u, k0, k1, w + 8);
    PHYS R = Rmin + dR * u24<PHYS>(w[0]);
    PHYS zc = cos(twopi * u24<PHYS>(w[8]));
    PHYS V, mu2, kappa;
    if (SYS == SYS_HEAR) {
      PHYS dV;
      PHYS iR = PHYS(1) / R;
      hear_V_dV<PHYS>(R, iR, V, dV);
      PHYS d = hear_dip<PHYS>(R, iR);
      mu2 = d * d;
      if constexpr (MOMENT == 2) {
        HeArSys<PHYS, PHYS, false> sys;
        mu2 = m2_geometry(sys, R, 1.0, a.inv_mu, a.inv_II, false) * (2.0 / 3.0);
      }
      kappa = -log(u24<PHYS>(w[5])) - log(u24<PHYS>(w[7])) * zc * zc;
    } else if (SYS == SYS_N2AR) {
      PHYS Phi = twopi * u24<PHYS>(w[1]);
      PHYS cT = PHYS(2) * u24<PHYS>(w[2]) - PHYS(1);
      PHYS ph = twopi * u24<PHYS>(w[3]);
      PHYS ct = PHYS(2) * u24<PHYS>(w[4]) - PHYS(1);
      PHYS sT = sqrt((PHYS(1) - cT) * (PHYS(1) + cT));
      PHYS st = sqrt((PHYS(1) - ct) * (PHYS(1) + ct));
      PHYS x = sT * st * cos(Phi - ph) + cT * ct;
      // N1-Ar and N2-Ar distances with the N2 axis at angle acos(x) to r^
      const PHYS h = PHYS(N2AR_L / 2.0), base = R * R + h * h, t = PHYS(2) * h * R * x;
      V = n2ar_pes_energy<PHYS>(sqrt(base - t), sqrt(base + t));
      if constexpr (MOMENT == 2) {
        N2ArSys<PHYS, PHYS, false> sys;
        sys.fold = fold;
        sys.dtab = nullptr;
        mu2 = m2_geometry(sys, R, x, a.inv_mu, a.inv_II, true) * (2.0 / 5.0);
      } else {
        const N2arDipBody<double> b = n2ar_dip_body(fold, double(R), double(x));
        mu2 = PHYS(b.dx * b.dx + b.dz * b.dz);
      }
      kappa = -log(u24<PHYS>(w[5])) - log(u24<PHYS>(w[6])) - log(u24<PHYS>(w[7])) * zc * zc;
    } else {
      // x = cos(angle between r^ and u^) from the sampled lab angles
      PHYS Phi = twopi * u24<PHYS>(w[1]);
      PHYS cT = PHYS(2) * u24<PHYS>(w[2]) - PHYS(1);
      PHYS ph = twopi * u24<PHYS>(w[3]);
      PHYS ct = PHYS(2) * u24<PHYS>(w[4]) - PHYS(1);
      PHYS sT = sqrt((PHYS(1) - cT) * (PHYS(1) + cT));
      PHYS st = sqrt((PHYS(1) - ct) * (PHYS(1) + ct));
      PHYS x = sT * st * cos(Phi - ph) + cT * ct;
      PHYS iR = PHYS(1) / R;
      V = co2ar_pes_value<PHYS, COMP>(tb->pes, tb->fpes, tb->rbound, tb->rlo, R, iR, x);
      PHYS dz, ax;
      co2ar_dip<PHYS, COMP>(tb->dipx, tb->dipz, tb->fdip, tb->rbound, tb->rlo, R, iR, x, dz, ax);
      mu2 = dz * dz + ax * ax * (PHYS(1) - x) * (PHYS(1) + x);
      if constexpr (MOMENT == 2) {
        Co2ArSys<PHYS, PHYS, COMP> sys;
        sys.tb = tb;
        mu2 = m2_geometry(sys, R, x, a.inv_mu, a.inv_II, true) * (2.0 / 5.0);
      }
      kappa = -log(u24<PHYS>(w[5])) - log(u24<PHYS>(w[6])) - log(u24<PHYS>(w[7])) * zc * zc;
    }
    PHYS base = R * R * mu2;
    if constexpr (PAIRED) {
      // w = R^2 |mu|^2 2^(-V log2(e) / kT) behind the filter on H = kappa kT + V; the
      // exponential by ex2.approx (relative error about 2^-22 plus the rounding of the
      // FP32 argument), the sums compensated as below
      const float2 kap = splat2(float(kappa)), Vv = splat2(float(V)), nV = splat2(-float(V)), bb = splat2(float(base));
      const float2 m1 = splat2(-1.f);
#pragma unroll
      for (int j = 0; j < M0_MAXT / 2; ++j) {
        if (2 * j < a.nT) {
          const float2 H = fma2(kap, make_float2(a.kT[2 * j], a.kT[2 * j + 1]), Vv);
          const float2 arg = mul2(nV, make_float2(a.l2e_kT[2 * j], a.l2e_kT[2 * j + 1]));
          float2 e = make_float2(ex2_approx(arg.x), ex2_approx(arg.y));
          if (a.pair_state == 1) {
            e.x = H.x >= 0.f ? e.x : 0.f;
            e.y = H.y >= 0.f ? e.y : 0.f;
          } else if (a.pair_state == 2) {
            e.x = H.x <= 0.f ? e.x : 0.f;
            e.y = H.y <= 0.f ? e.y : 0.f;
          }
          const float2 wv = mul2(bb, e);
          const float2 y = fma2(c2[j], m1, wv);         // wv - c
          const float2 tt = add2(s2[j], y);
          c2[j] = fma2(y, m1, fma2(s2[j], m1, tt));    // (tt - s) - y
          s2[j] = tt;
          q2[j] = fma2(wv, wv, q2[j]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < M0_MAXT; ++t) {
      if (!PAIRED && t < a.nT) {
        PHYS H = kappa / ikT[t] + V;
        bool keep = true;
        if (a.pair_state == 1) keep = (H >= PHYS(0));
        else if (a.pair_state == 2) keep = (H <= PHYS(0));
        AT wv = keep ? AT(base * exp(-V * ikT[t])) : AT(0);
        if constexpr (MOMENT == 2) wv *= AT(kappa / ikT[t]);  // (2K/nu) G with K = kappa kT
        // compensated accumulation of w, plain accumulation of w^2
        AT y = wv - c[t];
        AT tt = s[t] + y;
        c[t] = (tt - s[t]) - y;
        s[t] = tt;
        q[t] += wv * wv;
      }
    }
  }
  if constexpr (PAIRED) {
#pragma unroll
    for (int j = 0; j < M0_MAXT / 2; ++j) {
      s[2 * j] = s2[j].x;
      s[2 * j + 1] = s2[j].y;
      c[2 * j] = c2[j].x;
      c[2 * j + 1] = c2[j].y;
      q[2 * j] = q2[j].x;
      q[2 * j + 1] = q2[j].y;
    }
  }
  // block reduction in a fixed order
  __shared__ double red[2][M0_MAXT][8];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int t = 0; t < M0_MAXT; ++t) {
    double v = double(s[t]) - double(c[t]), vq = double(q[t]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v += __shfl_down_sync(0xffffffffu, v, o);
      vq += __shfl_down_sync(0xffffffffu, vq, o);
    }
    if (lane == 0) {
      red[0][t][warp] = v;
      red[1][t][warp] = vq;
    }
  }
  __syncthreads();
  if (threadIdx.x < M0_MAXT) {
    int t = threadIdx.x;
    double v = 0.0, vq = 0.0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) {
      v += red[0][t][wi];
      vq += red[1][t][wi];
    }
    partials[((size_t)blockIdx.x * M0_MAXT + t) * 2 + 0] = v;
    partials[((size_t)blockIdx.x * M0_MAXT + t) * 2 + 1] = vq;
  }
}

// fixed-order compensated sum of the block partials
__global__ void m0_finalize_kernel(const double *partials, int n_blocks, double *out) {
  int t = threadIdx.x;
  if (t >= M0_MAXT) return;
  double s = 0.0, c = 0.0, q = 0.0;
  for (int b = 0; b < n_blocks; ++b) {
    double y = partials[((size_t)b * M0_MAXT + t) * 2] - c;
    double tt = s + y;
    c = (tt - s) - y;
    s = tt;
    q += partials[((size_t)b * M0_MAXT + t) * 2 + 1];
  }
  out[t * 2] = s;
  out[t * 2 + 1] = q;
}

}  // namespace hh
