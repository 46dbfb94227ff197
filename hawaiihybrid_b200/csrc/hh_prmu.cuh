// PR_MU spectral function (src/hawaii.c:3148-3978): the spectrum of each trajectory's
// dipole, weighted by its initial radial velocity.
//
// The reference integrates a trajectory from R0 inward, keeps the lab dipole at
// t = (k+1) dt for k = 0..N-1 (zero after it leaves the R0 sphere), apodizes each
// component with Connes' window, takes its real FFT (gsl_fft_real_radix2_transform)
// and adds SF_COEFF pR/mu sum_c |F_c(i)|^2 into the spectrum for the first L
// frequencies (hawaii.c:3812-3825).
//
// GPU mapping, per chunk of trajectories whose dipole series are in HBM:
//   1. prmu_pack: complex series sqrt(w) a_j (x_j + i y_j) and sqrt(w) a_j z_j per
//      trajectory (w = SF_COEFF pR/mu of an included trajectory, 0 otherwise, a_j the
//      Connes window).  For a real series the FFT magnitudes are even, so
//      (|S_k|^2 + |S_{N-k}|^2) / 2 of the first series is w (|X_k|^2 + |Y_k|^2) and of
//      the second w |Z_k|^2;
//   2. stockham_batch: log2 N radix-2 passes over all series at once;
//   3. prmu_accum: one thread per frequency sums those terms over the series.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_consts.h"
#include "hh_traj.cuh"

namespace hh {

struct PrmuPackArgs {
  const void *series;         // [traj][slot][4] in the surface precision; slot k = sample at k dt
  const int *len;             // [item]: samples stored (forward items 2 t)
  const int *status;          // [item]: end status | 16 when the branch left the R0 sphere
  const double *qp;           // [traj][QP]: the drawn phase points of the chunk (pR at 5)
  int QP;
  long long n_traj;
  int N, stride;              // samples per trajectory; series slots per trajectory
  int allow_trunc;
  double coeff;               // SF_COEFF / mu
  double2 *z;                 // [2 traj][N]
  unsigned long long *counted;
  // spin weights of a LINEAR_MOLECULE_REQ_HALFINTEGER monomer (src/hawaii.c:3575-3594):
  // req_mode 2 and a positive weight select even_w / odd_w by the parity of
  // round(j_ini - 1.5), j_ini the requantized initial |j|; otherwise weight 1
  int req_mode;
  double even_w, odd_w;
};

// the trajectory weight of PR_MU from the drawn linear-monomer phase point
// (phi, p_phi, theta, p_theta at qp[6..9]): j_monomer (src/hawaii.c:398-431), then
// the requantized length
__device__ __forceinline__ double prmu_spin_weight(const PrmuPackArgs &a, const double *qp) {
  if (a.req_mode != 2 || !(a.even_w > 0.0 || a.odd_w > 0.0)) return 1.0;
  const double phi = qp[6], pphi = qp[7], th = qp[8], pth = qp[9];
  const double ct = cos(th) / sin(th);
  const double j0 = -pth * sin(phi) - pphi * cos(phi) * ct, j1 = pth * cos(phi) - pphi * sin(phi) * ct;
  const double jl = sqrt(j0 * j0 + j1 * j1 + pphi * pphi);
  const double jini = req_closest(2, jl);
  const long long j_int = llround(jini - 1.5);
  return (j_int % 2 == 0) ? a.even_w : a.odd_w;
}

template <typename PHYS>
__global__ void __launch_bounds__(256) prmu_pack_kernel(PrmuPackArgs a) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= a.n_traj * a.N) return;
  const long long t = i / a.N;
  const int j = (int)(i - t * a.N);
  const int st = a.status[2 * t];
  const bool include = (st & 15) == HH_ST_OK && ((st & 16) || a.allow_trunc);
  const double pr_mu = -a.qp[t * a.QP + 5];
  const double sw = include ? sqrt(a.coeff * pr_mu * prmu_spin_weight(a, a.qp + t * a.QP)) : 0.0;
  if (j == 0 && include) atomicAdd(a.counted, 1ull);
  double d[3] = {0.0, 0.0, 0.0};
  if (include && j + 1 <= a.len[2 * t]) {
    const PHYS *v = static_cast<const PHYS *>(a.series) + ((size_t)t * a.stride + j + 1) * 4;
    d[0] = double(v[0]);
    d[1] = double(v[1]);
    d[2] = double(v[2]);
  }
  // connes_apodization (src/hawaii.c:5401-5410) with tmax = N dt
  const double r = double(j) / double(a.N);
  const double f = sw * (1.0 - r * r) * (1.0 - r * r);
  a.z[(2 * t) * a.N + j] = make_double2(f * d[0], f * d[1]);
  a.z[(2 * t + 1) * a.N + j] = make_double2(f * d[2], 0.0);
}

// one Stockham radix-2 pass over B series of length L each (n = L / s, m = n / 2)
__global__ void __launch_bounds__(256) stockham_batch_kernel(const double2 *x, double2 *y, long long L,
                                                             long long s, long long B) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long half = L / 2;
  if (g >= B * half) return;
  const long long b = g / half, t = g - b * half;
  const double2 *xb = x + b * L;
  double2 *yb = y + b * L;
  const long long n = L / s, m = n / 2;
  const long long p = t / s, q = t - p * s;
  const double2 u = xb[q + s * p];
  const double2 v = xb[q + s * (p + m)];
  double sn, cs;
  sincospi(2.0 * double(p) / double(n), &sn, &cs);
  const double2 dd = make_double2(u.x - v.x, u.y - v.y);
  yb[q + s * (2 * p)] = make_double2(u.x + v.x, u.y + v.y);
  yb[q + s * (2 * p + 1)] = make_double2(dd.x * cs - dd.y * sn, dd.x * sn + dd.y * cs);
}

// sf[k] += sum over series of (|S_k|^2 + |S_{N-k}|^2) / 2, k < L
__global__ void __launch_bounds__(256) prmu_accum_kernel(const double2 *z, long long B, int N, int L,
                                                         double *sf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= L) return;
  const int kr = (N - k) % N;
  double acc = 0.0;
  for (long long b = 0; b < B; ++b) {
    const double2 u = z[b * N + k], v = z[b * N + kr];
    acc += 0.5 * (u.x * u.x + u.y * u.y + v.x * v.x + v.y * v.y);
  }
  sf[k] += acc;
}

}  // namespace hh
