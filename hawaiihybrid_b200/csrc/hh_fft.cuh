// CF -> SF transform (src/hawaii.c:5401-5410, 5478-5553, 5569-5601) in FP64.
//
// The reference apodizes C(t) with (1 - (t/tmax)^2)^2, packs the N samples into
// a 2N-point complex vector (Makhoul's half-sample shift, 1/(2N) scaling), runs
// a backward (exp(+i)) radix-2 FFT of length 2N and keeps the real part of the
// first N outputs, then scales to nu (cm^-1) and SF (J m^6 s).
//
// GPU mapping: one kernel apodizes and packs, log2(2N) Stockham autosort
// radix-2 passes (ping-pong between two buffers, twiddles from sincospi) do the
// FFT, one kernel scales.  The transform is a few microseconds of HBM traffic;
// it sits off the trajectory hot loop.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_consts.h"

namespace hh {

__global__ void idct_pack_kernel(double *cf, long long N, double dt, double2 *z) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long L = 2 * N;
  if (k >= L) return;
  double tmax = dt * double(N);
  if (k < N) {
    // Connes apodization, in place on the caller's C(t) like the reference
    double tc = dt * double(k);
    double r = tc / tmax;
    double f = (1.0 - r * r) * (1.0 - r * r);
    double v = cf[k] * f;
    cf[k] = v;
    double s, c;
    sincospi(double(k) / double(L), &s, &c);
    z[k] = make_double2(v * c / double(L), v * s / double(L));
  }
}

// second half of the packing needs the apodized values of the first half
__global__ void idct_pack2_kernel(const double *cf, long long N, double2 *z) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x + N;
  long long L = 2 * N;
  if (k >= L) return;
  if (k == N) {
    z[k] = make_double2(0.0, 0.0);
    return;
  }
  double v = cf[L - k];
  double s, c;
  sincospi(double(k) / double(L), &s, &c);
  z[k] = make_double2(-v * c / double(L), -v * s / double(L));
}

// one Stockham radix-2 pass: n = L/s, m = n/2
__global__ void stockham_pass_kernel(const double2 *x, double2 *y, long long L, long long s) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= L / 2) return;
  long long n = L / s, m = n / 2;
  long long p = t / s, q = t - p * s;
  double2 a = x[q + s * p];
  double2 b = x[q + s * (p + m)];
  double sn, cs;
  sincospi(2.0 * double(p) / double(n), &sn, &cs);  // backward: exp(+2 pi i p/n)
  double2 d = make_double2(a.x - b.x, a.y - b.y);
  y[q + s * (2 * p)] = make_double2(a.x + b.x, a.y + b.y);
  y[q + s * (2 * p + 1)] = make_double2(d.x * cs - d.y * sn, d.x * sn + d.y * cs);
}

__global__ void idct_finish_kernel(const double2 *z, long long N, double dt, double *nu,
                                   double *sf) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= N) return;
  double Xscale = 1.0 / HH_LIGHTSPEED_CM / HH_ATU / 2.0 / HH_PI;
  double Yscale = HH_ATU * HH_ADIPMOMU * HH_ADIPMOMU / (4.0 * HH_PI * HH_EPSILON0);
  double tmax = double(N) * dt;
  nu[i] = double(i) * HH_PI / tmax * Xscale;
  sf[i] = z[i].x * tmax / HH_PI * Yscale;
}

}  // namespace hh
