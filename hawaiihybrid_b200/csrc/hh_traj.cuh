// Persistent trajectory kernel: one half-trajectory (forward or momentum-
// inverted backward branch of src/hawaii.c:2116-2347) per thread, integrated
// with DOP853 and its 7th-order dense output, the induced dipole sampled at
// t_k = k*dt and mu0.mu(t_k) added into the ensemble C(t) in FP64.
//
// Work items are popped from a device counter, so uneven trajectory lengths
// (R > Rcut exits, long-lived orbiting pairs) rebalance across the grid.  Each
// item adds  w * mu0.mu(t_k)  for its samples, w = ppf * ALU^3 / 2, so the two
// branches together reproduce crln[k] = ppf * (fwd[k] + bwd[k]) / 2 * ALU^3
// (src/hawaii.c:2334-2337, 3008).
//
// Precision: PHYS is the type the surfaces are evaluated in (double for the
// plain path, float for the mixed path, with compensated sums); STG is the type
// of the stage derivatives and increments.  Integrator state, time, step size
// and the C(t) accumulation are FP64 in both paths.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "hh_consts.h"
#include "hh_dop853_tableau.h"
#include "hh_physics.cuh"

namespace hh {

enum { SYS_HEAR = 1, SYS_CO2AR = 2 };

struct TrajParams {
  double mu, II;
  double dt;
  int N;
  double Rcut;
  double rtol, atol;
  long long max_steps;        // internal steps allowed between two samples
  long long max_total_steps;  // internal steps allowed per half-trajectory
  double weight;              // +-ppf * ALU^3 / 2
  // test hook: half-trajectory (2*traj + dir) that reports status inject_status
  // at sample inject_k instead of storing it (-1: off)
  int inject_item, inject_k, inject_status;
};

struct TrajIO {
  const double *ic;           // [n_traj][qp] spherical phase points (reference layout)
  const int *items;           // optional explicit item list (item = 2*traj + dir)
  int n_items;
  unsigned int *queue;        // work counter
  double *crln;               // [N] accumulated C(t)
  unsigned long long *counters;  // [8]: steps, rejected, rhs, samples, dense, items, _, _
  unsigned int *status_hist;  // [HH_ST_COUNT]
  int *fail_flag;             // [n_traj] (nullptr on the compensation pass)
  int *fail_list;
  int *fail_count;
};

// ---- coefficient tables for CO2-Ar, staged in shared memory ----
template <typename T> struct Co2arTables {
  T pes[CO2AR_TABLE];
  T dipx[CO2AR_TABLE];
  T dipz[CO2AR_TABLE];
  T rbound[CO2AR_NINT];
  T rlo[CO2AR_NINT];
  int fpes[CO2AR_NINT];
  int fdip[CO2AR_NINT];
};

struct Co2arTablesGlobal {  // FP64 master copy in global memory
  double pes[CO2AR_TABLE];
  double dipx[CO2AR_TABLE];
  double dipz[CO2AR_TABLE];
  double rbound[CO2AR_NINT];
  double rlo[CO2AR_NINT];
  int fpes[CO2AR_NINT];
  int fdip[CO2AR_NINT];
};

template <typename T>
__device__ void load_tables(Co2arTables<T> *s, const Co2arTablesGlobal *g) {
  for (int i = threadIdx.x; i < CO2AR_TABLE; i += blockDim.x) {
    s->pes[i] = T(g->pes[i]);
    s->dipx[i] = T(g->dipx[i]);
    s->dipz[i] = T(g->dipz[i]);
  }
  for (int i = threadIdx.x; i < CO2AR_NINT; i += blockDim.x) {
    s->rbound[i] = T(g->rbound[i]);
    s->rlo[i] = T(g->rlo[i]);
    s->fpes[i] = g->fpes[i];
    s->fdip[i] = g->fdip[i];
  }
}

// ---- systems ----
template <typename PHYS, typename STG, bool COMP> struct HeArSys {
  static constexpr int N = 6;
  static constexpr int QP = 6;
  double inv_mu;
  __device__ void rhs(const double *y, STG *f) const {
    PHYS r0 = PHYS(y[0]), r1 = PHYS(y[1]), r2 = PHYS(y[2]);
    PHYS R2 = r0 * r0 + r1 * r1 + r2 * r2;
    PHYS R = sqrt(R2);
    PHYS V, dV;
    hear_V_dV<PHYS>(R, V, dV);
    PHYS g = dV / R;
    f[0] = STG(y[3] * inv_mu);
    f[1] = STG(y[4] * inv_mu);
    f[2] = STG(y[5] * inv_mu);
    f[3] = STG(-g * r0);
    f[4] = STG(-g * r1);
    f[5] = STG(-g * r2);
  }
  __device__ void dipole(const double *y, PHYS d[3]) const {
    PHYS r0 = PHYS(y[0]), r1 = PHYS(y[1]), r2 = PHYS(y[2]);
    PHYS R = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
    PHYS s = hear_dip<PHYS>(R) / R;
    d[0] = s * r0;
    d[1] = s * r1;
    d[2] = s * r2;
  }
};

template <typename PHYS, typename STG, bool COMP> struct Co2ArSys {
  static constexpr int N = 12;
  static constexpr int QP = 10;
  double inv_mu, inv_II;
  const Co2arTables<PHYS> *tb;
  __device__ void rhs(const double *y, STG *f) const {
    PHYS r[3] = {PHYS(y[0]), PHYS(y[1]), PHYS(y[2])};
    PHYS u[3] = {PHYS(y[6]), PHYS(y[7]), PHYS(y[8])};
    PHYS R = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    PHYS iR = PHYS(1) / R;
    PHYS iu = PHYS(1) / sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    PHYS rh[3] = {r[0] * iR, r[1] * iR, r[2] * iR};
    PHYS uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    PHYS x = rh[0] * uh[0] + rh[1] * uh[1] + rh[2] * uh[2];
    PHYS V, VR, Vx;
    co2ar_pes<PHYS, COMP>(tb->pes, tb->fpes, tb->rbound, tb->rlo, R, x, V, VR, Vx, false);
    PHYS a = VR - Vx * x * iR;  // dV/dr = a r^ + (Vx/R) u^
    PHYS b = Vx * iR;
    f[0] = STG(y[3] * inv_mu);
    f[1] = STG(y[4] * inv_mu);
    f[2] = STG(y[5] * inv_mu);
    f[3] = STG(-(a * rh[0] + b * uh[0]));
    f[4] = STG(-(a * rh[1] + b * uh[1]));
    f[5] = STG(-(a * rh[2] + b * uh[2]));
    // du/dt = (j x u)/I, evaluated in FP64 (kinematic part)
    f[6] = STG((y[10] * y[8] - y[11] * y[7]) * inv_II);
    f[7] = STG((y[11] * y[6] - y[9] * y[8]) * inv_II);
    f[8] = STG((y[9] * y[7] - y[10] * y[6]) * inv_II);
    // dj/dt = -Vx (u^ x r^)
    f[9] = STG(-Vx * (uh[1] * rh[2] - uh[2] * rh[1]));
    f[10] = STG(-Vx * (uh[2] * rh[0] - uh[0] * rh[2]));
    f[11] = STG(-Vx * (uh[0] * rh[1] - uh[1] * rh[0]));
  }
  __device__ void dipole(const double *y, PHYS d[3]) const {
    PHYS r[3] = {PHYS(y[0]), PHYS(y[1]), PHYS(y[2])};
    PHYS u[3] = {PHYS(y[6]), PHYS(y[7]), PHYS(y[8])};
    PHYS R = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    PHYS iR = PHYS(1) / R;
    PHYS iu = PHYS(1) / sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    PHYS rh[3] = {r[0] * iR, r[1] * iR, r[2] * iR};
    PHYS uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    PHYS x = rh[0] * uh[0] + rh[1] * uh[1] + rh[2] * uh[2];
    PHYS dz, ax;
    co2ar_dip<PHYS, COMP>(tb->dipx, tb->dipz, tb->fdip, tb->rbound, tb->rlo, R, x, dz, ax);
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = dz * rh[c] - ax * (uh[c] - x * rh[c]);
  }
};

// spherical phase point (reference layout, src/hawaii.h:210-284) -> Cartesian
template <int SYS>
__device__ __forceinline__ void qp_to_state(const double *qp, double *y) {
  double Phi = qp[0], pPhi = qp[1], Th = qp[2], pTh = qp[3], R = qp[4], pR = qp[5];
  double sT, cT, sP, cP;
  sincos(Th, &sT, &cT);
  sincos(Phi, &sP, &cP);
  double Rh[3] = {sT * cP, sT * sP, cT};
  double Thh[3] = {cT * cP, cT * sP, -sT};
  double Phh[3] = {-sP, cP, 0.0};
  double a = pTh / R, b = pPhi / (R * sT);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    y[i] = R * Rh[i];
    y[3 + i] = pR * Rh[i] + a * Thh[i] + b * Phh[i];
  }
  if (SYS == SYS_CO2AR) {
    double ph = qp[6], pph = qp[7], th = qp[8], pth = qp[9];
    double s, c, sp, cp;
    sincos(th, &s, &c);
    sincos(ph, &sp, &cp);
    double u[3] = {s * cp, s * sp, c};
    double thh[3] = {c * cp, c * sp, -s};
    double phh[3] = {-sp, cp, 0.0};
    double g = pph / s;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      y[6 + i] = u[i];
      y[9 + i] = pth * phh[i] - g * thh[i];  // j = u x p_u
    }
  }
}

// ---------------------------------------------------------------------------
// DOP853 (Hairer-Norsett-Wanner) with the standard step controller
// (safety 0.9, factors in [0.2, 10], exponent -1/8) and dense output.
// ---------------------------------------------------------------------------
template <class Sys, typename STG>
struct Dop853 {
  static constexpr int N = Sys::N;
  STG K[16][N];

  // one adaptive step from (t, y) with K[0] = f(t, y); returns 0 or a status
  __device__ int step(const Sys &sys, const TrajParams &P, double t, const double *y, double &h,
                      double &h_taken, double *y_new, unsigned &nrej, unsigned &nrhs) {
    bool rejected = false;
    for (;;) {
      // 10 * spacing of doubles above t (t >= 0 and finite)
      double min_step = 10.0 * (__longlong_as_double(__double_as_longlong(t) + 1) - t);
      if (!(h >= min_step)) return HH_ST_H_UNDERFLOW;
#pragma unroll
      for (int s = 1; s < 12; ++s) {
        double ys[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
          STG acc = STG(0);
#pragma unroll
          for (int j = 0; j < s; ++j)
            if (hh_dop853_a[s][j] != 0.0) acc += STG(hh_dop853_a[s][j]) * K[j][i];
          ys[i] = y[i] + h * double(acc);
        }
        sys.rhs(ys, K[s]);
      }
#pragma unroll
      for (int i = 0; i < N; ++i) {
        STG acc = STG(0);
#pragma unroll
        for (int j = 0; j < 12; ++j)
          if (hh_dop853_a[12][j] != 0.0) acc += STG(hh_dop853_a[12][j]) * K[j][i];
        y_new[i] = y[i] + h * double(acc);
      }
      sys.rhs(y_new, K[12]);
      nrhs += 12;
      double e5 = 0.0, e3 = 0.0;
#pragma unroll
      for (int i = 0; i < N; ++i) {
        double sc = P.atol + fmax(fabs(y[i]), fabs(y_new[i])) * P.rtol;
        STG a5 = STG(0), a3 = STG(0);
#pragma unroll
        for (int j = 0; j < 13; ++j) {
          if (hh_dop853_e5[j] != 0.0) a5 += STG(hh_dop853_e5[j]) * K[j][i];
          if (hh_dop853_e3[j] != 0.0) a3 += STG(hh_dop853_e3[j]) * K[j][i];
        }
        double q5 = double(a5) / sc, q3 = double(a3) / sc;
        e5 += q5 * q5;
        e3 += q3 * q3;
      }
      double err = (e5 == 0.0 && e3 == 0.0) ? 0.0 : fabs(h) * e5 / sqrt((e5 + 0.01 * e3) * N);
      if (err < 1.0) {
        double fac = (err == 0.0) ? 10.0 : fmin(10.0, 0.9 * pow(err, -0.125));
        if (rejected) fac = fmin(1.0, fac);
        h_taken = h;
        h = h * fac;
        return HH_ST_OK;
      }
      h *= fmax(0.2, 0.9 * pow(err, -0.125));
      rejected = true;
      ++nrej;
    }
  }

  // dense-output coefficients F[7][N] of the last step (needs K[0..12])
  __device__ void dense(const Sys &sys, const double *y_old, const double *y_new, double h,
                        STG (&F)[7][N], unsigned &nrhs) {
#pragma unroll
    for (int s = 13; s < 16; ++s) {
      double ys[N];
#pragma unroll
      for (int i = 0; i < N; ++i) {
        STG acc = STG(0);
#pragma unroll
        for (int j = 0; j < s; ++j)
          if (hh_dop853_a[s][j] != 0.0) acc += STG(hh_dop853_a[s][j]) * K[j][i];
        ys[i] = y_old[i] + h * double(acc);
      }
      sys.rhs(ys, K[s]);
    }
    nrhs += 3;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double dy = y_new[i] - y_old[i];
      F[0][i] = STG(dy);
      F[1][i] = STG(h * double(K[0][i]) - dy);
      F[2][i] = STG(2.0 * dy - h * (double(K[12][i]) + double(K[0][i])));
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        STG acc = STG(0);
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (hh_dop853_d[r][j] != 0.0) acc += STG(hh_dop853_d[r][j]) * K[j][i];
        F[3 + r][i] = STG(h * double(acc));
      }
    }
  }
};

template <int N, typename STG>
__device__ __forceinline__ void dense_eval(const double *y_old, const STG (&F)[7][N], double x,
                                           double *y) {
  double x1 = 1.0 - x;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double v = double(F[6][i]) * x;
    v = (v + double(F[5][i])) * x1;
    v = (v + double(F[4][i])) * x;
    v = (v + double(F[3][i])) * x1;
    v = (v + double(F[2][i])) * x;
    v = (v + double(F[1][i])) * x1;
    v = (v + double(F[0][i])) * x;
    y[i] = y_old[i] + v;
  }
}

template <class Sys>
__device__ __forceinline__ double state_R(const double *y) {
  return sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
}

// initial step size (Hairer's algorithm, error-estimator order 7)
template <class Sys, typename STG>
__device__ double initial_step(const Sys &sys, const TrajParams &P, const double *y0,
                               const STG *f0, double span, unsigned &nrhs) {
  constexpr int N = Sys::N;
  double d0 = 0.0, d1 = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double sc = P.atol + fabs(y0[i]) * P.rtol;
    double a = y0[i] / sc, b = double(f0[i]) / sc;
    d0 += a * a;
    d1 += b * b;
  }
  d0 = sqrt(d0 / N);
  d1 = sqrt(d1 / N);
  double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
  h0 = fmin(h0, span);
  double y1[N];
  STG f1[N];
#pragma unroll
  for (int i = 0; i < N; ++i) y1[i] = y0[i] + h0 * double(f0[i]);
  sys.rhs(y1, f1);
  ++nrhs;
  double d2 = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double sc = P.atol + fabs(y0[i]) * P.rtol;
    double a = (double(f1[i]) - double(f0[i])) / sc;
    d2 += a * a;
  }
  d2 = sqrt(d2 / N) / h0;
  double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / fmax(d1, d2), 0.125);
  return fmin(fmin(100.0 * h0, h1), span);
}

// ---------------------------------------------------------------------------
// one half-trajectory; returns its status, *hard = 1 for the failures that make
// the reference drop the whole trajectory
// ---------------------------------------------------------------------------
template <class Sys, typename PHYS, typename STG>
__device__ int run_half(const Sys &sys, const TrajParams &P, const double *y0, const PHYS mu0[3],
                        double *crln, unsigned &nsteps, unsigned &nrej, unsigned &nrhs,
                        unsigned &nsamp, unsigned &ndense, int &hard, int item) {
  constexpr int N = Sys::N;
  Dop853<Sys, STG> dop;
  double y[N], y_new[N];
#pragma unroll
  for (int i = 0; i < N; ++i) y[i] = y0[i];
  sys.rhs(y, dop.K[0]);
  ++nrhs;
  const double dt = P.dt;
  double h = initial_step<Sys, STG>(sys, P, y, dop.K[0], dt * double(P.N - 1), nrhs);
  double t = 0.0;
  int k = 1;
  long long since = 0, total = 0;
  PHYS prev = PHYS(0), curr = PHYS(0);
  hard = 0;
  while (k < P.N) {
    double ht;
    int rc = dop.step(sys, P, t, y, h, ht, y_new, nrej, nrhs);
    if (rc) return rc;
    ++nsteps;
    double t_new = t + ht;
    if (double(k) * dt <= t_new) {
      STG F[7][N];
      dop.dense(sys, y, y_new, ht, F, nrhs);
      ++ndense;
      do {
        double x = (double(k) * dt - t) / ht;
        double ys[N];
        dense_eval<N, STG>(y, F, x, ys);
        PHYS d[3];
        sys.dipole(ys, d);
        ++nsamp;
        if (isnan(d[0]) || isnan(d[1]) || isnan(d[2])) { hard = 1; return HH_ST_NAN_DIPOLE; }
        if (item == P.inject_item && k == P.inject_k) {
          hard = (P.inject_status >= HH_ST_NAN_DIPOLE);
          return P.inject_status;
        }
        prev = curr;
        curr = mu0[0] * d[0] + mu0[1] * d[1] + mu0[2] * d[2];
        if (fabs(double(curr)) > 1e100) { hard = 1; return HH_ST_OVERFLOW; }
        if (k > 1) {
          double ratio = fabs(double(curr) / double(prev));
          if (ratio > 1e10) { hard = 1; return HH_ST_JUMP; }
        }
        atomicAdd(&crln[k], P.weight * double(curr));
        ++k;
        since = 0;
        if (state_R<Sys>(ys) > P.Rcut) return HH_ST_OK;
      } while (k < P.N && double(k) * dt <= t_new);
    }
    t = t_new;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      y[i] = y_new[i];
      dop.K[0][i] = dop.K[12][i];
    }
    if (++since > P.max_steps || ++total > P.max_total_steps) return HH_ST_MAXSTEPS;
  }
  return HH_ST_OK;
}

__device__ __forceinline__ void warp_add_counter(unsigned long long *dst, unsigned v) {
  unsigned long long s = v;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(dst, s);
}

template <class Sys, typename PHYS, typename STG>
__device__ __forceinline__ void traj_body(const Sys &sys, const TrajParams &P, const TrajIO &io) {
  constexpr int N = Sys::N;
  constexpr int SYS = (N == 6) ? SYS_HEAR : SYS_CO2AR;
  unsigned nsteps = 0, nrej = 0, nrhs = 0, nsamp = 0, ndense = 0, nitems = 0;
  for (;;) {
    unsigned idx = atomicAdd(io.queue, 1u);
    if (idx >= (unsigned)io.n_items) break;
    int item = io.items ? io.items[idx] : (int)idx;
    int traj = item >> 1, dir = item & 1;
    double y0[N];
    qp_to_state<SYS>(io.ic + (size_t)traj * Sys::QP, y0);
    PHYS mu0[3];
    sys.dipole(y0, mu0);
    if (dir) {
      // invert_momenta (src/hawaii.c:1171-1188): p -> -p, j -> -j
#pragma unroll
      for (int i = 3; i < 6; ++i) y0[i] = -y0[i];
#pragma unroll
      for (int i = 9; i < N; ++i) y0[i] = -y0[i];
    }
    PHYS c0 = mu0[0] * mu0[0] + mu0[1] * mu0[1] + mu0[2] * mu0[2];
    int hard = 0;
    int st = run_half<Sys, PHYS, STG>(sys, P, y0, mu0, io.crln, nsteps, nrej, nrhs, nsamp,
                                      ndense, hard, item);
    // the t = 0 term is added by branches that are not dropped, so a replay
    // with the opposite weight removes exactly what a dropped trajectory added
    if (!hard) atomicAdd(&io.crln[0], P.weight * double(c0));
    atomicAdd(&io.status_hist[st], 1u);
    ++nitems;
    if (hard && io.fail_flag) {
      if (atomicExch(&io.fail_flag[traj], 1) == 0) {
        int slot = atomicAdd(io.fail_count, 1);
        io.fail_list[slot] = traj;
      }
    }
  }
  warp_add_counter(&io.counters[0], nsteps);
  warp_add_counter(&io.counters[1], nrej);
  warp_add_counter(&io.counters[2], nrhs);
  warp_add_counter(&io.counters[3], nsamp);
  warp_add_counter(&io.counters[4], ndense);
  warp_add_counter(&io.counters[5], nitems);
}

template <int SYS, typename PHYS, typename STG, bool COMP>
__global__ void __launch_bounds__(128) traj_kernel(TrajParams P, TrajIO io,
                                                   const Co2arTablesGlobal *gtab) {
  if (SYS == SYS_HEAR) {
    HeArSys<PHYS, STG, COMP> sys;
    sys.inv_mu = 1.0 / P.mu;
    traj_body<HeArSys<PHYS, STG, COMP>, PHYS, STG>(sys, P, io);
  } else {
    extern __shared__ unsigned char smem_raw[];
    Co2arTables<PHYS> *tb = reinterpret_cast<Co2arTables<PHYS> *>(smem_raw);
    load_tables<PHYS>(tb, gtab);
    __syncthreads();
    Co2ArSys<PHYS, STG, COMP> sys;
    sys.inv_mu = 1.0 / P.mu;
    sys.inv_II = 1.0 / P.II;
    sys.tb = tb;
    traj_body<Co2ArSys<PHYS, STG, COMP>, PHYS, STG>(sys, P, io);
  }
}

}  // namespace hh
