// Persistent trajectory kernel: one half-trajectory (forward or momentum-
// inverted backward branch of src/hawaii.c:2116-2347) per lane, integrated
// with DOP853 and its 7th-order dense output, the induced dipole sampled at
// t_k = k*dt and mu0.mu(t_k) added into the ensemble C(t) in FP64.
//
// Work items are popped from a device counter, so uneven trajectory lengths
// (R > Rcut exits, long-lived orbiting pairs) rebalance across the grid.  Each
// item adds  w * mu0.mu(t_k)  for its samples, w = ppf * ALU^3 / 2, so the two
// branches together reproduce crln[k] = ppf * (fwd[k] + bwd[k]) / 2 * ALU^3
// (src/hawaii.c:2334-2337, 3008).
//
// Execution is warp-synchronous: every round, all lanes of a warp refill
// finished items, attempt one step, run the dense-output stages and emit their
// samples together, so the warp stays converged (one instruction stream, all
// lanes busy) instead of each lane wandering through its own item.
//
// Precision: PHYS is the type the surfaces are evaluated in (double for the
// plain path, float for the mixed path); STG is the type of the stage points,
// stage derivatives and dense-output increments.  Integrator state, time, step
// size and the C(t) accumulation are FP64 in both paths.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "hh_ch4co2.cuh"
#include "hh_consts.h"
#include "hh_dop853_tableau.h"
#include "hh_n2ar.cuh"
#include "hh_physics.cuh"

namespace hh {

enum { SYS_HEAR = 1, SYS_CO2AR = 2, SYS_N2AR = 3, SYS_CH4CO2 = 4 };

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
  // FP32 stages only: rounding-noise level of the stage derivatives, in units
  // of their magnitude, added to the error tolerance
  double noise_floor;
  // PR_MU samples (src/hawaii.c:3661-3688): a NaN dipole leaves its sample at zero
  // and no other per-sample test runs; the branch ends after R > Rcut
  int prmu;
  // PR_MU requantization of the linear monomer (REQ kernels only): 1 integer, 2
  // half-integer angular momentum (LINEAR_MOLECULE_REQ_INTEGER / _HALFINTEGER), 0 none;
  // the torque cache length and limit that switch it (src/hawaii.c:3604-3662)
  int req_mode, req_len;
  double req_limit;
  // bulk kernel: the block's warps start every block_sync-th round together (a block
  // barrier), so they walk the step code in step and share its instruction fetches;
  // 0: no barrier
  int block_sync;
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
  long long traj_per_iter;    // trajectories per iteration; item -> C(t) slice of its iteration
  uint4 *item_trace;          // optional per-item (steps, samples, t_start, t_end) in ns
  const void *dipnet;         // N2-Ar: the folded dipole models (N2arDipFold), global memory
  const void *pesnet;         // N2-Ar: the PES network (N2arPesNet) in the surface precision
  const void *diptab;         // N2-Ar mixed path: the dipole table (float4, hh_n2ar.cuh) or nullptr
  const double *sat_w;        // CORRELATION_ARRAY: [n_traj][n_sat] weights (nullptr: one C(t))
  int n_sat;                  // satellite temperatures; their C(t) are consecutive N-slices
  // CH4-CO2: samples are written as records (r, quaternion, u) in the surface
  // precision, HH_REC_WORDS words each, at traj * rec_stride + slot (slot 0: t = 0;
  // k: forward sample k; N - 1 + k: backward sample k), for the batched dipole
  void *records;
  int rec_stride;             // 2 * MaxTrajectoryLength - 1
  int *rec_len;               // [item]: samples stored (k = 1 .. rec_len)
  int *rec_status;            // [item]: end status of the integration
  double inv_I1[3];           // 1 / principal moments of CH4
  Ch4Co2Lj lj;
  // Zimmermann estimate: the lab-frame dipole of every stored sample, 4 values of
  // the surface precision per slot (slots as for records), instead of mu0 . mu(t_k)
  // added into crln; rec_len receives the stored samples per item
  void *series;
  int fwd_only;               // items are the forward branches only (item = 2 * index)
  // hand-off of the last items of a launch to the solo kernel (one warp per item):
  // the bulk kernel counts closed items in *done; once n_items - *done <= handoff_at
  // its warps store the state of their open items in `handoff` (slots counted by
  // *n_handoff) and stop; the solo kernel resumes them (cursor *solo_cursor), then
  // takes what is left in the queue.  handoff == nullptr: no hand-off.
  void *handoff;
  unsigned int *n_handoff;
  unsigned int *solo_cursor;
  unsigned int *done;
  unsigned int handoff_at;
  // deferred samples (plain C(t)): the kernel interpolates only r at the sample
  // times (the R > Rcut exit) and writes one SampleCtx per dense-output step into
  // `ctx` (index from *ctx_count; none past ctx_cap); the sample kernels of
  // hh_defer.cuh then evaluate the dipoles, accumulate C(t) and apply the per-sample
  // tests.  At an item's end the kernel writes its status to item_status instead of
  // adding the t = 0 term and counting the status.  ctx == nullptr: in-kernel samples.
  void *ctx;
  unsigned long long *ctx_count;
  unsigned long long ctx_cap;
  int *item_status;           // [item]
  void *item_mu0;             // [item][4] surface precision: mu0 and |mu0|^2
  // precomputed item starts (ItemStart per item, item_start_kernel) or nullptr: the
  // kernel then loads an item's initial state instead of running item_setup, whose
  // lane-divergent cost otherwise stalls the whole warp (and, with the block barrier,
  // the block) at every refill
  const void *setup;
};
constexpr int HH_REC_WORDS = 12;  // r[3], q[4], u[3], padding

// initial state of an item as item_setup makes it
template <int N, typename PHYS, typename STG> struct alignas(16) ItemStart {
  double y0[N];
  double h;
  STG f0[N];
  PHYS mu0[3];
};

// dense-output context of one step's stored samples k0 .. k0 + n - 1 of an item:
// y(t0 + x h) = qold + sum_r F[r] (x, 1 - x alternating powers), x = (k dt - t0) inv_h;
// prev: the item's previous context (-1 for its first)
// (field order: 16-byte aligned groups for vector loads)
template <typename STG, int NQ> struct alignas(16) SampleCtx {
  double qold[NQ];
  double t0, inv_h;
  int item, k0, n, prev;
  STG F[7][NQ];
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// ---- coefficient tables for CO2-Ar, staged in shared memory ----
// FP32 surface rows for the paired evaluation of the value c and the derivative dc of a
// radial function (co2ar_pes_grad_f2): 20 words per (interval, l),
//   (a3, 0 | a2, 3 a3), (a1, 2 a2 | a0, a1)       Horner of the (c, dc) pair in t
//   (b4, -4 b4 | b5, -5 b5), (b6, -6 b6 | b7, -7 b7)   against (R^-k, R^-(k+1))
//   (A, A k, k, 0)                                  the exponential A e^(k R)
constexpr int CO2AR_PAIR_WORDS = 20;
template <typename T> struct Co2arTables {
  T pes[CO2AR_TABLE];
  T dipx[CO2AR_TABLE];
  T dipz[CO2AR_TABLE];
  T rbound[CO2AR_NINT];
  T rlo[CO2AR_NINT];
  int fpes[CO2AR_NINT];
  int fdip[CO2AR_NINT];
  float4 pes2[sizeof(T) == 4 ? CO2AR_NINT * CO2AR_NL * CO2AR_PAIR_WORDS / 4 : 1];  // FP32 tables only
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
  if constexpr (sizeof(T) == 4) {
    float *w = reinterpret_cast<float *>(s->pes2);
    for (int e = threadIdx.x; e < CO2AR_NINT * CO2AR_NL * CO2AR_PAIR_WORDS; e += blockDim.x) {
      const double *r = g->pes + (e / CO2AR_PAIR_WORDS) * CO2AR_ROW;
      const int k = e % CO2AR_PAIR_WORDS;
      double v = 0.0;
      switch (k) {
        case 0: v = r[3]; break;
        case 2: v = r[2]; break;
        case 3: v = 3.0 * r[3]; break;
        case 4: v = r[1]; break;
        case 5: v = 2.0 * r[2]; break;
        case 6: v = r[0]; break;
        case 7: v = r[1]; break;
        case 8: v = r[4]; break;
        case 9: v = -4.0 * r[4]; break;
        case 10: v = r[5]; break;
        case 11: v = -5.0 * r[5]; break;
        case 12: v = r[6]; break;
        case 13: v = -6.0 * r[6]; break;
        case 14: v = r[7]; break;
        case 15: v = -7.0 * r[7]; break;
        case 16: v = r[8]; break;
        case 17: v = r[8] * r[9]; break;
        case 18: v = r[9]; break;
        default: v = 0.0;  // words 1 and 19
      }
      w[e] = float(v);
    }
  }
}

// ---- systems ----
// SOLO_ (every system): the solo kernel's instance, one trajectory per warp
template <typename PHYS, typename STG, bool COMP, bool SOLO_ = false> struct HeArSys {
  static constexpr bool SOLO = SOLO_;
  static constexpr int N = 6;
  static constexpr int QP = 6;
  // components the dipole and the R > Rcut test read: r
  static constexpr int NQ = 3;
  static constexpr bool RECORDS = false;
  static constexpr bool EST64 = true;  // FP64 error-estimate sums (err_terms)
  static constexpr int MOM2 = 6;  // no second momentum block
  static __device__ __forceinline__ constexpr int qidx(int i) { return i; }
  double inv_mu;
  // y in FP64 (the state) or in the stage precision (stage points)
  template <typename YT> __device__ void rhs(const YT *y, STG *f) const {
    PHYS r0 = PHYS(y[0]), r1 = PHYS(y[1]), r2 = PHYS(y[2]);
    PHYS R2 = r0 * r0 + r1 * r1 + r2 * r2;
    PHYS iR = inv_sqrt(R2);
    PHYS R = R2 * iR;
    PHYS V, dV;
    hear_V_dV<PHYS>(R, iR, V, dV);
    PHYS g = dV * iR;
    // dr/dt = p/mu in the stage precision
    f[0] = STG(STG(y[3]) * STG(inv_mu));
    f[1] = STG(STG(y[4]) * STG(inv_mu));
    f[2] = STG(STG(y[5]) * STG(inv_mu));
    f[3] = STG(-g * r0);
    f[4] = STG(-g * r1);
    f[5] = STG(-g * r2);
  }
  __device__ void dipole(const double *y, PHYS d[3]) const {
    PHYS r0 = PHYS(y[0]), r1 = PHYS(y[1]), r2 = PHYS(y[2]);
    PHYS R2 = r0 * r0 + r1 * r1 + r2 * r2;
    PHYS iR = inv_sqrt(R2);
    PHYS s = hear_dip<PHYS>(R2 * iR, iR) * iR;
    d[0] = s * r0;
    d[1] = s * r1;
    d[2] = s * r2;
  }
};

// V_R and V_x of the CO2-Ar surface, called out of line.  A DOP853 step with
// its dense output evaluates the right-hand side 15 times; inlined, the surface
// code is repeated at each of those sites and the loop no longer fits the
// instruction cache.  One shared copy costs a call per evaluation instead.
template <typename T> struct PesGrad {
  T VR, Vx;
};
// FP32 without compensation: the value c and derivative dc of each radial function as
// one (c, dc) pair through the paired FP32 instructions (fma2), from the pes2 rows; the
// sums over l as co2ar_pes forms them
__device__ __forceinline__ PesGrad<float> co2ar_pes_grad_f2(const Co2arTables<float> *tb, float R, float iR,
                                                           float x) {
  const int i = co2ar_interval<float>(R, tb->rbound);
  float P[11], dP[11];
  legendre10(x, P, dP);
  const float2 t = splat2(R - tb->rlo[i]);
  const int fl = tb->fpes[i];
  float2 q4 = make_float2(0.f, 0.f), q5 = q4, q6 = q4, q7 = q4;
  if (fl & 1) {
    const float iR2 = iR * iR, iR4 = iR2 * iR2;
    q4 = make_float2(iR4, iR4 * iR);   // (R^-4, R^-5)
    q5 = mul2(q4, splat2(iR));         // (R^-5, R^-6)
    q6 = mul2(q5, splat2(iR));
    q7 = mul2(q6, splat2(iR));
  }
  float aR = 0.f, ax = 0.f;
  const float4 *rows = tb->pes2 + (size_t)i * CO2AR_NL * (CO2AR_PAIR_WORDS / 4);
#pragma unroll
  for (int li = 0; li < CO2AR_NL; ++li) {
    const float4 *rw = rows + li * (CO2AR_PAIR_WORDS / 4);
    const float4 a = rw[0], b = rw[1];
    float2 c = fma2(make_float2(a.x, a.y), t, make_float2(a.z, a.w));
    c = fma2(c, t, make_float2(b.x, b.y));
    c = fma2(c, t, make_float2(b.z, b.w));
    if (fl & 1) {
      const float4 p = rw[2], q = rw[3];
      c = fma2(make_float2(p.x, p.y), q4, c);
      c = fma2(make_float2(p.z, p.w), q5, c);
      c = fma2(make_float2(q.x, q.y), q6, c);
      c = fma2(make_float2(q.z, q.w), q7, c);
    }
    if (fl & 2) {
      const float4 e = rw[4];
      c = fma2(make_float2(e.x, e.y), splat2(expf(e.z * R)), c);
    }
    aR = fmaf(P[2 * li], c.y, aR);
    ax = fmaf(dP[2 * li], c.x, ax);
  }
  const float sc = float(1.0 / HH_HTOCM);
  return {aR * sc, ax * sc};
}

template <typename T, bool COMP>
__device__ __noinline__ PesGrad<T> co2ar_pes_grad(const Co2arTables<T> *tb, T R, T iR, T x) {
  if constexpr (sizeof(T) == 4 && !COMP) {
    return co2ar_pes_grad_f2(tb, R, iR, x);
  } else {
    T V, VR, Vx;
    co2ar_pes<T, COMP>(tb->pes, tb->fpes, tb->rbound, tb->rlo, R, iR, x, V, VR, Vx, false);
    return {VR, Vx};
  }
}

// Body-frame dipole sums (d_z, a_x) of CO2-Ar, out of line for the same reason:
// the sample loop evaluates two pooled samples per lane and the item set-up one
// more, and each inlined copy repeats the whole dipole surface.
template <typename T> struct DipSums {
  T dz, ax;
};
template <typename T, bool COMP>
__device__ __noinline__ DipSums<T> co2ar_dip_sums(const Co2arTables<T> *tb, T R, T iR, T x) {
  T dz, ax;
  co2ar_dip<T, COMP>(tb->dipx, tb->dipz, tb->fdip, tb->rbound, tb->rlo, R, iR, x, dz, ax);
  return {dz, ax};
}

template <typename PHYS, typename STG, bool COMP, bool SOLO_ = false> struct Co2ArSys {
  static constexpr bool SOLO = SOLO_;
  static constexpr int N = 12;
  static constexpr int QP = 10;
  // components the dipole and the R > Rcut test read: r and u
  static constexpr int NQ = 6;
  static constexpr bool RECORDS = false;
  static constexpr bool EST64 = false;
  static constexpr int MOM2 = 9;  // j
  static __device__ __forceinline__ constexpr int qidx(int i) { return i < 3 ? i : i + 3; }
  double inv_mu, inv_II;
  const Co2arTables<PHYS> *tb;
  // y in FP64 (the state) or in the stage precision (stage points)
  template <typename YT> __device__ void rhs(const YT *y, STG *f) const {
    PHYS r[3] = {PHYS(y[0]), PHYS(y[1]), PHYS(y[2])};
    PHYS u[3] = {PHYS(y[6]), PHYS(y[7]), PHYS(y[8])};
    PHYS R2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    PHYS iR = inv_sqrt(R2);
    PHYS R = R2 * iR;
    PHYS iu = inv_sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    PHYS rh[3] = {r[0] * iR, r[1] * iR, r[2] * iR};
    PHYS uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    PHYS x = rh[0] * uh[0] + rh[1] * uh[1] + rh[2] * uh[2];
    const PesGrad<PHYS> g = co2ar_pes_grad<PHYS, COMP>(tb, R, iR, x);
    const PHYS VR = g.VR, Vx = g.Vx;
    PHYS a = VR - Vx * x * iR;  // dV/dr = a r^ + (Vx/R) u^
    PHYS b = Vx * iR;
    // kinematics in the stage precision: dr/dt = p/mu, du/dt = (j x u)/I
    const STG p0 = STG(y[3]), p1 = STG(y[4]), p2 = STG(y[5]);
    const STG u0 = STG(y[6]), u1 = STG(y[7]), u2 = STG(y[8]);
    const STG j0 = STG(y[9]), j1 = STG(y[10]), j2 = STG(y[11]);
    const STG im = STG(inv_mu), iI = STG(inv_II);
    f[0] = p0 * im;
    f[1] = p1 * im;
    f[2] = p2 * im;
    f[3] = STG(-(a * rh[0] + b * uh[0]));
    f[4] = STG(-(a * rh[1] + b * uh[1]));
    f[5] = STG(-(a * rh[2] + b * uh[2]));
    f[6] = (j1 * u2 - j2 * u1) * iI;
    f[7] = (j2 * u0 - j0 * u2) * iI;
    f[8] = (j0 * u1 - j1 * u0) * iI;
    // dj/dt = -Vx (u^ x r^)
    f[9] = STG(-Vx * (uh[1] * rh[2] - uh[2] * rh[1]));
    f[10] = STG(-Vx * (uh[2] * rh[0] - uh[0] * rh[2]));
    f[11] = STG(-Vx * (uh[0] * rh[1] - uh[1] * rh[0]));
  }
  // q = (r[3], u[3])
  __device__ void dipole(const double *q, PHYS d[3]) const {
    PHYS r[3] = {PHYS(q[0]), PHYS(q[1]), PHYS(q[2])};
    PHYS u[3] = {PHYS(q[3]), PHYS(q[4]), PHYS(q[5])};
    PHYS R2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    PHYS iR = inv_sqrt(R2);
    PHYS iu = inv_sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    PHYS rh[3] = {r[0] * iR, r[1] * iR, r[2] * iR};
    PHYS uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    PHYS x = rh[0] * uh[0] + rh[1] * uh[1] + rh[2] * uh[2];
    const DipSums<PHYS> ds = co2ar_dip_sums<PHYS, COMP>(tb, R2 * iR, iR, x);
    const PHYS dz = ds.dz, ax = ds.ax;
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = dz * rh[c] - ax * (uh[c] - x * rh[c]);
  }
};

// N2-Ar: rigid N2 (sites at +-L/2 u^) and Ar, PIP-NN surfaces of hh_n2ar.cuh.
// With a = (L/2) u^, d1 = |r - a| and d2 = |r + a| (N1-Ar, N2-Ar):
//   dV/dr = g1 (r - a)/d1 + g2 (r + a)/d2,  dV/du^ = (L/2)(-g1 (r - a)/d1 + g2 (r + a)/d2)
//   dp/dt = -dV/dr,  dj/dt = -u^ x dV/du^,  du/dt = (j x u)/I.
// Dipole: mu = d_z r^ + d_x (u^ - x r^)/|u^ - x r^| with the body-frame (d_x, d_z) at
// (R, x = r^.u^): the Euler-angle rotation of the reference (examples/correlation_n2_ar.cpp:52-76)
// maps body z to r^ and body x to the in-plane normal to r^ on the N1 side.
// SOLO_: the solo kernel's instance (one trajectory per warp), whose right-hand side
// the 32 lanes evaluate cooperatively (n2ar_pes_grad_coop)
template <typename PHYS, typename STG, bool COMP, bool SOLO_ = false> struct N2ArSys {
  static constexpr bool SOLO = SOLO_;
  static constexpr int N = 12;
  static constexpr int QP = 10;
  static constexpr int NQ = 6;
  static constexpr bool RECORDS = false;
  static constexpr bool EST64 = false;
  static constexpr int MOM2 = 9;  // j
  static __device__ __forceinline__ constexpr int qidx(int i) { return i < 3 ? i : i + 3; }
  double inv_mu, inv_II;
  const N2arDipFold *fold;      // shared-memory copies
  const N2arPesNet<PHYS> *pes;
  const float4 *dtab;           // mixed path: the dipole table (hh_n2ar.cuh), global memory
  template <typename YT> __device__ void rhs(const YT *y, STG *f) const {
    const PHYS r[3] = {PHYS(y[0]), PHYS(y[1]), PHYS(y[2])};
    const PHYS u[3] = {PHYS(y[6]), PHYS(y[7]), PHYS(y[8])};
    const PHYS iu = inv_sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const PHYS h = PHYS(N2AR_L / 2.0);
    const PHYS uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    PHYS e1[3], e2[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      e1[c] = r[c] - h * uh[c];
      e2[c] = r[c] + h * uh[c];
    }
    const PHYS i1 = inv_sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
    const PHYS i2 = inv_sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    N2arGrad<PHYS> g;
    if constexpr (SOLO)
      g = n2ar_pes_grad_coop<PHYS>(pes, PHYS(1) / i1, PHYS(1) / i2);
    else
      g = n2ar_pes_grad<PHYS>(pes, PHYS(1) / i1, PHYS(1) / i2);
    const PHYS a1 = g.g1 * i1, a2 = g.g2 * i2;
    PHYS Gr[3], Gu[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Gr[c] = a1 * e1[c] + a2 * e2[c];
      Gu[c] = h * (a2 * e2[c] - a1 * e1[c]);
    }
    const STG p0 = STG(y[3]), p1 = STG(y[4]), p2 = STG(y[5]);
    const STG u0 = STG(y[6]), u1 = STG(y[7]), u2 = STG(y[8]);
    const STG j0 = STG(y[9]), j1 = STG(y[10]), j2 = STG(y[11]);
    const STG im = STG(inv_mu), iI = STG(inv_II);
    f[0] = p0 * im;
    f[1] = p1 * im;
    f[2] = p2 * im;
    f[3] = STG(-Gr[0]);
    f[4] = STG(-Gr[1]);
    f[5] = STG(-Gr[2]);
    f[6] = (j1 * u2 - j2 * u1) * iI;
    f[7] = (j2 * u0 - j0 * u2) * iI;
    f[8] = (j0 * u1 - j1 * u0) * iI;
    f[9] = STG(-(uh[1] * Gu[2] - uh[2] * Gu[1]));
    f[10] = STG(-(uh[2] * Gu[0] - uh[0] * Gu[2]));
    f[11] = STG(-(uh[0] * Gu[1] - uh[1] * Gu[0]));
  }
  // q = (r[3], u[3]); the body-frame dipole is the FP64 network on the FP64 path and
  // the FP32 table of hh_n2ar.cuh (the network outside its R range) on the mixed path
  __device__ void dipole(const double *q, PHYS d[3]) const {
    const double R2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    const double iR = rsqrt(R2);
    const double iu = rsqrt(q[3] * q[3] + q[4] * q[4] + q[5] * q[5]);
    const double rh[3] = {q[0] * iR, q[1] * iR, q[2] * iR};
    const double uh[3] = {q[3] * iu, q[4] * iu, q[5] * iu};
    const double x = rh[0] * uh[0] + rh[1] * uh[1] + rh[2] * uh[2];
    const double e[3] = {uh[0] - x * rh[0], uh[1] - x * rh[1], uh[2] - x * rh[2]};
    const double en2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
    const double ie = en2 > 0.0 ? rsqrt(en2) : 0.0;
    N2arDipBody<double> b;
    if constexpr (sizeof(PHYS) == 4)
      b = dtab ? n2ar_dip_body_mixed(dtab, fold, R2 * iR, x, sqrt(en2)) : n2ar_dip_body(fold, R2 * iR, x);
    else
      b = n2ar_dip_body(fold, R2 * iR, x);
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = PHYS(b.dz * rh[c] + b.dx * e[c] * ie);
  }
};

// find_closest_integer / find_closest_half_integer (src/hawaii.c:360-393): the
// requantized |j| of the linear monomer.  The half-integer rule returns 0 below 0.25,
// 0.5 below 1 (the nearer of 0.5 and 1.5) and floor(j) + 0.5 above (the nearer of
// floor(j) + 0.5 and floor(j) + 1.5).
__device__ __forceinline__ double req_closest(int mode, double j) {
  if (mode == 1) return round(j);
  if (j < 0.25) return 0.0;
  if (j < 1.0) return 0.5;
  return floor(j) + 0.5;
}

// trajectory_apply_requantization (src/trajectory.c:93-136) on the Cartesian angular
// momentum j of the linear monomer: j scaled to the requantized length (the reference
// scales p_phi and p_theta, to which j is linear; zero when |j| <= 1e-15)
__device__ __forceinline__ void req_rescale(int mode, double &j0, double &j1, double &j2) {
  const double jl = sqrt(j0 * j0 + j1 * j1 + j2 * j2);
  const double s = jl > 1e-15 ? req_closest(mode, jl) / jl : 0.0;
  j0 *= s;
  j1 *= s;
  j2 *= s;
}

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
  if (SYS != SYS_HEAR) {
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
// The stage derivatives K stay in registers (all indices compile-time).
// Intermediate stage points are formed in the stage precision from a copy of
// the state in that precision: the right-hand side reads them in that precision
// anyway, and an FP32 stage point carries one rounding more than the FP32
// conversion of an FP64 one.  The 8th-order solution is formed in FP64.
// ---------------------------------------------------------------------------
template <int N, typename STG, int S>
__device__ __forceinline__ void stage_point(const STG (&K)[16][N], const STG *ys0, STG hs,
                                            STG *ys) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    STG acc = STG(0);
#pragma unroll
    for (int j = 0; j < S; ++j)
      if (hh_dop853_a[S][j] != 0.0) acc += STG(hh_dop853_a[S][j]) * K[j][i];
    ys[i] = ys0[i] + hs * acc;
  }
}

template <int N, typename STG>
__device__ __forceinline__ void solution_point(const STG (&K)[16][N], const double *y, double h,
                                               double *y_new) {
#pragma unroll
  for (int i = 0; i < N; ++i) {
    STG acc = STG(0);
#pragma unroll
    for (int j = 0; j < 12; ++j)
      if (hh_dop853_a[12][j] != 0.0) acc += STG(hh_dop853_a[12][j]) * K[j][i];
    y_new[i] = y[i] + h * double(acc);
  }
}

// scaled error estimates of component i (column i of K): the 5th- and 3rd-order
// estimates sum_j e_j K_j are stage sums, formed in the stage precision like the
// stage points; their scaling by the tolerance atol + max(|y|, |y_new|) rtol, the
// norm and the step controller are FP64.  FP32 stages: the estimate cannot resolve
// errors below the rounding noise of the stage derivatives, so that noise widens the
// scale.  (Measured on the CO2-Ar workload at rtol 3e-8: FP64 estimate sums let the
// steps grow, 4 % fewer, past what the FP32 stages resolve, and the C(t) error within
// the FP64 horizon rose from 1.9e-5 to 1.8e-4 while the kernel ran 12 % slower.)
// EST64: the estimate sums in FP64 (He-Ar: with its 6 state components they cost
// little, and its non-chaotic C(t) follows FP64 to 6e-5 with them against 1.6e-4
// with stage-precision sums)
template <typename STG, bool EST64, int NK>
__device__ __forceinline__ void err_terms(const STG (&K)[16][NK], int i, double y, double y_new, double h,
                                          const TrajParams &P, double &q5, double &q3) {
  double sc = P.atol + fmax(fabs(y), fabs(y_new)) * P.rtol;
  using ET = typename std::conditional<EST64, double, STG>::type;
  ET a5s = ET(0), a3s = ET(0), m5s = ET(0);
#pragma unroll
  for (int j = 0; j < 13; ++j) {
    if (hh_dop853_e5[j] != 0.0) {
      const ET t = ET(hh_dop853_e5[j]) * ET(K[j][i]);
      a5s += t;
      if (sizeof(STG) == 4) m5s += fabs(t);
    }
    if (hh_dop853_e3[j] != 0.0) a3s += ET(hh_dop853_e3[j]) * ET(K[j][i]);
  }
  const double a5 = double(a5s), a3 = double(a3s), m5 = double(m5s);
  if (sizeof(STG) == 4) sc += fabs(h) * P.noise_floor * m5;
  const double isc = 1.0 / sc;
  q5 = a5 * isc;
  q3 = a3 * isc;
}

// stages 1..12 of one step attempt from (y, K[0] = f(y)); y_new is the 8th-order
// solution and K[12] = f(y_new); returns the error norm
template <class Sys, typename STG>
__device__ __forceinline__ double step_attempt(const Sys &sys, const TrajParams &P,
                                               STG (&K)[16][Sys::N], const double *y, double h,
                                               double *y_new) {
  constexpr int N = Sys::N;
  STG ys0[N];
#pragma unroll
  for (int i = 0; i < N; ++i) ys0[i] = STG(y[i]);
  const STG hs = STG(h);
#define HH_STAGE(S)                                 \
  {                                                 \
    STG ys[N];                                      \
    stage_point<N, STG, S>(K, ys0, hs, ys);         \
    sys.rhs(ys, K[S]);                              \
  }
  HH_STAGE(1) HH_STAGE(2) HH_STAGE(3) HH_STAGE(4) HH_STAGE(5) HH_STAGE(6)
  HH_STAGE(7) HH_STAGE(8) HH_STAGE(9) HH_STAGE(10) HH_STAGE(11)
#undef HH_STAGE
  solution_point<N, STG>(K, y, h, y_new);
  sys.rhs(y_new, K[12]);
  // error control in FP64 on both paths: the 5th- and 3rd-order estimates are
  // FP64 sums of the stage derivatives, scaled and normed in FP64
  double e5 = 0.0, e3 = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double q5, q3;
    err_terms<STG, Sys::EST64>(K, i, y[i], y_new[i], h, P, q5, q3);
    e5 += q5 * q5;
    e3 += q3 * q3;
  }
  if (e5 == 0.0 && e3 == 0.0) return 0.0;
  return fabs(h) * e5 / sqrt((e5 + 0.01 * e3) * N);
}

// err^(-1/8) for the step controller
__device__ __forceinline__ double inv_eighth_root(double err) {
  return 1.0 / sqrt(sqrt(sqrt(err)));
}

// the three extra stages of the dense output and its coefficients F[7][NQ] for
// the components the samples read
template <class Sys, typename STG>
__device__ __forceinline__ void dense_stages(const Sys &sys, STG (&K)[16][Sys::N], const double *y_old,
                                             const double *y_new, double h, STG (&F)[7][Sys::NQ]) {
  constexpr int N = Sys::N;
  STG ys0[N];
#pragma unroll
  for (int i = 0; i < N; ++i) ys0[i] = STG(y_old[i]);
  const STG hs = STG(h);
#define HH_STAGE(S)                                 \
  {                                                 \
    STG ys[N];                                      \
    stage_point<N, STG, S>(K, ys0, hs, ys);         \
    sys.rhs(ys, K[S]);                              \
  }
  HH_STAGE(13) HH_STAGE(14) HH_STAGE(15)
#undef HH_STAGE
#pragma unroll
  for (int c = 0; c < Sys::NQ; ++c) {
    const int i = Sys::qidx(c);
    double dy = y_new[i] - y_old[i];
    F[0][c] = STG(dy);
    F[1][c] = STG(h * double(K[0][i]) - dy);
    F[2][c] = STG(2.0 * dy - h * (double(K[12][i]) + double(K[0][i])));
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      STG acc = STG(0);
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (hh_dop853_d[r][j] != 0.0) acc += STG(hh_dop853_d[r][j]) * K[j][i];
      F[3 + r][c] = STG(h * double(acc));
    }
  }
}

// ---- solo kernel: one trajectory per warp, component `lane` of the state per lane ----
// The stage sums, the 8th-order solution, the error terms and the dense-output
// coefficients of component i are formed by lane i with the same operations in
// the same order as the per-lane functions above; the stage points are gathered
// by shuffles and every lane evaluates the right-hand side on the full point.  The
// error norm is summed over the components in order.  A trajectory therefore takes
// the same steps in either kernel.
template <int N, typename T> __device__ __forceinline__ T pick_component(const T (&v)[N], int c) {
  T r = v[0];
#pragma unroll
  for (int i = 1; i < N; ++i)
    if (c == i) r = v[i];
  return r;
}

// K[S] of this lane's component from the stage point built from K[0..S-1]
template <class Sys, typename STG, int S>
__device__ __forceinline__ void cp_stage(const Sys &sys, STG (&K)[16][1], STG ys0, STG hs, int c) {
  constexpr int N = Sys::N;
  STG acc = STG(0);
#pragma unroll
  for (int j = 0; j < S; ++j)
    if (hh_dop853_a[S][j] != 0.0) acc += STG(hh_dop853_a[S][j]) * K[j][0];
  const STG ysc = ys0 + hs * acc;
  STG ys[N], f[N];
#pragma unroll
  for (int i = 0; i < N; ++i) ys[i] = __shfl_sync(0xffffffffu, ysc, i);
  sys.rhs(ys, f);
  K[S][0] = pick_component<N>(f, c);
}

template <class Sys, typename STG>
__device__ __forceinline__ double step_attempt_cp(const Sys &sys, const TrajParams &P, STG (&K)[16][1],
                                                  double y, double h, double &y_new) {
  constexpr int N = Sys::N;
  const int lane = threadIdx.x & 31;
  const int c = lane < N ? lane : N - 1;
  const STG ys0 = STG(y);
  const STG hs = STG(h);
  cp_stage<Sys, STG, 1>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 2>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 3>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 4>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 5>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 6>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 7>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 8>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 9>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 10>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 11>(sys, K, ys0, hs, c);
  {
    STG acc = STG(0);
#pragma unroll
    for (int j = 0; j < 12; ++j)
      if (hh_dop853_a[12][j] != 0.0) acc += STG(hh_dop853_a[12][j]) * K[j][0];
    y_new = y + h * double(acc);
    double yn[N];
    STG f[N];
#pragma unroll
    for (int i = 0; i < N; ++i) yn[i] = __shfl_sync(0xffffffffu, y_new, i);
    sys.rhs(yn, f);
    K[12][0] = pick_component<N>(f, c);
  }
  double q5, q3;
  err_terms<STG, Sys::EST64>(K, 0, y, y_new, h, P, q5, q3);
  double e5 = 0.0, e3 = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double v5 = __shfl_sync(0xffffffffu, q5, i), v3 = __shfl_sync(0xffffffffu, q3, i);
    e5 += v5 * v5;
    e3 += v3 * v3;
  }
  if (e5 == 0.0 && e3 == 0.0) return 0.0;
  return fabs(h) * e5 / sqrt((e5 + 0.01 * e3) * N);
}

// stages 13..15 and this lane's dense-output coefficients F[0..6]
template <class Sys, typename STG>
__device__ __forceinline__ void dense_stages_cp(const Sys &sys, STG (&K)[16][1], double y_old, double y_new,
                                                double h, STG (&F)[7]) {
  constexpr int N = Sys::N;
  const int lane = threadIdx.x & 31;
  const int c = lane < N ? lane : N - 1;
  const STG ys0 = STG(y_old);
  const STG hs = STG(h);
  cp_stage<Sys, STG, 13>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 14>(sys, K, ys0, hs, c);
  cp_stage<Sys, STG, 15>(sys, K, ys0, hs, c);
  double dy = y_new - y_old;
  F[0] = STG(dy);
  F[1] = STG(h * double(K[0][0]) - dy);
  F[2] = STG(2.0 * dy - h * (double(K[12][0]) + double(K[0][0])));
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    STG acc = STG(0);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      if (hh_dop853_d[r][j] != 0.0) acc += STG(hh_dop853_d[r][j]) * K[j][0];
    F[3 + r] = STG(h * double(acc));
  }
}

// dense output y(t_old + x h) = y_old + x(F0 + (1-x)(F1 + x(F2 + ... ))); the
// increment is formed in STG precision and added to the FP64 state
template <class Sys, typename STG>
__device__ __forceinline__ void dense_eval(const double *y_old, const STG (&F)[7][Sys::NQ], double x,
                                           double *q) {
  const STG xs = STG(x), x1 = STG(1) - STG(x);
#pragma unroll
  for (int i = 0; i < Sys::NQ; ++i) {
    STG v = F[6][i] * xs;
    v = (v + F[5][i]) * x1;
    v = (v + F[4][i]) * xs;
    v = (v + F[3][i]) * x1;
    v = (v + F[2][i]) * xs;
    v = (v + F[1][i]) * x1;
    v = (v + F[0][i]) * xs;
    q[i] = y_old[Sys::qidx(i)] + double(v);
  }
}

// Per-item set-up, out of line (once per half-trajectory): Cartesian initial
// state (momenta inverted for the backward branch), mu0, f(y0) and the initial
// step size of Hairer's algorithm (error-estimator order 7).
template <class Sys, typename PHYS, typename STG>
__device__ __noinline__ void item_setup(const Sys &sys, const TrajParams &P, const double *qp,
                                        int dir, double *y0, STG *f0, PHYS *mu0, double *h_out) {
  constexpr int N = Sys::N;
  if constexpr (Sys::N == 19) {
    ch4co2_qp_to_state(qp, nullptr, y0);
  } else {
    qp_to_state<(N == 6) ? SYS_HEAR : SYS_CO2AR>(qp, y0);
    // PR_MU requantization at the start of the trajectory (src/hawaii.c:3558): the
    // switch is on when a trajectory starts
    if constexpr (N == 12)
      if (P.req_mode) req_rescale(P.req_mode, y0[9], y0[10], y0[11]);
  }
  double q0[Sys::NQ];
#pragma unroll
  for (int c = 0; c < Sys::NQ; ++c) q0[c] = y0[Sys::qidx(c)];
  sys.dipole(q0, mu0);
  if (dir) {
    // invert_momenta (src/hawaii.c:1171-1188): p -> -p, j -> -j (and L)
#pragma unroll
    for (int i = 3; i < 6; ++i) y0[i] = -y0[i];
#pragma unroll
    for (int i = Sys::MOM2; i < N; ++i) y0[i] = -y0[i];
  }
  sys.rhs(y0, f0);
  // the sampled window bounds the first step (one sample interval when N = 1,
  // where only the t = 0 term is kept)
  const double span = P.dt * double(P.N > 1 ? P.N - 1 : 1);
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
  double d2 = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double sc = P.atol + fabs(y0[i]) * P.rtol;
    double a = (double(f1[i]) - double(f0[i])) / sc;
    d2 += a * a;
  }
  d2 = sqrt(d2 / N) / h0;
  double h1 = (d1 <= 1e-15 && d2 <= 1e-15) ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / fmax(d1, d2), 0.125);
  *h_out = fmin(fmin(100.0 * h0, h1), span);
}

// per-warp pool of dense-output contexts for the pooled sample evaluation
// jobs per chunk: one per lane (measured against 64 and 128: 16 % and 35 % more
// trajectories/s than those on the CO2-Ar bench)
constexpr int SAMPLE_CHUNK = 32;
template <typename STG, typename PHYS, int NQ> struct WarpSamples {
  STG F[7][NQ][32];
  double qold[NQ][32];
  double t0[32];
  double inv_h[32];
  double *crln[32];
  const double *satw[32];
  PHYS mu0[3][32];
  PHYS prev[32];   // the owner's last stored sample before this round
  PHYS tail[32];   // the owner's last sample of the previous chunk
  PHYS last[32];   // the owner's last stored sample
  PHYS res[SAMPLE_CHUNK];
  int kst[32];
  int off[32];
  int item[32];
  unsigned cut[32];  // (end << 3) | reason; end = index past the last stored sample
};

__device__ __forceinline__ void warp_add_counter(unsigned long long *dst, unsigned v) {
  unsigned long long s = v;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(dst, s);
}

// state of an open item between the bulk and the solo kernel
template <int N, typename PHYS, typename STG> struct HandoffState {
  double y[N];
  STG f0[N];  // f(y) (first stage of the next step)
  double t, h;
  PHYS mu0[3], curr;
  int item, k, since, total, flags;  // flags: rejected | exited << 1
  int req;                           // requantization switch and torque runs (REQ kernels)
  unsigned steps, samples, t_begin;  // item trace so far
  int last_ctx;                      // deferred samples: the item's last context
};

// ---------------------------------------------------------------------------
// warp-synchronous persistent loop over half-trajectory items
// ---------------------------------------------------------------------------
// REQ: PR_MU requantization of the linear monomer (src/hawaii.c:3604-3662,
// src/trajectory.c:146-183).  Steps land on every sample time, where the reference's
// make_step returns; at sample k the switch of sample k - 1 decides whether j is
// requantized (and the stages restarted from the new state), then the torque |dj/dt|
// at sample k enters the switch: on once the last req_len torques are all <= the
// limit, off once they are all >= it.  The torque cache starts as zeros, i.e. with
// req_len values below the limit.
template <class Sys, typename PHYS, typename STG, bool REQ = false>
__device__ __forceinline__ void traj_body(const Sys &sys, const TrajParams &P, const TrajIO &io,
                                          WarpSamples<STG, PHYS, Sys::NQ> *ws_block) {
  constexpr int N = Sys::N;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  WarpSamples<STG, PHYS, Sys::NQ> *ws = ws_block + (threadIdx.x >> 5);
  const double dt = P.dt;
  unsigned nsteps = 0, nrej = 0, nrhs = 0, nsamp = 0, ndense = 0, nitems = 0;
  // per-lane item state
  // bulk: the whole state per lane; solo: component `lane` (clamped to N - 1) per lane
  constexpr int NL = Sys::SOLO ? 1 : N;
  const int comp = lane < N ? lane : N - 1;
  STG K[16][NL];
  double y[NL], y_new[NL];
  double t = 0.0, h = 0.0;
  PHYS mu0[3] = {PHYS(0), PHYS(0), PHYS(0)};
  PHYS curr = PHYS(0);  // the item's last stored sample
  double *crln = io.crln;
  const double *satw = nullptr;  // this trajectory's satellite weights
  int item = -1;           // -1: needs an item, -2: queue exhausted
  // deferred samples: contexts instead of in-kernel dipoles (plain C(t) only)
  const bool defer = !Sys::RECORDS && io.ctx != nullptr;
  int last_ctx = -1;       // deferred samples: the item's last context
  int k = 1;
  int since = 0, total = 0;
  bool rejected = false;
  bool exited = false;  // the item ended by R > Rcut
  // REQ: bit 0 the requantization switch, bits 1..15 the run of trailing torques <= the
  // limit, bits 16..30 the run of trailing torques >= the limit (each capped at req_len)
  int req = 0;
  const int req_cap = REQ ? min(P.req_len, 16383) : 0;
  unsigned long long t_begin = 0ull;
  unsigned s0 = 0, m0 = 0;
  // the owner of the warp's item in solo mode (every other lane mirrors it); all
  // lanes own their items in bulk mode
  const bool owner = !Sys::SOLO || lane == 0;
  using Handoff = HandoffState<Sys::N, PHYS, STG>;
  // start item `it` from its phase point (all lanes of the warp that call it)
  auto start_item = [&](int it) {
    item = it;
    const int traj = item >> 1;
    crln = io.crln + (size_t)(traj / io.traj_per_iter) * (size_t)P.N;
    satw = io.sat_w ? io.sat_w + (size_t)traj * io.n_sat : nullptr;
    if (io.item_trace) t_begin = globaltimer_ns();
    s0 = nsteps;
    m0 = nsamp;
    // out-of-line set-up writes through pointers to temporaries only, so
    // y, K and mu0 never become addressable and stay in registers
    double y_t[N];
    STG f_t[N];
    PHYS mu_t[3];
    if (io.setup) {
      const auto *st = static_cast<const ItemStart<N, PHYS, STG> *>(io.setup) + item;
#pragma unroll
      for (int i = 0; i < N; ++i) {
        y_t[i] = st->y0[i];
        f_t[i] = st->f0[i];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) mu_t[c] = st->mu0[c];
      h = st->h;
    } else {
      item_setup<Sys, PHYS, STG>(sys, P, io.ic + (size_t)traj * Sys::QP, item & 1, y_t, f_t, mu_t, &h);
    }
    if constexpr (Sys::SOLO) {
      y[0] = pick_component<N>(y_t, comp);
      K[0][0] = pick_component<N>(f_t, comp);
    } else {
#pragma unroll
      for (int i = 0; i < N; ++i) {
        y[i] = y_t[i];
        K[0][i] = f_t[i];
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) mu0[c] = mu_t[c];
    if (owner) {
      if constexpr (Sys::RECORDS) {
        if ((item & 1) == 0) {
          PHYS *rec = static_cast<PHYS *>(io.records) + (size_t)traj * io.rec_stride * HH_REC_WORDS;
#pragma unroll
          for (int c = 0; c < Sys::NQ; ++c) rec[c] = PHYS(y_t[Sys::qidx(c)]);
        }
      } else {
        if (io.series && (item & 1) == 0) {
          PHYS *sv = static_cast<PHYS *>(io.series) + (size_t)traj * io.rec_stride * 4;
#pragma unroll
          for (int c = 0; c < 3; ++c) sv[c] = mu_t[c];
        }
      }
    }
    nrhs += 2;
    t = 0.0;
    k = 1;
    since = total = 0;
    rejected = false;
    exited = false;
    curr = PHYS(0);
    if constexpr (REQ) req = 1 | (req_cap << 1);
    last_ctx = -1;
    if (defer && owner) {
      PHYS *m = static_cast<PHYS *>(io.item_mu0) + (size_t)item * 4;
#pragma unroll
      for (int c = 0; c < 3; ++c) m[c] = mu_t[c];
      m[3] = mu_t[0] * mu_t[0] + mu_t[1] * mu_t[1] + mu_t[2] * mu_t[2];
    }
  };
  auto item_of = [&](unsigned idx) {
    return io.items ? io.items[idx] : (io.fwd_only ? 2 * (int)idx : (int)idx);
  };
  bool handing = false;  // bulk mode: this warp hands its open items to the solo kernel
  unsigned round = 0;
  int sync_round = 0;    // bulk mode: rounds since the last block barrier
  for (;;) {
    if constexpr (!Sys::SOLO) {
      // ---- hand-off: once few items remain open, store them for the solo kernel ----
      if (io.handoff && !handing && ((++round & 7u) == 0u)) {
        unsigned done = 0;
        if (lane == 0) done = *reinterpret_cast<volatile unsigned int *>(io.done);
        done = __shfl_sync(FULL, done, 0);
        handing = (unsigned)io.n_items - done <= io.handoff_at;
      }
      if (handing) {
        if (item >= 0) {
          Handoff *hs = static_cast<Handoff *>(io.handoff) + atomicAdd(io.n_handoff, 1u);
#pragma unroll
          for (int i = 0; i < N; ++i) {
            hs->y[i] = y[i];
            hs->f0[i] = K[0][i];
          }
          hs->t = t;
          hs->h = h;
#pragma unroll
          for (int c = 0; c < 3; ++c) hs->mu0[c] = mu0[c];
          hs->curr = curr;
          hs->item = item;
          hs->k = k;
          hs->since = since;
          hs->total = total;
          hs->flags = (rejected ? 1 : 0) | (exited ? 2 : 0);
          hs->req = req;
          hs->steps = nsteps - s0;
          hs->samples = nsamp - m0;
          hs->t_begin = (unsigned)(t_begin & 0xffffffffu);
          hs->last_ctx = last_ctx;
        }
        item = -2;
      }
      // ---- refill: lanes without an item take the next ones (one atomic per warp) ----
      const bool need = (item == -1);
      const unsigned needmask = __ballot_sync(FULL, need);
      if (needmask) {
        unsigned base = 0;
        const int leader = __ffs(needmask) - 1;
        if (lane == leader) base = atomicAdd(io.queue, (unsigned)__popc(needmask));
        base = __shfl_sync(FULL, base, leader);
        if (need) {
          const unsigned idx = base + __popc(needmask & ((1u << lane) - 1u));
          if (idx < (unsigned)io.n_items) start_item(item_of(idx));
          else item = -2;
        }
      }
    } else {
      // ---- solo refill: the warp resumes a handed-off item, else takes the next
      // one from the queue; every lane holds the same item ----
      if (item == -1) {
        unsigned idx = 0;
        if (lane == 0) idx = atomicAdd(io.solo_cursor, 1u);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx < *io.n_handoff) {
          const Handoff *hs = static_cast<const Handoff *>(io.handoff) + idx;
          y[0] = hs->y[comp];
          K[0][0] = hs->f0[comp];
          t = hs->t;
          h = hs->h;
#pragma unroll
          for (int c = 0; c < 3; ++c) mu0[c] = hs->mu0[c];
          curr = hs->curr;
          item = hs->item;
          k = hs->k;
          since = hs->since;
          total = hs->total;
          rejected = (hs->flags & 1) != 0;
          req = hs->req;
          exited = (hs->flags & 2) != 0;
          s0 = nsteps - hs->steps;
          m0 = nsamp - hs->samples;
          t_begin = hs->t_begin;
          last_ctx = hs->last_ctx;
          const int traj = item >> 1;
          crln = io.crln + (size_t)(traj / io.traj_per_iter) * (size_t)P.N;
          satw = io.sat_w ? io.sat_w + (size_t)traj * io.n_sat : nullptr;
        } else {
          unsigned q = 0;
          if (lane == 0) q = atomicAdd(io.queue, 1u);
          q = __shfl_sync(FULL, q, 0);
          if (q < (unsigned)io.n_items) start_item(item_of(q));
          else item = -2;
        }
      }
    }
    bool all_done = __all_sync(FULL, item == -2);
    if constexpr (!Sys::SOLO) {
      // block-uniform exit with the round barrier, every block_sync-th round (every
      // warp takes every round; between barriers no warp leaves)
      if (P.block_sync) {
        all_done = (sync_round == 0) ? (__syncthreads_and(all_done ? 1 : 0) != 0) : false;
        if (++sync_round == P.block_sync) sync_round = 0;
      }
    }
    if (all_done) break;
    const bool active = (item >= 0);

    // ---- one step attempt for every lane that holds an item ----
    int status = -1;  // >= 0: this lane's item ended with that status this round
    int hard = 0;
    bool accepted = false;
    bool landed = false;  // REQ: the step ends exactly at sample time k dt
    double h_taken = 0.0;
    if (active) {
      // 10 * spacing of doubles above t (t >= 0 and finite)
      const double min_step = 10.0 * (__longlong_as_double(__double_as_longlong(t) + 1) - t);
      double h_att = h;
      bool clamp = false;
      if constexpr (REQ) {
        const double to_k = double(k) * dt - t;
        if (h_att >= to_k) {
          h_att = to_k;
          clamp = true;
        }
      }
      if (!(h_att >= min_step)) {
        status = HH_ST_H_UNDERFLOW;
      } else {
        double err;
        if constexpr (Sys::SOLO)
          err = step_attempt_cp<Sys, STG>(sys, P, K, y[0], h_att, y_new[0]);
        else
          err = step_attempt<Sys, STG>(sys, P, K, y, h_att, y_new);
        nrhs += 12;
        if (err < 1.0) {
          double fac = (err == 0.0) ? 10.0 : fmin(10.0, 0.9 * inv_eighth_root(err));
          if (rejected) fac = fmin(1.0, fac);
          rejected = false;
          h_taken = h_att;
          // a step shortened to land on a sample time keeps the longer proposal
          h = clamp ? fmax(h, h_att * fac) : h_att * fac;
          landed = clamp;
          accepted = true;
          ++nsteps;
        } else {
          h = h_att * fmax(0.2, 0.9 * inv_eighth_root(err));
          rejected = true;
          ++nrej;
        }
      }
    }

    // ---- dense output and samples for steps that passed a sample time ----
    // The steps of the 32 lanes pass very different numbers of sample times
    // (none inside a collision, dozens in free flight), so the samples are
    // pooled: each lane publishes its dense-output context to shared memory,
    // and all lanes evaluate the pooled (owner, k) jobs in chunks.  A sample
    // the reference would not have stored (after an R > Rcut exit or a
    // failure) is cut off per owner with an atomicMin on (end, reason).
    bool pending = accepted && (landed || double(k) * dt <= t + h_taken);
    const double t_land = double(k) * dt;  // REQ: the sample time a landed step ends at
    if (__any_sync(FULL, pending)) {
      int cnt = 0;
      int nsafe = 0;  // deferred samples: stored without per-sample R > Rcut tests
      if (pending) {
        STG F[7][Sys::NQ];
        if constexpr (Sys::SOLO) {
          // this lane's component; published below by the lane that holds it
          STG Fc[7];
          if constexpr (REQ) {
            // the sample is the step's end point: y_old + dy at x = 1
            Fc[0] = STG(y_new[0] - y[0]);
#pragma unroll
            for (int r = 1; r < 7; ++r) Fc[r] = STG(0);
          } else {
            dense_stages_cp<Sys, STG>(sys, K, y[0], y_new[0], h_taken, Fc);
          }
#pragma unroll
          for (int cq = 0; cq < Sys::NQ; ++cq)
            if (Sys::qidx(cq) == lane) {
#pragma unroll
              for (int r = 0; r < 7; ++r) ws->F[r][cq][0] = Fc[r];
              ws->qold[cq][0] = y[0];
            }
        } else {
          if constexpr (REQ) {
#pragma unroll
            for (int c = 0; c < Sys::NQ; ++c) {
              F[0][c] = STG(y_new[Sys::qidx(c)] - y[Sys::qidx(c)]);
#pragma unroll
              for (int r = 1; r < 7; ++r) F[r][c] = STG(0);
            }
          } else {
            dense_stages<Sys, STG>(sys, K, y, y_new, h_taken, F);
          }
        }
        if (!REQ) nrhs += 3;
        ++ndense;
        const double t_new = t + h_taken;
        int kl = (int)fmin(floor(t_new / dt), double(P.N - 1));
        while (kl + 1 <= P.N - 1 && double(kl + 1) * dt <= t_new) ++kl;
        while (kl > k && double(kl) * dt > t_new) --kl;
        if (REQ && landed) kl = k;
        cnt = owner ? kl - k + 1 : 0;  // solo mode: the owner's samples, evaluated by all lanes
        if constexpr (!Sys::SOLO && !Sys::RECORDS) {
          // deferred samples: no sample of the step can pass R > Rcut when the bound
          // |r(x)| <= max(|r_old|, |r_old + F0|) + sum_i c_i |F_i| of the dense-output
          // polynomial y = y_old + F0 x + F1 x(1-x) + F2 x^2(1-x) + ... + F6 x^4(1-x)^3
          // (c_i the maxima of its basis on [0, 1]; |r_old + F0 x| is convex in x) stays
          // below Rcut with a margin for the FP32 evaluation; such steps store all
          // their samples without pooled tests
          if (defer && cnt > 0) {
            constexpr double cb[7] = {0.0, 0.25, 4.0 / 27.0, 1.0 / 16.0, 108.0 / 3125.0, 1.0 / 64.0,
                                      6912.0 / 823543.0};
            double ro2 = 0.0, rn2 = 0.0, f02 = 0.0, tail = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const double qo = y[Sys::qidx(c)], f0 = double(F[0][c]);
              ro2 += qo * qo;
              rn2 += (qo + f0) * (qo + f0);
              f02 += f0 * f0;
            }
#pragma unroll
            for (int r = 1; r < 7; ++r) {
              const double a0 = F[r][0], a1 = F[r][1], a2 = F[r][2];
              tail += cb[r] * sqrt(a0 * a0 + a1 * a1 + a2 * a2);
            }
            const double bound = fmax(sqrt(ro2), sqrt(rn2)) + tail;
            if (bound + 1e-5 * (sqrt(f02) + tail) + 1e-12 * bound < P.Rcut) {
              nsafe = cnt;
              nsamp += cnt;  // evaluated by the sample kernels
              cnt = 0;
            }
          }
        }
        if (owner) {
          if constexpr (!Sys::SOLO) {
#pragma unroll
            for (int r = 0; r < 7; ++r)
#pragma unroll
              for (int c = 0; c < Sys::NQ; ++c) ws->F[r][c][lane] = F[r][c];
#pragma unroll
            for (int c = 0; c < Sys::NQ; ++c) ws->qold[c][lane] = y[Sys::qidx(c)];
          }
#pragma unroll
          for (int c = 0; c < 3; ++c) ws->mu0[c][lane] = mu0[c];
          ws->t0[lane] = t;
          ws->inv_h[lane] = 1.0 / h_taken;
          ws->prev[lane] = curr;
          ws->crln[lane] = crln;
          ws->satw[lane] = satw;
          ws->kst[lane] = k;
          ws->item[lane] = item;
          ws->cut[lane] = 0xffffffffu;
        }
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
      }
      const int my_off = incl - cnt;
      const int pooled = __shfl_sync(FULL, incl, 31);
      ws->off[lane] = my_off;
      __syncwarp();
      for (int base = 0; base < pooled; base += SAMPLE_CHUNK) {
        const int m = min(SAMPLE_CHUNK, pooled - base);
        // (1) evaluate: each lane takes jobs jj = lane, lane + 32
        int own[SAMPLE_CHUNK / 32];
        int kks[SAMPLE_CHUNK / 32];
        bool nan_[SAMPLE_CHUNK / 32], out_[SAMPLE_CHUNK / 32];
#pragma unroll
        for (int u = 0; u < SAMPLE_CHUNK / 32; ++u) {
          const int jj = lane + 32 * u;
          own[u] = -1;
          if (jj < m) {
            const int j = base + jj;
            int o = 0;  // owner: the largest lane whose offset is <= j
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
              if (o + step <= 31 && ws->off[o + step] <= j) o += step;
            const int kk = ws->kst[o] + (j - ws->off[o]);
            const double x = (double(kk) * dt - ws->t0[o]) * ws->inv_h[o];
            const STG xs = STG(x), x1 = STG(1) - STG(x);
            double q[Sys::NQ];
#pragma unroll
            for (int c = 0; c < Sys::NQ; ++c) {
              if (c >= 3 && defer) {  // deferred: only r, for the R > Rcut test
                q[c] = 0.0;
                continue;
              }
              STG v = ws->F[6][c][o] * xs;
              v = (v + ws->F[5][c][o]) * x1;
              v = (v + ws->F[4][c][o]) * xs;
              v = (v + ws->F[3][c][o]) * x1;
              v = (v + ws->F[2][c][o]) * xs;
              v = (v + ws->F[1][c][o]) * x1;
              v = (v + ws->F[0][c][o]) * xs;
              q[c] = ws->qold[c][o] + double(v);
            }
            ++nsamp;
            own[u] = o;
            kks[u] = kk;
            out_[u] = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] > P.Rcut * P.Rcut;
            if constexpr (Sys::RECORDS) {
              const int it = ws->item[o];
              const size_t slot = (size_t)(it >> 1) * io.rec_stride + ((it & 1) ? P.N - 1 + kk : kk);
              PHYS *rec = static_cast<PHYS *>(io.records) + slot * HH_REC_WORDS;
#pragma unroll
              for (int c = 0; c < Sys::NQ; ++c) rec[c] = PHYS(q[c]);
              nan_[u] = false;
              ws->res[jj] = PHYS(1);
            } else if (defer) {
              nan_[u] = false;
              ws->res[jj] = PHYS(1);
            } else {
              PHYS d[3];
              sys.dipole(q, d);
              nan_[u] = isnan(d[0]) || isnan(d[1]) || isnan(d[2]);
              ws->res[jj] = ws->mu0[0][o] * d[0] + ws->mu0[1][o] * d[1] + ws->mu0[2][o] * d[2];
              if (io.series) {
                const int it = ws->item[o];
                const size_t slot = (size_t)(it >> 1) * io.rec_stride + ((it & 1) ? P.N - 1 + kk : kk);
                PHYS *sv = static_cast<PHYS *>(io.series) + slot * 4;
                const bool zero = P.prmu && nan_[u];
#pragma unroll
                for (int c = 0; c < 3; ++c) sv[c] = zero ? PHYS(0) : d[c];
              }
              if (P.prmu && nan_[u]) out_[u] = false;
            }
          }
        }
        __syncwarp();
        // (2) the reference's per-sample tests (src/hawaii.c:2183-2243), in its order
#pragma unroll
        for (int u = 0; u < SAMPLE_CHUNK / 32; ++u) {
          const int o = own[u];
          if (o >= 0) {
            const int jj = lane + 32 * u;
            const int j = base + jj;
            const PHYS val = ws->res[jj];
            unsigned code = 0xffffffffu;
            if (Sys::RECORDS || P.prmu || defer) {
              // a record's or a deferred sample's dipole checks run after the batched
              // evaluation; PR_MU has none
              if (out_[u]) code = (unsigned(j + 1) << 3);
            } else if (nan_[u]) code = (unsigned(j) << 3) | 1u;
            else if (ws->item[o] == P.inject_item && kks[u] == P.inject_k) code = (unsigned(j) << 3) | 4u;
            else if (fabs(double(val)) > 1e100) code = (unsigned(j) << 3) | 2u;
            else {
              const PHYS pv = (j == ws->off[o]) ? ws->prev[o] : (jj == 0 ? ws->tail[o] : ws->res[jj - 1]);
              if (kks[u] > 1 && fabs(double(val) / double(pv)) > 1e10) code = (unsigned(j) << 3) | 3u;
              else if (out_[u]) code = (unsigned(j + 1) << 3);  // stored, then the branch ends
            }
            if (code != 0xffffffffu) atomicMin(&ws->cut[o], code);
          }
        }
        __syncwarp();
        // (3) commit the samples before each owner's cut
#pragma unroll
        for (int u = 0; u < SAMPLE_CHUNK / 32; ++u) {
          const int o = own[u];
          if (o >= 0) {
            const int jj = lane + 32 * u;
            const int j = base + jj;
            const PHYS val = ws->res[jj];
            const unsigned cut = ws->cut[o];
            const int end_o = (o == 31) ? pooled : ws->off[o + 1];
            const int stop = (cut == 0xffffffffu) ? end_o : min(end_o, int(cut >> 3));
            const int chunk_end = min(end_o, base + m);
            if (j < stop) {
              if (Sys::RECORDS || io.series || defer) {
                // written in (1), or by the sample kernels
              } else if (io.n_sat == 0) {
                atomicAdd(&ws->crln[o][kks[u]], P.weight * double(val));
              } else {
                const double *w = ws->satw[o];
                for (int s = 0; s < io.n_sat; ++s)
                  atomicAdd(&ws->crln[o][(size_t)s * P.N + kks[u]], P.weight * w[s] * double(val));
              }
              // the owner's last stored sample so far (a cut found in a later
              // chunk lies past every sample of this one)
              if (j == min(stop, chunk_end) - 1) ws->last[o] = val;
            }
            if (j == chunk_end - 1) ws->tail[o] = val;
          }
        }
        __syncwarp();
      }
      if constexpr (!Sys::RECORDS) {
        if (defer) {
          // one context per owner with stored samples (one atomic per warp)
          int nc = 0;
          if (pending && owner) {
            const unsigned cut = ws->cut[lane];
            nc = nsafe + ((cut == 0xffffffffu) ? my_off + cnt : min(my_off + cnt, int(cut >> 3))) - my_off;
          }
          const unsigned wm = __ballot_sync(FULL, nc > 0);
          if (wm) {
            unsigned long long cbase = 0;
            const int leader = __ffs(wm) - 1;
            if (lane == leader) cbase = atomicAdd(io.ctx_count, (unsigned long long)__popc(wm));
            cbase = __shfl_sync(FULL, cbase, leader);
            if (nc > 0) {
              const unsigned long long idx = cbase + __popc(wm & ((1u << lane) - 1u));
              if (idx < io.ctx_cap) {
                const int col = Sys::SOLO ? 0 : lane;
                auto *cx = static_cast<SampleCtx<STG, Sys::NQ> *>(io.ctx) + idx;
#pragma unroll
                for (int r = 0; r < 7; ++r)
#pragma unroll
                  for (int c = 0; c < Sys::NQ; ++c) cx->F[r][c] = ws->F[r][c][col];
#pragma unroll
                for (int c = 0; c < Sys::NQ; ++c) cx->qold[c] = ws->qold[c][col];
                cx->t0 = ws->t0[lane];
                cx->inv_h = ws->inv_h[lane];
                cx->item = item;
                cx->k0 = k;
                cx->n = nc;
                cx->prev = last_ctx;
              }
              // past the capacity the host repeats the call with a larger buffer
              last_ctx = (int)idx;
            }
          }
        }
      }
      if (pending && owner) {
        const unsigned cut = ws->cut[lane];
        const int stop = (cut == 0xffffffffu) ? my_off + cnt : min(my_off + cnt, int(cut >> 3));
        const int committed = nsafe + stop - my_off;
        if (committed > 0) {
          k += committed;
          curr = ws->last[lane];
          since = 0;
        }
        if (cut != 0xffffffffu) {
          switch (cut & 7u) {
            case 0: status = HH_ST_OK; exited = true; break;  // R > Rcut
            case 1: status = HH_ST_NAN_DIPOLE; hard = 1; break;
            case 2: status = HH_ST_OVERFLOW; hard = 1; break;
            case 3: status = HH_ST_JUMP; hard = 1; break;
            default:
              status = P.inject_status;
              hard = (P.inject_status >= HH_ST_NAN_DIPOLE);
              break;
          }
        }
      }
      if constexpr (Sys::SOLO) {
        // the other lanes follow the owner's progress
        k = __shfl_sync(FULL, k, 0);
        curr = __shfl_sync(FULL, curr, 0);
        since = __shfl_sync(FULL, since, 0);
        status = __shfl_sync(FULL, status, 0);
        hard = __shfl_sync(FULL, hard, 0);
        exited = __shfl_sync(FULL, exited ? 1 : 0, 0) != 0;
      }
      __syncwarp();
    }

    // ---- advance accepted lanes; close finished items ----
    if (active && status < 0 && accepted) {
      if constexpr (REQ) {
        if (landed) {
          // torque |dj/dt| at the sample from f(y_new) (the potential depends on q only,
          // so the rescale below leaves it unchanged)
          double a[3];
          if constexpr (Sys::SOLO) {
#pragma unroll
            for (int i = 0; i < 3; ++i) a[i] = double(__shfl_sync(FULL, K[12][0], Sys::MOM2 + i));
          } else {
#pragma unroll
            for (int i = 0; i < 3; ++i) a[i] = double(K[12][Sys::MOM2 + i]);
          }
          const double tq = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
          if (req & 1) {
            // requantization with the switch of the previous sample, then the stages
            // restart from the new state (CVodeReInit in make_step)
            if constexpr (Sys::SOLO) {
              double j[3];
#pragma unroll
              for (int i = 0; i < 3; ++i) j[i] = __shfl_sync(FULL, y_new[0], Sys::MOM2 + i);
              req_rescale(P.req_mode, j[0], j[1], j[2]);
#pragma unroll
              for (int i = 0; i < 3; ++i)
                if (comp == Sys::MOM2 + i) y_new[0] = j[i];
              double yn[N];
              STG f[N];
#pragma unroll
              for (int i = 0; i < N; ++i) yn[i] = __shfl_sync(FULL, y_new[0], i);
              sys.rhs(yn, f);
              K[12][0] = pick_component<N>(f, comp);
            } else {
              req_rescale(P.req_mode, y_new[Sys::MOM2], y_new[Sys::MOM2 + 1], y_new[Sys::MOM2 + 2]);
              sys.rhs(y_new, K[12]);
            }
            nrhs += 1;
          }
          int le = (req >> 1) & 0x7fff, ge = (req >> 16) & 0x7fff;
          le = tq <= P.req_limit ? min(le + 1, req_cap) : 0;
          ge = tq >= P.req_limit ? min(ge + 1, req_cap) : 0;
          int on = req & 1;
          if (le >= P.req_len) on = 1;
          else if (ge >= P.req_len) on = 0;
          req = on | (le << 1) | (ge << 16);
        }
        t = landed ? t_land : t + h_taken;
      } else {
        t += h_taken;
      }
#pragma unroll
      for (int i = 0; i < NL; ++i) {
        y[i] = y_new[i];
        K[0][i] = K[12][i];  // FSAL
      }
      if (k >= P.N) status = HH_ST_OK;
      else if (++since > P.max_steps || ++total > P.max_total_steps) status = HH_ST_MAXSTEPS;
    }
    if constexpr (!Sys::SOLO) {
      if (io.done) {
        const unsigned closing = __ballot_sync(FULL, active && status >= 0);
        if (lane == 0 && closing) atomicAdd(io.done, (unsigned)__popc(closing));
      }
    }
    if (Sys::RECORDS && active && status >= 0) {
      if (owner) {
        io.rec_len[item] = k - 1;
        io.rec_status[item] = status;
        if (io.item_trace) {
          const unsigned long long t_end = globaltimer_ns();
          io.item_trace[item] = make_uint4(nsteps - s0, nsamp - m0, (unsigned)(t_begin & 0xffffffffu),
                                           (unsigned)(t_end & 0xffffffffu));
        }
      }
      ++nitems;
      item = -1;
    }
    if (!Sys::RECORDS && active && status >= 0 && !owner) item = -1;
    if (!Sys::RECORDS && active && status >= 0 && owner) {
      const int traj = item >> 1;
      // the t = 0 term is added by branches that are not dropped, so a replay
      // with the opposite weight removes exactly what a dropped trajectory added
      if (io.series) {
        io.rec_len[item] = k - 1;
        if (io.rec_status) io.rec_status[item] = status | (exited ? 16 : 0);
      }
      if (defer) {
        // the sample kernels add the t = 0 term and count the status
        io.item_status[item] = status;
      } else if (!hard && !io.series) {
        const PHYS c0 = mu0[0] * mu0[0] + mu0[1] * mu0[1] + mu0[2] * mu0[2];
        if (io.n_sat == 0) {
          atomicAdd(&crln[0], P.weight * double(c0));
        } else {
          for (int s = 0; s < io.n_sat; ++s)
            atomicAdd(&crln[(size_t)s * P.N], P.weight * satw[s] * double(c0));
        }
      }
      if (io.item_trace) {
        const unsigned long long t_end = globaltimer_ns();
        io.item_trace[item] = make_uint4(nsteps - s0, nsamp - m0, (unsigned)(t_begin & 0xffffffffu),
                                         (unsigned)(t_end & 0xffffffffu));
      }
      if (!defer) atomicAdd(&io.status_hist[status], 1u);
      ++nitems;
      if (hard && io.fail_flag) {
        if (atomicExch(&io.fail_flag[traj], 1) == 0) {
          const int slot = atomicAdd(io.fail_count, 1);
          io.fail_list[slot] = traj;
        }
      }
      item = -1;
    }
  }
  if (!owner) nsteps = nrej = nrhs = ndense = nitems = 0;  // solo mode: counted once per item
  warp_add_counter(&io.counters[0], nsteps);
  warp_add_counter(&io.counters[1], nrej);
  warp_add_counter(&io.counters[2], nrhs);
  warp_add_counter(&io.counters[3], nsamp);
  warp_add_counter(&io.counters[4], ndense);
  warp_add_counter(&io.counters[5], nitems);
}

template <typename PHYS> __host__ __device__ constexpr size_t smem_tables_bytes() {
  return (sizeof(Co2arTables<PHYS>) + 15) / 16 * 16;
}

// block-wide copy of `bytes` (a multiple of 8) from global to shared memory
__device__ __forceinline__ void load_words(void *dst, const void *src, size_t bytes) {
  const double *s = static_cast<const double *>(src);
  double *d = static_cast<double *>(dst);
  for (size_t i = threadIdx.x; i < bytes / 8; i += blockDim.x) d[i] = s[i];
}

// block shape of traj_kernel.  Both precision paths use every register (255), so
// 8 warps run per SM whatever the block shape; 4 and 8 warps per block differ in
// the copies of the surface tables per SM and in how blocks drain at the end of a
// launch.  The bulk kernel is compiled for both (TRAJ_WARPS_CANDIDATES) and the
// library times them on the first large call per system and precision (the
// autotuner in hh_api.cu); traj_warps is the default before that and the block
// shape of the solo kernel.  TRAJ_MIN_BLOCKS is the blocks per SM the register
// allocation must allow.
template <typename PHYS> constexpr int traj_warps() { return sizeof(PHYS) == 8 ? 8 : 4; }
template <typename PHYS> constexpr int traj_threads() { return 32 * traj_warps<PHYS>(); }
constexpr int TRAJ_WARPS_CANDIDATES[2] = {4, 8};
constexpr int TRAJ_MIN_BLOCKS = 1;

// dynamic shared memory of traj_kernel: coefficient tables (CO2-Ar) + one pool per warp
template <int SYS, typename PHYS, typename STG, int WARPS = traj_warps<PHYS>()>
constexpr size_t traj_smem_bytes() {
  return (SYS == SYS_CO2AR   ? smem_tables_bytes<PHYS>()
          : SYS == SYS_N2AR ? sizeof(N2arDipFold) + sizeof(N2arPesNet<PHYS>)
                            : 0) +
         WARPS * sizeof(WarpSamples<STG, PHYS, (SYS == SYS_HEAR ? 3 : SYS == SYS_CH4CO2 ? 10 : 6)>);
}

// SOLO: one item per warp (the solo kernel of the hand-off); WARPS: warps per block
// REQ: PR_MU requantization compiled in (linear-molecule systems only)
template <int SYS, typename PHYS, typename STG, bool COMP, bool SOLO = false, int WARPS = traj_warps<PHYS>(),
          bool REQ = false>
__global__ void __launch_bounds__(32 * WARPS, TRAJ_MIN_BLOCKS)
    traj_kernel(TrajParams P, TrajIO io, const Co2arTablesGlobal *gtab) {
  static_assert(!REQ || SYS == SYS_CO2AR || SYS == SYS_N2AR, "requantization of a linear monomer");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if constexpr (SYS == SYS_HEAR) {
    using Sys = HeArSys<PHYS, STG, COMP, SOLO>;
    Sys sys;
    sys.inv_mu = 1.0 / P.mu;
    auto *ws = reinterpret_cast<WarpSamples<STG, PHYS, Sys::NQ> *>(smem_raw);
    traj_body<Sys, PHYS, STG>(sys, P, io, ws);
  } else if constexpr (SYS == SYS_CH4CO2) {
    using Sys = Ch4Co2Sys<PHYS, STG, COMP, SOLO>;
    Sys sys;
    sys.inv_mu = 1.0 / P.mu;
    sys.inv_II = 1.0 / P.II;
#pragma unroll
    for (int k = 0; k < 3; ++k) sys.inv_I1[k] = io.inv_I1[k];
    sys.lj = io.lj;
    auto *ws = reinterpret_cast<WarpSamples<STG, PHYS, Sys::NQ> *>(smem_raw);
    traj_body<Sys, PHYS, STG>(sys, P, io, ws);
  } else if constexpr (SYS == SYS_N2AR) {
    using Sys = N2ArSys<PHYS, STG, COMP, SOLO>;
    Sys sys;
    sys.inv_mu = 1.0 / P.mu;
    sys.inv_II = 1.0 / P.II;
    N2arDipFold *fold = reinterpret_cast<N2arDipFold *>(smem_raw);
    N2arPesNet<PHYS> *pes = reinterpret_cast<N2arPesNet<PHYS> *>(smem_raw + sizeof(N2arDipFold));
    load_words(fold, io.dipnet, sizeof(N2arDipFold));
    load_words(pes, io.pesnet, sizeof(N2arPesNet<PHYS>));
    __syncthreads();
    sys.fold = fold;
    sys.pes = pes;
    sys.dtab = static_cast<const float4 *>(io.diptab);
    auto *ws = reinterpret_cast<WarpSamples<STG, PHYS, Sys::NQ> *>(smem_raw + sizeof(N2arDipFold) +
                                                                   sizeof(N2arPesNet<PHYS>));
    traj_body<Sys, PHYS, STG, REQ>(sys, P, io, ws);
  } else {
    using Sys = Co2ArSys<PHYS, STG, COMP, SOLO>;
    Co2arTables<PHYS> *tb = reinterpret_cast<Co2arTables<PHYS> *>(smem_raw);
    load_tables<PHYS>(tb, gtab);
    __syncthreads();
    Sys sys;
    sys.inv_mu = 1.0 / P.mu;
    sys.inv_II = 1.0 / P.II;
    sys.tb = tb;
    auto *ws = reinterpret_cast<WarpSamples<STG, PHYS, Sys::NQ> *>(smem_raw + smem_tables_bytes<PHYS>());
    traj_body<Sys, PHYS, STG, REQ>(sys, P, io, ws);
  }
}


// Item starts of a launch's items (io.items or 0 .. n_items - 1), one thread per item:
// item_setup as the trajectory kernel would run it at the item's refill (the same
// out-of-line function of the same system type, so the values are bit-identical).
// CO2-Ar (surface tables in shared memory), N2-Ar (the networks in shared memory) and
// CH4-CO2.
template <int SYS, typename PHYS, typename STG>
__global__ void __launch_bounds__(256) item_start_kernel(TrajParams P, TrajIO io, const Co2arTablesGlobal *gtab,
                                                        void *out) {
  static_assert(SYS == SYS_CO2AR || SYS == SYS_N2AR || SYS == SYS_CH4CO2, "item starts of a linear or rotor system");
  using Sys = typename std::conditional<
      SYS == SYS_CO2AR, Co2ArSys<PHYS, STG, false, false>,
      typename std::conditional<SYS == SYS_N2AR, N2ArSys<PHYS, STG, false, false>,
                                Ch4Co2Sys<PHYS, STG, false, false>>::type>::type;
  extern __shared__ __align__(16) unsigned char is_smem[];
  Sys sys;
  sys.inv_mu = 1.0 / P.mu;
  sys.inv_II = 1.0 / P.II;
  if constexpr (SYS == SYS_CO2AR) {
    Co2arTables<PHYS> *tb = reinterpret_cast<Co2arTables<PHYS> *>(is_smem);
    load_tables<PHYS>(tb, gtab);
    __syncthreads();
    sys.tb = tb;
  } else if constexpr (SYS == SYS_N2AR) {
    N2arDipFold *fold = reinterpret_cast<N2arDipFold *>(is_smem);
    N2arPesNet<PHYS> *pes = reinterpret_cast<N2arPesNet<PHYS> *>(is_smem + sizeof(N2arDipFold));
    load_words(fold, io.dipnet, sizeof(N2arDipFold));
    load_words(pes, io.pesnet, sizeof(N2arPesNet<PHYS>));
    __syncthreads();
    sys.fold = fold;
    sys.pes = pes;
    sys.dtab = static_cast<const float4 *>(io.diptab);
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) sys.inv_I1[k] = io.inv_I1[k];
    sys.lj = io.lj;
  }
  auto *o = static_cast<ItemStart<Sys::N, PHYS, STG> *>(out);
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < io.n_items; idx += gridDim.x * blockDim.x) {
    const int item = io.items ? io.items[idx] : idx;
    double y[Sys::N], h;
    STG f[Sys::N];
    PHYS mu[3];
    item_setup<Sys, PHYS, STG>(sys, P, io.ic + (size_t)(item >> 1) * Sys::QP, item & 1, y, f, mu, &h);
    ItemStart<Sys::N, PHYS, STG> &st = o[item];
#pragma unroll
    for (int i = 0; i < Sys::N; ++i) {
      st.y0[i] = y[i];
      st.f0[i] = f[i];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) st.mu0[c] = mu[c];
    st.h = h;
  }
}

}  // namespace hh
