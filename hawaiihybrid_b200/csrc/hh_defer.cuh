// Deferred sample evaluation of the plain C(t) path.
//
// The trajectory kernel runs at 8 warps per SM (its stage arrays fill the register
// file), which leaves the dipole evaluation at the sample times latency-bound: a
// dense-output step of a free-flight segment stores dozens of samples, each an
// interpolation plus a surface evaluation of a few hundred dependent instructions.
// With io.ctx set the kernel interpolates only r (for the reference's R > Rcut exit,
// src/hawaii.c:2244) and writes one SampleCtx per dense-output step; the kernels here
// then run the per-sample work at full occupancy:
//   defer_eval_co2ar_kernel (CO2-Ar) and defer_eval_kernel (N2-Ar)
//                       pooled (context, sample) pairs, 32 lanes per warp round (two
//                       samples per lane for CO2-Ar): y(t_k) from the context, the
//                       dipole, mu0 . mu(t_k) into C(t_k), and the reference's
//                       per-sample tests (src/hawaii.c:2183-2243: NaN dipole, |value| >
//                       1e100, |value / previous| > 1e10 for k > 1) within the context,
//                       and the failure-injection hook of the in-kernel path (hard
//                       statuses only); the first failure per item is kept as
//                       (k << 3) | reason with atomicMin;
//   defer_jump_kernel   the jump test across contexts (first sample of a context
//                       against the last of the item's previous context);
//   defer_items_kernel  per item: the status (a sample failure, else the integration's),
//                       the t = 0 term |mu0|^2 of items that did not fail, and the
//                       list of failed trajectories.
// A failed trajectory is replayed with the opposite weight by the host, which
// removes everything it added; the replay takes the same path, so its samples are
// exactly those the first pass accumulated.  Samples after a failure are therefore
// accumulated too (only NaN and infinite values are skipped, in both passes), which
// leaves C(t) as the in-kernel path makes it: failed trajectories contribute nothing.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hh_traj.cuh"

namespace hh {

constexpr int DEFER_THREADS = 256;
// block size of the sample kernels: CO2-Ar in blocks of two warps, which fit into the
// registers that finished solo-kernel warps release while the solo kernel still runs
template <int SYS> constexpr int defer_eval_threads() { return SYS == SYS_CO2AR ? 64 : DEFER_THREADS; }
// words of the context counter block: the count the trajectory kernels advance, the
// largest count of a call, and the snapshot of the count after the bulk kernel
constexpr int DEFER_COUNT = 0, DEFER_PEAK = 1, DEFER_SNAP = 2, DEFER_WORDS = 3;

struct DeferArgs {
  const void *ctx;                      // SampleCtx<STG, NQ>[ctx_cap]
  const unsigned long long *ctx_count;  // contexts written (may exceed ctx_cap)
  unsigned long long ctx_cap;
  // the sample launch's contexts: [*ctx_lo, *ctx_hi), nullptr standing for 0 and
  // *ctx_count; warp w of the grid takes the groups of 32 that start at
  // lo + 32 (w + r W), W warps in the grid (a shared cursor, which balances the end
  // of a launch better, ran 10 to 30 % slower at a launch of 10^8 contexts)
  const unsigned long long *ctx_lo, *ctx_hi;
  const int *items;                     // defer_items_kernel: explicit item list or nullptr
  int n_items;
  const int *item_status;               // [item]
  const void *item_mu0;                 // [item][4] PHYS: mu0, |mu0|^2
  unsigned *item_fail;                  // [item] (k << 3) | reason of the first failure, ~0u none
  void *first_v, *last_v;               // [ctx] PHYS: the context's first and last sample value
  double *crln;                         // C(t) slices, traj_per_iter trajectories each
  long long traj_per_iter;
  double inv_traj_per_iter;             // 1 / traj_per_iter
  unsigned int *status_hist;
  int *fail_flag, *fail_list, *fail_count;  // fail_flag == nullptr: replay pass
  long long traj_base;                  // the launch's first trajectory in the call (fail list)
  unsigned long long *peak;             // largest context count of the call's launches
};

__device__ __forceinline__ unsigned long long defer_count(const DeferArgs &a) {
  const unsigned long long c = *a.ctx_count;
  return c < a.ctx_cap ? c : a.ctx_cap;
}
__device__ __forceinline__ unsigned long long defer_hi(const DeferArgs &a) {
  const unsigned long long c = a.ctx_hi ? *a.ctx_hi : *a.ctx_count;
  return c < a.ctx_cap ? c : a.ctx_cap;
}
__device__ __forceinline__ unsigned long long defer_lo(const DeferArgs &a) {
  const unsigned long long c = a.ctx_lo ? *a.ctx_lo : 0ull;
  return c < a.ctx_cap ? c : a.ctx_cap;
}
// After the bulk trajectory kernel: the count of the contexts it wrote (all complete
// at the kernel boundary).
__global__ void defer_snapshot_kernel(unsigned long long *counts) { counts[DEFER_SNAP] = counts[DEFER_COUNT]; }

// the dipole of the bound system with its surfaces staged in shared memory
template <int SYS, typename PHYS, typename STG> struct DeferSys;

// CO2-Ar dipole surface for the sample kernel.  The z and x rows of one (interval, l)
// are interleaved so that each radial coefficient is a (z, x) pair: 16 FP32 words,
// (a0 a1 | a2 a3 | b4 b5 | b6 b7) as pairs, four 16-byte loads at most.  The dipole
// intervals carry no exponential terms (the library checks this when it builds the
// tables and keeps CO2-Ar samples in the trajectory kernel otherwise).  The interval
// is found by one lookup of floor(4 R) (every interval bound is a multiple of 1/4
// bohr, so the lookup gives the reference's `R < bound` interval exactly).  The sums
// are those of co2ar_dip (l = 0, 2, .., 10 in order).
struct DeferCo2arDip {
  float4 row[CO2AR_NINT][CO2AR_NL][4];  // [interval][l / 2][16 words]
  float rlo[CO2AR_NINT];
  int fdip[CO2AR_NINT];
  unsigned char ivl[164];               // interval of R in [j / 4, (j + 1) / 4), j <= 160
};
template <typename PHYS, typename STG> struct DeferSys<SYS_CO2AR, PHYS, STG> {
  static constexpr int NQ = 6;
  static constexpr size_t smem() { return (sizeof(DeferCo2arDip) + 15) / 16 * 16; }
  const DeferCo2arDip *t;
  __device__ void init(unsigned char *sm, const Co2arTablesGlobal *g, const TrajIO &) {
    auto *d = reinterpret_cast<DeferCo2arDip *>(sm);
    float *w = reinterpret_cast<float *>(d->row);
    constexpr int NW = CO2AR_NINT * CO2AR_NL * 16;
    for (int e = threadIdx.x; e < NW; e += blockDim.x) {
      // word k: coefficient k / 2 of the z (even k) or x (odd k) row
      const int k = e % 16, li = (e / 16) % CO2AR_NL, i = e / (16 * CO2AR_NL);
      const double *src = ((k & 1) ? g->dipx : g->dipz) + (i * CO2AR_NL + li) * CO2AR_ROW;
      w[e] = float(src[k >> 1]);
    }
    for (int i = threadIdx.x; i < CO2AR_NINT; i += blockDim.x) {
      d->rlo[i] = float(g->rlo[i]);
      d->fdip[i] = g->fdip[i];
    }
    for (int j = threadIdx.x; j < 164; j += blockDim.x) {
      const double r = 0.25 * j;
      int i = 0;
      while (i < CO2AR_NINT - 1 && !(r < g->rbound[i])) ++i;
      d->ivl[j] = (unsigned char)i;
    }
    t = d;
  }
  // the (z, x) radial functions of one l: the cubic in tt = R - R_lo, then the
  // inverse powers where the interval has them
  __device__ __forceinline__ float2 radial2(const float4 *rw, float2 tt, float2 i4, float2 i5, float2 i6,
                                            float2 i7, int fl) const {
    const float4 a = rw[0], b = rw[1];
    float2 c = fma2(make_float2(b.z, b.w), tt, make_float2(b.x, b.y));
    c = fma2(c, tt, make_float2(a.z, a.w));
    c = fma2(c, tt, make_float2(a.x, a.y));
    if (fl & 1) {
      const float4 p = rw[2], q = rw[3];
      c = fma2(make_float2(p.x, p.y), i4, c);
      c = fma2(make_float2(p.z, p.w), i5, c);
      c = fma2(make_float2(q.x, q.y), i6, c);
      c = fma2(make_float2(q.z, q.w), i7, c);
    }
    return c;
  }
  // sum_l P_l(x) z_l(R) and sum_l P_l'(x) x_l(R) of one sample
  __device__ __forceinline__ void sums(float R, float iR, const float2 (&P)[11], const float2 (&dP)[11], bool second,
                                       float &dz, float &ax) const {
    const int i = t->ivl[min(int(R * 4.f), 163)];
    const float2 tt = splat2(R - t->rlo[i]);
    const int fl = t->fdip[i];
    const float iR2 = iR * iR, iR4 = iR2 * iR2, iR5 = iR4 * iR, iR6 = iR5 * iR, iR7 = iR6 * iR;
    const float2 i4 = splat2(iR4), i5 = splat2(iR5), i6 = splat2(iR6), i7 = splat2(iR7);
    dz = 0.f;
    ax = 0.f;
#pragma unroll
    for (int li = 0; li < CO2AR_NL; ++li) {
      const float2 c = radial2(t->row[i][li], tt, i4, i5, i6, i7, fl);
      const float p = second ? P[2 * li].y : P[2 * li].x, dp = second ? dP[2 * li].y : dP[2 * li].x;
      dz = fmaf(p, c.x, dz);
      ax = fmaf(dp, c.y, ax);
    }
  }
  // the dipoles of two samples, positions q[c] = (first, second)
  __device__ __forceinline__ void dipole2(const float2 (&q)[6], float2 (&d)[3]) const {
    const float2 R2 = fma2(q[2], q[2], fma2(q[1], q[1], mul2(q[0], q[0])));
    const float2 U2 = fma2(q[5], q[5], fma2(q[4], q[4], mul2(q[3], q[3])));
    const float2 iR = make_float2(rsqrtf(R2.x), rsqrtf(R2.y));
    const float2 iu = make_float2(rsqrtf(U2.x), rsqrtf(U2.y));
    float2 rh[3], uh[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      rh[c] = mul2(q[c], iR);
      uh[c] = mul2(q[3 + c], iu);
    }
    const float2 x = fma2(rh[2], uh[2], fma2(rh[1], uh[1], mul2(rh[0], uh[0])));
    const float2 R = mul2(R2, iR);
    // Legendre P_l and P_l' of both samples: (l + 1) P_{l+1} = (2l + 1) x P_l - l P_{l-1},
    // P_{l+1}' = P_{l-1}' + (2l + 1) P_l
    float2 P[11], dP[11];
    P[0] = splat2(1.f);
    P[1] = x;
    dP[0] = splat2(0.f);
    dP[1] = splat2(1.f);
#pragma unroll
    for (int l = 1; l < 10; ++l) {
      const float2 ax = mul2(splat2(float(2 * l + 1)), x);
      P[l + 1] = mul2(fma2(ax, P[l], mul2(splat2(-float(l)), P[l - 1])), splat2(float(1.0 / double(l + 1))));
      dP[l + 1] = fma2(splat2(float(2 * l + 1)), P[l], dP[l - 1]);
    }
    float dzA, axA, dzB, axB;
    sums(R.x, iR.x, P, dP, false, dzA, axA);
    sums(R.y, iR.y, P, dP, true, dzB, axB);
    const float2 dz = make_float2(dzA, dzB);
    const float2 nax = make_float2(-axA, -axB), nx = make_float2(-x.x, -x.y);
    // dz r^ - ax (u^ - x r^)
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = fma2(nax, fma2(nx, rh[c], uh[c]), mul2(dz, rh[c]));
  }
};
template <typename PHYS, typename STG> struct DeferSys<SYS_N2AR, PHYS, STG> {
  static constexpr int NQ = 6;
  static constexpr size_t smem() { return sizeof(N2arDipFold); }
  N2ArSys<PHYS, STG, false, false> sys;
  __device__ void init(unsigned char *sm, const Co2arTablesGlobal *, const TrajIO &io) {
    auto *fold = reinterpret_cast<N2arDipFold *>(sm);
    load_words(fold, io.dipnet, sizeof(N2arDipFold));
    sys.fold = fold;
    sys.pes = nullptr;
    sys.dtab = static_cast<const float4 *>(io.diptab);
  }
  static constexpr bool FLOAT_Q = false;
  __device__ __forceinline__ void dipole(const double *q, PHYS d[3]) const { sys.dipole(q, d); }
};

// The C(t) slice of an item: its trajectory's iteration, (item / 2) / traj_per_iter,
// from the reciprocal (off by one at most for counts below 2^31) and corrected.
__device__ __forceinline__ double *crln_slice(const DeferArgs &a, const TrajParams &P, int item) {
  const long long t = item >> 1;
  long long q = (long long)(double(t) * a.inv_traj_per_iter);
  const long long r = t - q * a.traj_per_iter;
  if (r < 0) --q;
  else if (r >= a.traj_per_iter) ++q;
  return a.crln + (size_t)q * (size_t)P.N;
}

// The reference's tests of one sample value (src/hawaii.c:2183-2243) on an FP32 value:
// a NaN dipole; the failure-injection hook; |v| > 1e100, which is v = +-inf in FP32;
// and |v / pv| > 1e10 against the previous sample of the same context (for k > 1),
// as |v| > 1e10 |pv| (1e10 is exact in FP32; a zero pv fails any v != 0, NaN fails
// neither).  (k << 3) | reason, or ~0u.
__device__ __forceinline__ unsigned sample_code(float v, bool nan, int kk, bool inject, bool jump, float pv) {
  if (nan) return (unsigned(kk) << 3) | 1u;
  if (inject) return (unsigned(kk) << 3) | 4u;
  if (isinf(v)) return (unsigned(kk) << 3) | 2u;
  if (jump && fabsf(v) > 1e10f * fabsf(pv)) return (unsigned(kk) << 3) | 3u;
  return 0xffffffffu;
}

// the context in 16-byte loads: qold, (t0, inv_h), (item, k0, n, prev), F
template <int NQ>
__device__ __forceinline__ void load_ctx(const SampleCtx<float, NQ> *cp, double (&qo)[NQ], double2 &th, int4 &hd,
                                         float (&F)[7 * NQ]) {
#pragma unroll
  for (int i = 0; i < NQ / 2; ++i) {
    const double2 v2 = reinterpret_cast<const double2 *>(cp->qold)[i];
    qo[2 * i] = v2.x;
    qo[2 * i + 1] = v2.y;
  }
  th = *reinterpret_cast<const double2 *>(&cp->t0);
  hd = *reinterpret_cast<const int4 *>(&cp->item);
#pragma unroll
  for (int i = 0; i < 7 * NQ / 4; ++i) {
    const float4 v4 = reinterpret_cast<const float4 *>(&cp->F[0][0])[i];
    F[4 * i] = v4.x;
    F[4 * i + 1] = v4.y;
    F[4 * i + 2] = v4.z;
    F[4 * i + 3] = v4.w;
  }
#pragma unroll
  for (int i = 4 * (7 * NQ / 4); i < 7 * NQ; ++i) F[i] = (&cp->F[0][0])[i];
}

// The warp's 32 contexts (base + lane) and the exclusive prefix sum of `units`
// (samples, or pairs of samples) over the lanes; returns the warp's total.
__device__ __forceinline__ int warp_prefix(int units, int lane, int &off) {
  int incl = units;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  off = incl - units;
  return __shfl_sync(0xffffffffu, incl, 31);
}

// The lane that owns unit j of the round: the largest lane whose offset is <= j.
__device__ __forceinline__ int warp_owner(int off, int j) {
  int o = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1) {
    const int oc = __shfl_sync(0xffffffffu, off, o + step);
    if (oc <= j) o += step;
  }
  return o;
}

// N2-Ar: one sample per lane, the position in FP64 as the trajectory kernel forms it.
template <int SYS, typename PHYS, typename STG>
__global__ void __launch_bounds__(DEFER_THREADS, 1) defer_eval_kernel(DeferArgs a, TrajParams P, TrajIO io,
                                                                      const Co2arTablesGlobal *gtab) {
  using DS = DeferSys<SYS, PHYS, STG>;
  constexpr int NQ = DS::NQ;
  using Ctx = SampleCtx<STG, NQ>;
  static_assert(SYS == SYS_N2AR, "CO2-Ar samples go through defer_eval_co2ar_kernel");
  static_assert(sizeof(STG) == 4 && sizeof(PHYS) == 4 && NQ % 2 == 0 && sizeof(Ctx) % 16 == 0, "vector loads of the context");
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char df_smem[];
  DS ds;
  ds.init(df_smem, gtab, io);
  __syncthreads();
  const unsigned long long lo = defer_lo(a), count = defer_hi(a);
  const Ctx *ctx = static_cast<const Ctx *>(a.ctx);
  const PHYS *mu0s = static_cast<const PHYS *>(a.item_mu0);
  PHYS *first_v = static_cast<PHYS *>(a.first_v);
  PHYS *last_v = static_cast<PHYS *>(a.last_v);
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long base = lo + gw * 32; base < count; base += nw * 32) {
    const unsigned long long ci = base + lane;
    const int n = ci < count ? ctx[ci].n : 0;
    int off;
    const int total = warp_prefix(n, lane, off);
    PHYS tail = PHYS(0);  // the last sample of the previous round
    for (int j0 = 0; j0 < total; j0 += 32) {
      const int j = j0 + lane;
      const int o = warp_owner(off, j);
      const int jj = j - __shfl_sync(FULL, off, o);
      const bool valid = j < total;
      PHYS v = PHYS(0);
      bool nan = false;
      int kk = 0, item = 0, nn = 0;
      if (valid) {
        double qo[NQ];
        double2 th;
        int4 hd;
        STG F[7 * NQ];
        load_ctx<NQ>(ctx + base + o, qo, th, hd, F);
        item = hd.x;
        nn = hd.z;
        kk = hd.y + jj;
        const double x = (double(kk) * P.dt - th.x) * th.y;
        const STG xs = STG(x), x1 = STG(1) - STG(x);
        PHYS d[3];
        // the trajectory kernel's interpolation (hh_traj.cuh) in its order
        double q[NQ];
#pragma unroll
        for (int cq = 0; cq < NQ; ++cq) {
          STG w = F[6 * NQ + cq] * xs;
          w = (w + F[5 * NQ + cq]) * x1;
          w = (w + F[4 * NQ + cq]) * xs;
          w = (w + F[3 * NQ + cq]) * x1;
          w = (w + F[2 * NQ + cq]) * xs;
          w = (w + F[1 * NQ + cq]) * x1;
          w = (w + F[0 * NQ + cq]) * xs;
          q[cq] = qo[cq] + double(w);
        }
        ds.dipole(q, d);
        nan = isnan(d[0]) || isnan(d[1]) || isnan(d[2]);
        const float4 m = *reinterpret_cast<const float4 *>(mu0s + (size_t)item * 4);
        v = m.x * d[0] + m.y * d[1] + m.z * d[2];
      }
      // the previous sample of the same context: lane - 1, or the last of the
      // previous round (jj == 0 is the cross-context case of defer_jump_kernel)
      PHYS pv = __shfl_up_sync(FULL, v, 1);
      if (lane == 0) pv = tail;
      tail = __shfl_sync(FULL, v, 31);
      if (valid) {
        const unsigned code =
            sample_code(v, nan, kk, item + 2 * a.traj_base == P.inject_item && kk == P.inject_k, jj > 0 && kk > 1, pv);
        if (code != 0xffffffffu) atomicMin(&a.item_fail[item], code);
        if (!isnan(v) && !isinf(v)) atomicAdd(&crln_slice(a, P, item)[kk], P.weight * double(v));
        if (jj == 0) first_v[base + o] = v;
        if (jj == nn - 1) last_v[base + o] = v;
      }
    }
  }
}

// CO2-Ar: two consecutive samples of one context per lane.  The pair shares the
// context loads, the owner search and the set-up, and its arithmetic runs on
// (first, second) float2 pairs: the dense-output interpolation and the dipole
// (paired FP32, fma2).  The position is formed in FP32, y_old + F0 x + F1 x(1-x) +
// F2 x^2(1-x) + ... + F6 x^4(1-x)^3 with the basis formed once and one FMA per term.
// A context with an odd count ends in a single sample: the second half of its last
// pair is computed but neither tested nor accumulated.  20 warps per SM (96 registers a
// thread, no spills) ran faster than 16 (128) and than 24 or 32 (80 or 64, with spills).
template <typename PHYS, typename STG>
__global__ void __launch_bounds__(defer_eval_threads<SYS_CO2AR>(), 20 * 32 / defer_eval_threads<SYS_CO2AR>())
    defer_eval_co2ar_kernel(DeferArgs a, TrajParams P, TrajIO io, const Co2arTablesGlobal *gtab) {
  using DS = DeferSys<SYS_CO2AR, float, float>;
  constexpr int NQ = DS::NQ;
  using Ctx = SampleCtx<float, NQ>;
  static_assert(sizeof(STG) == 4 && sizeof(PHYS) == 4 && sizeof(Ctx) % 16 == 0, "vector loads of the context");
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char df_smem[];
  DS ds;
  ds.init(df_smem, gtab, io);
  __syncthreads();
  const unsigned long long lo = defer_lo(a), count = defer_hi(a);
  const Ctx *ctx = static_cast<const Ctx *>(a.ctx);
  const float *mu0s = static_cast<const float *>(a.item_mu0);
  float *first_v = static_cast<float *>(a.first_v);
  float *last_v = static_cast<float *>(a.last_v);
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long base = lo + gw * 32; base < count; base += nw * 32) {
    const unsigned long long ci = base + lane;
    const int n = ci < count ? ctx[ci].n : 0;
    int off;
    const int total = warp_prefix((n + 1) >> 1, lane, off);  // pairs
    float tail = 0.f;  // the last sample of the previous round
    for (int u0 = 0; u0 < total; u0 += 32) {
      const int u = u0 + lane;
      const int o = warp_owner(off, u);
      const int jj = 2 * (u - __shfl_sync(FULL, off, o));  // the pair's first sample in its context
      const bool valid = u < total;
      float vA = 0.f, vB = 0.f;
      bool nanA = false, nanB = false, two = false;
      int kk = 0, item = 0, nn = 0;
      if (valid) {
        double qo[NQ];
        double2 th;
        int4 hd;
        float F[7 * NQ];
        load_ctx<NQ>(ctx + base + o, qo, th, hd, F);
        item = hd.x;
        nn = hd.z;
        kk = hd.y + jj;
        two = jj + 1 < nn;
        const double xa = (double(kk) * P.dt - th.x) * th.y;
        const double xb = (double(kk + 1) * P.dt - th.x) * th.y;
        const float2 xs = make_float2(float(xa), float(xb));
        const float2 x1 = make_float2(1.f - xs.x, 1.f - xs.y);
        float2 bs[7];
        bs[0] = xs;
        bs[1] = mul2(xs, x1);
        bs[2] = mul2(bs[1], xs);
        bs[3] = mul2(bs[2], x1);
        bs[4] = mul2(bs[3], xs);
        bs[5] = mul2(bs[4], x1);
        bs[6] = mul2(bs[5], xs);
        float2 q[NQ];
#pragma unroll
        for (int c = 0; c < NQ; ++c) {
          float2 w = mul2(splat2(F[c]), bs[0]);
#pragma unroll
          for (int r = 1; r < 7; ++r) w = fma2(splat2(F[r * NQ + c]), bs[r], w);
          q[c] = add2(splat2(float(qo[c])), w);
        }
        float2 d[3];
        ds.dipole2(q, d);
        nanA = isnan(d[0].x) || isnan(d[1].x) || isnan(d[2].x);
        nanB = isnan(d[0].y) || isnan(d[1].y) || isnan(d[2].y);
        const float4 m = *reinterpret_cast<const float4 *>(mu0s + (size_t)item * 4);
        const float2 v = fma2(splat2(m.z), d[2], fma2(splat2(m.y), d[1], mul2(splat2(m.x), d[0])));
        vA = v.x;
        vB = v.y;
      }
      // the previous sample of the first: the last of the previous pair (lane - 1, or
      // lane 31 of the previous round), which holds two samples whenever it is in the
      // same context (only a context's last pair can be single); jj == 0 is the
      // cross-context case of defer_jump_kernel.  The second's previous is the first.
      float pvA = __shfl_up_sync(FULL, vB, 1);
      if (lane == 0) pvA = tail;
      tail = __shfl_sync(FULL, vB, 31);
      if (valid) {
        const int inj = P.inject_item == item + 2 * a.traj_base ? P.inject_k : -1;
        unsigned code = sample_code(vA, nanA, kk, kk == inj, jj > 0 && kk > 1, pvA);
        if (two) code = min(code, sample_code(vB, nanB, kk + 1, kk + 1 == inj, kk + 1 > 1, vA));
        if (code != 0xffffffffu) atomicMin(&a.item_fail[item], code);
        double *crln = crln_slice(a, P, item);
        if (!isnan(vA) && !isinf(vA)) atomicAdd(&crln[kk], P.weight * double(vA));
        if (two && !isnan(vB) && !isinf(vB)) atomicAdd(&crln[kk + 1], P.weight * double(vB));
        if (jj == 0) first_v[base + o] = vA;
        if (jj + 1 >= nn - 1) last_v[base + o] = two ? vB : vA;
      }
    }
  }
}

template <typename PHYS, typename STG, int NQ>
__global__ void __launch_bounds__(DEFER_THREADS) defer_jump_kernel(DeferArgs a, TrajParams P) {
  using Ctx = SampleCtx<STG, NQ>;
  const unsigned long long count = defer_count(a);
  const Ctx *ctx = static_cast<const Ctx *>(a.ctx);
  const PHYS *first_v = static_cast<const PHYS *>(a.first_v);
  const PHYS *last_v = static_cast<const PHYS *>(a.last_v);
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const int4 hd = *reinterpret_cast<const int4 *>(&ctx[i].item);  // item, k0, n, prev
    const int prev = hd.w, k0 = hd.y, item = hd.x;
    if (prev < 0 || k0 <= 1) continue;
    if (item + 2 * a.traj_base == P.inject_item && k0 == P.inject_k) continue;  // the injected failure comes first
    const PHYS v = first_v[i], pv = last_v[prev];
    if (fabs(double(v)) > 1e10 * fabs(double(pv))) atomicMin(&a.item_fail[item], (unsigned(k0) << 3) | 3u);
  }
}

template <typename PHYS>
__global__ void __launch_bounds__(DEFER_THREADS) defer_items_kernel(DeferArgs a, TrajParams P) {
  const PHYS *mu0s = static_cast<const PHYS *>(a.item_mu0);
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(a.peak, *a.ctx_count);
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < a.n_items; idx += gridDim.x * blockDim.x) {
    const int item = a.items ? a.items[idx] : idx;
    const unsigned fc = a.item_fail[item];
    a.item_fail[item] = 0xffffffffu;  // clean for the next pass
    const bool hard = fc != 0xffffffffu;
    int status = a.item_status[item];
    if (hard) {
      const unsigned r = fc & 7u;
      status = r == 1u ? HH_ST_NAN_DIPOLE : r == 2u ? HH_ST_OVERFLOW : r == 3u ? HH_ST_JUMP : P.inject_status;
    }
    atomicAdd(&a.status_hist[status], 1u);
    const int traj = item >> 1;
    if (!hard) {
      double *crln = a.crln + (size_t)(traj / a.traj_per_iter) * (size_t)P.N;
      atomicAdd(&crln[0], P.weight * double(mu0s[(size_t)item * 4 + 3]));
    } else if (a.fail_flag) {
      if (atomicExch(&a.fail_flag[traj], 1) == 0) {
        const int slot = atomicAdd(a.fail_count, 1);
        a.fail_list[slot] = (int)(traj + a.traj_base);
      }
    }
  }
}

}  // namespace hh
