// Deferred sample evaluation of the plain C(t) path.
//
// The trajectory kernel runs at 8 warps per SM (its stage arrays fill the register
// file), which leaves the dipole evaluation at the sample times latency-bound: a
// dense-output step of a free-flight segment stores dozens of samples, each an
// interpolation plus a surface evaluation of a few hundred dependent instructions.
// With io.ctx set the kernel interpolates only r (for the reference's R > Rcut exit,
// src/hawaii.c:2244) and writes one SampleCtx per dense-output step; the kernels here
// then run the per-sample work at full occupancy:
//   defer_eval_kernel   pooled (context, sample) pairs, 32 per warp round: y(t_k) from
//                       the context, the dipole, mu0 . mu(t_k) into C(t_k), and the
//                       reference's per-sample tests (src/hawaii.c:2183-2243: NaN
//                       dipole, |value| > 1e100, |value / previous| > 1e10 for k > 1)
//                       within the context, and the failure-injection hook of the
//                       in-kernel path (hard statuses only); the first failure per item
//                       is kept as (k << 3) | reason with atomicMin;
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

struct DeferArgs {
  const void *ctx;                      // SampleCtx<STG, NQ>[ctx_cap]
  const unsigned long long *ctx_count;  // contexts written (may exceed ctx_cap)
  unsigned long long ctx_cap;
  const int *items;                     // defer_items_kernel: explicit item list or nullptr
  int n_items;
  const int *item_status;               // [item]
  const void *item_mu0;                 // [item][4] PHYS: mu0, |mu0|^2
  unsigned *item_fail;                  // [item] (k << 3) | reason of the first failure, ~0u none
  void *first_v, *last_v;               // [ctx] PHYS: the context's first and last sample value
  double *crln;                         // C(t) slices, traj_per_iter trajectories each
  long long traj_per_iter;
  unsigned int *status_hist;
  int *fail_flag, *fail_list, *fail_count;  // fail_flag == nullptr: replay pass
  long long traj_base;                  // the launch's first trajectory in the call (fail list)
  unsigned long long *peak;             // largest context count of the call's launches
};

__device__ __forceinline__ unsigned long long defer_count(const DeferArgs &a) {
  const unsigned long long c = *a.ctx_count;
  return c < a.ctx_cap ? c : a.ctx_cap;
}

// the dipole of the bound system with its surfaces staged in shared memory
template <int SYS, typename PHYS, typename STG> struct DeferSys;
// CO2-Ar dipole surface for the sample kernel: the rows of the x and z tables padded to
// 12 FP32 words (a0..a3 | b4..b7 | A k 0 0), three 16-byte loads each, and the
// interval found by one lookup of floor(4 R) (every interval bound is a multiple of
// 1/4 bohr, so the lookup gives the reference's `R < bound` interval exactly).  The
// sums are those of co2ar_dip (plain, l = 0, 2, .., 10 in order).
struct DeferCo2arDip {
  float4 row[CO2AR_NINT][2][CO2AR_NL][3];  // [interval][x, z][l / 2][12 words]
  float rlo[CO2AR_NINT];
  int fdip[CO2AR_NINT];
  unsigned char ivl[164];                  // interval of R in [j / 4, (j + 1) / 4), j <= 160
};
template <typename PHYS, typename STG> struct DeferSys<SYS_CO2AR, PHYS, STG> {
  static constexpr int NQ = 6;
  static constexpr size_t smem() { return (sizeof(DeferCo2arDip) + 15) / 16 * 16; }
  const DeferCo2arDip *t;
  __device__ void init(unsigned char *sm, const Co2arTablesGlobal *g, const TrajIO &) {
    auto *d = reinterpret_cast<DeferCo2arDip *>(sm);
    float *w = reinterpret_cast<float *>(d->row);
    constexpr int NW = CO2AR_NINT * 2 * CO2AR_NL * 12;
    for (int e = threadIdx.x; e < NW; e += blockDim.x) {
      const int k = e % 12, li = (e / 12) % CO2AR_NL, c = (e / (12 * CO2AR_NL)) % 2, i = e / (24 * CO2AR_NL);
      const double *src = (c == 0 ? g->dipx : g->dipz) + (i * CO2AR_NL + li) * CO2AR_ROW;
      w[e] = k < CO2AR_ROW ? float(src[k]) : 0.f;
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
  __device__ __forceinline__ float radial(const float4 *rw, float R, float tt, float iR4, float iR5, float iR6,
                                          float iR7, int fl) const {
    const float4 a = rw[0];
    float c = ((a.w * tt + a.z) * tt + a.y) * tt + a.x;
    if (fl & 1) {
      const float4 b = rw[1];
      c += b.x * iR4 + b.y * iR5 + b.z * iR6 + b.w * iR7;
    }
    if (fl & 2) {
      const float4 e = rw[2];
      c += e.x * expf(e.y * R);
    }
    return c;
  }
  static constexpr bool FLOAT_Q = true;  // takes the sample position in FP32
  __device__ __forceinline__ void dipole(const float *q, PHYS d[3]) const {
    const float r[3] = {q[0], q[1], q[2]};
    const float u[3] = {q[3], q[4], q[5]};
    const float R2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const float iR = rsqrtf(R2);
    const float iu = rsqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const float rh[3] = {r[0] * iR, r[1] * iR, r[2] * iR};
    const float uh[3] = {u[0] * iu, u[1] * iu, u[2] * iu};
    const float x = rh[0] * uh[0] + rh[1] * uh[1] + rh[2] * uh[2];
    const float R = R2 * iR;
    const int i = t->ivl[min(int(R * 4.f), 163)];
    const float tt = R - t->rlo[i];
    const int fl = t->fdip[i];
    float P[11], dP[11];
    legendre10(x, P, dP);
    const float iR2 = iR * iR, iR4 = iR2 * iR2, iR5 = iR4 * iR, iR6 = iR5 * iR, iR7 = iR6 * iR;
    float dz = 0.f, ax = 0.f;
#pragma unroll
    for (int li = 0; li < CO2AR_NL; ++li) {
      const float av = radial(t->row[i][0][li], R, tt, iR4, iR5, iR6, iR7, fl);
      const float bv = radial(t->row[i][1][li], R, tt, iR4, iR5, iR6, iR7, fl);
      dz += P[2 * li] * bv;
      ax += dP[2 * li] * av;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) d[c] = PHYS(dz * rh[c] - ax * (uh[c] - x * rh[c]));
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

template <int SYS, typename PHYS, typename STG>
__global__ void __launch_bounds__(DEFER_THREADS, SYS == SYS_CO2AR ? 4 : 1) defer_eval_kernel(DeferArgs a, TrajParams P, TrajIO io,
                                                                   const Co2arTablesGlobal *gtab) {
  using DS = DeferSys<SYS, PHYS, STG>;
  constexpr int NQ = DS::NQ;
  using Ctx = SampleCtx<STG, NQ>;
  static_assert(sizeof(STG) == 4 && sizeof(PHYS) == 4 && NQ % 2 == 0 && sizeof(Ctx) % 16 == 0, "vector loads of the context");
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char df_smem[];
  DS ds;
  ds.init(df_smem, gtab, io);
  __syncthreads();
  const unsigned long long count = defer_count(a);
  const Ctx *ctx = static_cast<const Ctx *>(a.ctx);
  const PHYS *mu0s = static_cast<const PHYS *>(a.item_mu0);
  PHYS *first_v = static_cast<PHYS *>(a.first_v);
  PHYS *last_v = static_cast<PHYS *>(a.last_v);
  const int lane = threadIdx.x & 31;
  const unsigned long long gw = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nw = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long base = gw * 32; base < count; base += nw * 32) {
    // the warp's 32 contexts and the prefix sum of their sample counts
    const unsigned long long ci = base + lane;
    const int n = ci < count ? ctx[ci].n : 0;
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += v;
    }
    const int off = incl - n;
    const int total = __shfl_sync(FULL, incl, 31);
    PHYS tail = PHYS(0);  // the last sample of the previous round
    for (int j0 = 0; j0 < total; j0 += 32) {
      const int j = j0 + lane;
      int o = 0;  // owner: the largest lane whose offset is <= j
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int oc = __shfl_sync(FULL, off, o + step);
        if (oc <= j) o += step;
      }
      const int jj = j - __shfl_sync(FULL, off, o);
      const bool valid = j < total;
      PHYS v = PHYS(0);
      bool nan = false;
      int kk = 0, item = 0, nn = 0;
      if (valid) {
        // the context in 16-byte loads: qold, (t0, inv_h), (item, k0, n, prev), F
        const Ctx *cp = ctx + base + o;
        double qo[NQ];
#pragma unroll
        for (int i = 0; i < NQ / 2; ++i) {
          const double2 v2 = reinterpret_cast<const double2 *>(cp->qold)[i];
          qo[2 * i] = v2.x;
          qo[2 * i + 1] = v2.y;
        }
        const double2 th = *reinterpret_cast<const double2 *>(&cp->t0);
        const int4 hd = *reinterpret_cast<const int4 *>(&cp->item);
        STG F[7 * NQ];
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
        item = hd.x;
        nn = hd.z;
        kk = hd.y + jj;
        const double x = (double(kk) * P.dt - th.x) * th.y;
        const STG xs = STG(x), x1 = STG(1) - STG(x);
        PHYS d[3];
        if constexpr (DS::FLOAT_Q) {
          // y = y_old + F0 x + F1 x(1-x) + F2 x^2(1-x) + ... + F6 x^4(1-x)^3 with the
          // basis formed once and one FMA per term; the position in FP32
          STG bs[7];
          bs[0] = xs;
          bs[1] = xs * x1;
          bs[2] = bs[1] * xs;
          bs[3] = bs[2] * x1;
          bs[4] = bs[3] * xs;
          bs[5] = bs[4] * x1;
          bs[6] = bs[5] * xs;
          float qf[NQ];
#pragma unroll
          for (int cq = 0; cq < NQ; ++cq) {
            STG w = F[cq] * bs[0];
#pragma unroll
            for (int r = 1; r < 7; ++r) w = fmaf(F[r * NQ + cq], bs[r], w);
            qf[cq] = float(qo[cq]) + w;
          }
          ds.dipole(qf, d);
        } else {
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
        }
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
        // the reference's tests on an FP32 value: |v| > 1e100 is v = +-inf, and
        // |v / pv| > 1e10 is |v| > 1e10 |pv| (1e10 is exact in FP32; a zero pv fails
        // any v != 0, NaN fails neither)
        unsigned code = 0xffffffffu;
        if (nan) code = (unsigned(kk) << 3) | 1u;
        else if (item + 2 * a.traj_base == P.inject_item && kk == P.inject_k) code = (unsigned(kk) << 3) | 4u;
        else if (isinf(v)) code = (unsigned(kk) << 3) | 2u;
        else if (jj > 0 && kk > 1 && fabsf(v) > 1e10f * fabsf(pv)) code = (unsigned(kk) << 3) | 3u;
        if (code != 0xffffffffu) atomicMin(&a.item_fail[item], code);
        if (!isnan(v) && !isinf(v)) {
          double *crln = a.crln + (size_t)((item >> 1) / a.traj_per_iter) * (size_t)P.N;
          atomicAdd(&crln[kk], P.weight * double(v));
        }
        if (jj == 0) first_v[base + o] = v;
        if (jj == nn - 1) last_v[base + o] = v;
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
