// CH4-CO2 dipole on the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
// Per radial piece p the dipole of PES-IDS/ai_ids_ch4_co2.cpp:672-1067 is a bilinear
// form in the two sets of real harmonics (hh_ch4co2_dip.cuh has the entry stream):
//   mu_c(r) = sum_n Y1_n(r) T_c[r, n],   T_c[r, n] = sum_{k, j} Y2_k(r) x(r)^j B_c,p[n, 4k + j]
// with n over the 196 Y1 functions (l1 <= 13, m-major, cos then sin), k over the 91 Y2
// functions, j over the 4 powers of x = R - centre_p of the piece's cubic, and B the
// folded coefficients (zero where the reference has no term).  For a tile of 128
// records of one piece the inner sum is a GEMM
//   T_c (128 x 196) = A (128 x 364) . B_c,p^T,   A[r, 4k + j] = Y2_k(r) x(r)^j,
// run on the tensor cores in TF32 with a three-product split for FP32 accuracy
// (A = A_hi + A_lo with A_hi the TF32 part the tensor core reads and A_lo = A - A_hi;
// B = B_hi + B_lo rounded on the host; T = A_hi B_hi + A_hi B_lo + A_lo B_hi: the
// dropped A_lo B_lo is about 2^-20 of a product).  The outer sum over n (196 FMAs per
// component) and the rotation to the lab frame run on the CUDA cores from TMEM.  The
// harmonics' recurrences take their integer-only square roots from constant tables,
// so neither the split nor the recurrences use the transcendental pipe.
//
// Mapping (one CTA of 17 warps per SM, persistent over the 128-record tasks):
//   - 16 producer warps, four per TMEM lane quadrant: the four threads of record t
//     (one per quarter) compute its geometry and x powers, walk its Y2 with a
//     generator (in registers) and write their column groups of each A chunk into
//     shared memory in the canonical no-swizzle K-major layout (8-row x 16-byte core
//     matrices; K-adjacent cores 128 B apart, 8-row groups 512 B apart);
//   - K is walked in chunks of 16 (23 chunks for K = 368, the last 4 columns zero);
//     the chunk's B_hi | B_lo image (built on the host in the same layout) arrives by
//     one bulk copy (cp.async.bulk, this GPU's memory only, no multicast) into a ring
//     of three stages;
//   - one issuing warp (one lane) issues the copies two chunks ahead and the
//     tcgen05.mma instructions of each chunk (M = 128, N = 208, K = 8 each) and
//     commits them to the stage's mbarrier, which frees the stage; producers and
//     issuer meet only at mbarriers, so A production, copies and MMAs overlap;
//   - TMEM holds two 208-column accumulators: pass 0 computes components 0 and 1,
//     pass 1 component 2 (the three would need 624 of the 512 columns);
//   - after a pass the producers read their TMEM lanes (tcgen05.ld 32x32b) and form
//     sum_n Y1_n T[t, n] with Y1 generated by its recurrence in column order (pass 0:
//     the two halves take one component each).
// Every mbarrier wait is bounded: on a timeout the CTA records the error in *err,
// stops issuing work, waits (bounded) for what it issued and frees its TMEM.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_ch4co2_dip.cuh"
#include "hh_ch4co2_tc_layout.h"

namespace hh {

constexpr int CH4TC_A_BYTES = CH4TC_M * CH4TC_KC * 4;    // one A image (hi or lo): 8 KB
constexpr int CH4TC_STAGE_B = 2 * CH4TC_IMG0;            // B_hi | B_lo of the widest pass
constexpr int CH4TC_STAGES = 3;
// dynamic shared memory: 3 stages x (A_hi, A_lo, B_hi | B_lo) = 204 KB, 1 KB alignment
constexpr size_t CH4TC_SMEM = CH4TC_STAGES * (2 * CH4TC_A_BYTES + CH4TC_STAGE_B) + 1024;
constexpr unsigned CH4TC_TMEM_COLS = 512;
constexpr unsigned CH4TC_COL1 = 256;            // TMEM column of the second accumulator
constexpr long long CH4TC_WAIT_LIMIT = 1LL << 24;  // polls of an mbarrier before giving up

struct Ch4TcArgs {
  const float *records;       // FP32 records (r, quaternion, u, pad)
  const int *sorted;          // record index per task slot, -1 for padding (tasks of 128)
  const long long *warp0;     // first task of each piece; [NSEG] = total tasks
  const unsigned char *blob;  // B images (ch4tc_blob_off), 16-byte aligned
  float *mu;                  // [record][4] lab-frame dipole
  double centre[CH4_NSEG];
  long long max_tasks, task_step;  // as Ch4DipArgs: a timing run takes a spread-out subset
  int *err;                   // set when an mbarrier wait gave up
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: no swizzle, K-major, LBO 128 B (K-adjacent core
// matrices), SBO 512 B (8-row groups), descriptor version 1
__device__ __forceinline__ uint64_t ch4tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(512u >> 4) << 32) |
         (1ull << 46);
}

// instruction descriptor: D F32, A and B TF32, both K-major, N = 208, M = 128
constexpr uint32_t CH4TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(CH4TC_N >> 3) << 17) |
                                 ((uint32_t)(CH4TC_M >> 4) << 24);

// the TF32 part the tensor core reads of an FP32 operand: its low 13 mantissa bits
// cleared (one integer AND, no conversion instruction); v - tf32_hi(v) is exact in FP32
__device__ __forceinline__ float tf32_hi(float v) { return __uint_as_float(__float_as_uint(v) & 0xFFFFE000u); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// bounded wait for the phase of parity `par`; false on a timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned par) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < CH4TC_WAIT_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(par)
        : "memory");
    if (done) return true;
  }
  return false;
}

// one bulk copy of `bytes` from global memory into shared memory, completing on `bar`
__device__ __forceinline__ void ch4tc_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void ch4tc_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(CH4TC_IDESC), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void ch4tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Coefficients of the harmonics' recurrences, set once per context by the host: for
// (l, m) with l > m the normalised three-term recurrence Q_l = alpha z Q_(l-1) -
// beta Q_(l-2), i.e. alpha =
// (2l - 1) / sqrt(l^2 - m^2), beta = sqrt((l - 1)^2 - m^2) / sqrt(l^2 - m^2) (alpha =
// sqrt(2m + 1), beta = 0 at l = m + 1), and per m the factor pm_m of (x + i y)^m
// (pm_0 = 1, pm_m = -pm_(m-1) sqrt((2m - 1) / 2m)): the recurrence of ch4_dipole_kernel
// with its integer-only square roots taken out of the loop.
__constant__ float c_ch4tc_alpha[CH4_L1 + 1][CH4_L1 + 1];  // [m][l]
__constant__ float c_ch4tc_beta[CH4_L1 + 1][CH4_L1 + 1];
__constant__ float c_ch4tc_pm[CH4_L1 + 1];

// first Y2 index of m (order of ch4_y2: m = 0..12, l = m..12 even, cos then sin)
HH_TC_HD constexpr int ch4tc_y2_off(int m2) {
  int c = 0;
  for (int m = 0; m < m2; ++m) c += (m == 0 ? 1 : 2) * (CH4_L2 / 2 + 1 - (m + 1) / 2);  // even l in [m, L2]
  return c;
}
static_assert(ch4tc_y2_off(CH4_L2 + 1) == CH4_NY2, "Y2 count");

// (cos, sin) of m phi as (x + i y)^m (the harmonics' unnormalised azimuthal factor)
__device__ __forceinline__ void ch4tc_cs_m(float x, float y, int m, float &C, float &Sn) {
  C = 1.f;
  Sn = 0.f;
  for (int i = 0; i < m; ++i) {
    const float c = C * x - Sn * y;
    Sn = C * y + Sn * x;
    C = c;
  }
}

// sum over the Y1 columns of m in [m0, m1) (m-major, l = m..13, cos then sin) of
// Y1_n(n1) T_i[n] for NA accumulators at TMEM addresses taddr[i] (this thread's lane),
// the recurrence of Y1 shared between them; m0 and m1 are uniform across the warp
// (tcgen05.ld is a warp-wide load)
template <int NA>
__device__ __forceinline__ void ch4tc_y1_dot(const uint32_t (&taddr)[NA], const float n1[3], int m0, int m1,
                                             float (&acc)[NA]) {
  const int c_begin = ch4tc_y1_col(m0, m0, 0, CH4_L1);
  const int c_end = (m1 > CH4_L1) ? CH4TC_NY1 : ch4tc_y1_col(m1, m1, 0, CH4_L1);
  float C, Sn;
  ch4tc_cs_m(n1[0], n1[1], m0, C, Sn);
  float pm = c_ch4tc_pm[m0], qa = 1.f, qb = 0.f, ys_pending = 0.f;
  int m = m0, l = m0;
  bool first = true, sin_next = false;
#pragma unroll
  for (int i = 0; i < NA; ++i) acc[i] = 0.f;
#pragma unroll 1
  for (int c0 = c_begin & ~15; c0 < c_end; c0 += 16) {
    float v[NA][16];
#pragma unroll
    for (int i = 0; i < NA; ++i) tmem_ld16(taddr[i] + (uint32_t)c0, v[i]);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int c = c0 + k;
      if (c >= c_begin && c < c_end) {
        float y;
        if (sin_next) {
          y = ys_pending;
          sin_next = false;
        } else {
          if (first) {
            first = false;
          } else if (l == CH4_L1) {
            ++m;
            l = m;
            const float cc = C * n1[0] - Sn * n1[1];
            Sn = C * n1[1] + Sn * n1[0];
            C = cc;
            pm = c_ch4tc_pm[m];
            qa = 1.f;
            qb = 0.f;
          } else {
            ++l;
            const float q = c_ch4tc_alpha[m][l] * n1[2] * qa - c_ch4tc_beta[m][l] * qb;
            qb = qa;
            qa = q;
          }
          y = pm * C * qa;
          if (m > 0) {
            ys_pending = pm * Sn * qa;
            sin_next = true;
          }
        }
#pragma unroll
        for (int i = 0; i < NA; ++i) acc[i] = fmaf(y, v[i][k], acc[i]);
      }
    }
  }
}

// The Y2 of one record in the order of ch4_y2 (m = 0..12, even l = m..12, cos then
// sin for m > 0), one value per next(): (cos, sin)(m phi) as (x + i y)^m times pm_m,
// and the normalised three-term recurrence in l, run as a generator so that a thread
// walks the A columns chunk by chunk without a table.
struct Ch4TcY2Gen {
  float x, y, z, C, Sn, pm, qa, qb, pend;
  int m, l;
  bool sin_next;
  __device__ __forceinline__ void reset(float x_, float y_, float z_) {
    x = x_;
    y = y_;
    z = z_;
    C = 1.f;
    Sn = 0.f;
    pm = c_ch4tc_pm[0];
    qa = 1.f;
    qb = 0.f;
    pend = 0.f;
    m = 0;
    l = 0;
    sin_next = false;
  }
  // the first value of m = m0 next: (cos, sin)(m0 phi) by ch4tc_cs_m, whose products are
  // those of the rotations a walk from m = 0 makes, so the values are the same
  __device__ __forceinline__ void start(float x_, float y_, float z_, int m0) {
    reset(x_, y_, z_);
    ch4tc_cs_m(x, y, m0, C, Sn);
    m = m0;
    l = m0;
    pm = c_ch4tc_pm[m0];
  }
  // to the next (m, l): l + 1 by the recurrence, or m + 1 with l = m
  __device__ __forceinline__ void advance() {
    if (l == CH4_L2) {
      ++m;
      l = m;
      const float c = C * x - Sn * y;
      Sn = C * y + Sn * x;
      C = c;
      pm = c_ch4tc_pm[m];
      qa = 1.f;
      qb = 0.f;
    } else {
      ++l;
      const float q = c_ch4tc_alpha[m][l] * z * qa - c_ch4tc_beta[m][l] * qb;
      qb = qa;
      qa = q;
    }
  }
  // the next of the 91 values (not called past the last)
  __device__ __forceinline__ float next() {
    if (sin_next) {
      sin_next = false;
      return pend;
    }
    if (l & 1) advance();  // odd l: no value, on to the even l after it
    const float v = pm * C * qa;
    if (m > 0) {
      pend = pm * Sn * qa;
      sin_next = true;
    }
    advance();
    return v;
  }
};

// Warp roles (17 warps): warps 0..15 produce the A chunks and run the epilogue, four
// per TMEM lane quadrant; thread t < 512 works on record row = t % 128 and its quarter
// qt = t / 128 takes
//   - column group qt of every A chunk (its 4 powers of x, hi and lo): chunk c's group qt
//     holds Y2 index 23 qt + c (ch4tc_k_of), so the thread's generator walks only its
//     quarter of the Y2 sequence, one value per chunk;
//   - the Y1 columns of m in its quarter's range (CH4TC_Y1_M) of components 0 and 1 in
//     pass 0, with one Y1 recurrence for both, and of component 2 in pass 1;
// the partial sums meet in shared memory and quarter 0 finishes the record.  Warp 16
// (one lane) issues the B copies and the MMAs.  The two sides meet only at mbarriers:
//   full_a[s]  the 16 producer warps wrote stage s's A (after fence.proxy.async);
//   full_b[s]  stage s's B copy landed (complete_tx);
//   empty[s]   the MMAs that read stage s are done (tcgen05.commit): A and B of the
//              chunk three later may be written;
//   tfree      the producers read the accumulators of a pass: the next pass's MMAs
//              may overwrite them.
// Chunk g uses stage g % 3, and the n-th completion of a stage's barriers belongs to
// its chunk 3 n + stage.  Every wait is bounded; a thread whose wait gives up sets
// bad_s and skips its work up to the next agreement point (the producers' pass-end
// barrier, a reduction over bad_s), where all producers leave together.
constexpr int CH4TC_PRODUCERS = 4 * CH4TC_M;
constexpr int CH4TC_THREADS = CH4TC_PRODUCERS + 32;
__constant__ int CH4TC_Y1_M[5] = {0, 2, 4, 7, CH4_L1 + 1};  // the quarters' m ranges of Y1
static_assert(CH4TC_QLEN == CH4TC_NCHUNK && 4 * CH4TC_QLEN >= CH4_NY2, "one Y2 per quarter and chunk");

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// barrier 1 over the 512 producer threads; true if any of them passed `bad`
__device__ __forceinline__ bool ch4tc_producers_sync_or(bool bad) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)bad), "n"(CH4TC_PRODUCERS)
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(CH4TC_THREADS, 1) ch4_dipole_tc_kernel(Ch4TcArgs a) {
  extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
  unsigned char *smem = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
  // stage s: A_hi, A_lo, B (hi | lo)
  constexpr size_t STAGE_BYTES = 2 * CH4TC_A_BYTES + CH4TC_STAGE_B;
  auto stA = [&](int s, int lo) { return smem + (size_t)s * STAGE_BYTES + (size_t)lo * CH4TC_A_BYTES; };
  auto stB = [&](int s) { return smem + (size_t)s * STAGE_BYTES + 2 * CH4TC_A_BYTES; };
  __shared__ __align__(8) uint64_t bar_fa[CH4TC_STAGES], bar_fb[CH4TC_STAGES], bar_empty[CH4TC_STAGES], bar_tfree;
  __shared__ uint32_t tmem_base_s;
  __shared__ volatile int bad_s;
  __shared__ long long w0[CH4_NSEG + 1];
  __shared__ float part_s[3][4][CH4TC_M];  // the quarters' partial sums, per component
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i <= CH4_NSEG; i += blockDim.x) w0[i] = a.warp0[i];
  if (t == 0) {
    for (int s = 0; s < CH4TC_STAGES; ++s) {
      mbar_init(&bar_fa[s], CH4TC_PRODUCERS / 32);
      mbar_init(&bar_fb[s], 1);
      mbar_init(&bar_empty[s], 1);
    }
    mbar_init(&bar_tfree, CH4TC_PRODUCERS / 32);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    bad_s = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(CH4TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const long long total = min((w0[CH4_NSEG] + a.task_step - 1) / a.task_step, a.max_tasks);
  auto seg_of = [&](long long task) {
    int s = 0;
    while (s < CH4_NSEG - 1 && w0[s + 1] <= task) ++s;
    return s;
  };
  auto fail = [&]() {
    if (!bad_s) {
      bad_s = 1;
      atomicExch(a.err, 1);
    }
  };

  if (warp == CH4TC_PRODUCERS / 32) {
    // ---------------- issuer: B copies and MMAs (one lane) ----------------
    if (lane == 0) {
      // the chunk walk (task, pass q, chunk c) of this CTA, for the copies two ahead
      struct Walk {
        long long task;
        int q, c;
      };
      auto step = [&](Walk &w) -> bool {
        if (++w.c == CH4TC_NCHUNK) {
          w.c = 0;
          if (++w.q == 2) {
            w.q = 0;
            w.task += gridDim.x;
          }
        }
        return w.task < total;
      };
      long long seg_task = -1;
      int seg_cached = 0;
      auto issue_load = [&](const Walk &w, int s) {
        if (w.task != seg_task) {
          seg_task = w.task;
          seg_cached = seg_of(w.task * a.task_step);
        }
        const unsigned bytes = w.q == 0 ? 2 * CH4TC_IMG0 : 2 * CH4TC_IMG1;
        ch4tc_load(stB(s), a.blob + ch4tc_blob_off(seg_cached, w.q, w.c), bytes, &bar_fb[s]);
      };
      unsigned gl = 0, gm = 0;  // copies issued, chunks whose MMAs were committed
      Walk ld{(long long)blockIdx.x, 0, 0};
      bool more = ld.task < total;
      for (int i = 0; i < 2 && more; ++i) {
        issue_load(ld, (int)(gl % CH4TC_STAGES));
        ++gl;
        more = step(ld);
      }
      unsigned g = 0, np = 0;
      for (long long task = blockIdx.x; task < total && !bad_s; task += gridDim.x) {
        for (int q = 0; q < 2 && !bad_s; ++q, ++np) {
          const int ntile = q == 0 ? 2 : 1;
          // the previous pass's accumulators have been read
          if (np > 0 && !mbar_wait(&bar_tfree, (np - 1) & 1)) {
            fail();
            break;
          }
          tc_fence_after();
          for (int c = 0; c < CH4TC_NCHUNK; ++c, ++g) {
            const int s = g % CH4TC_STAGES;
            const unsigned par = (g / CH4TC_STAGES) & 1;
            if (!mbar_wait(&bar_fa[s], par) || !mbar_wait(&bar_fb[s], par)) {
              fail();
              break;
            }
            tc_fence_after();
            const uint32_t a_hi = smem_u32(stA(s, 0)), a_lo = smem_u32(stA(s, 1));
            const uint32_t b_hi = smem_u32(stB(s));
            const uint32_t b_lo = b_hi + (q == 0 ? CH4TC_IMG0 : CH4TC_IMG1);
#pragma unroll 1
            for (int nt = 0; nt < ntile; ++nt) {
              const uint32_t d = tmem + (nt == 0 ? 0u : CH4TC_COL1);
              const uint32_t boff = (uint32_t)nt * (CH4TC_N / 8) * 512u;
#pragma unroll
              for (int ks = 0; ks < 2; ++ks) {
                const uint32_t ko = (uint32_t)ks * 256u;
                const uint32_t first_acc = (c == 0 && ks == 0) ? 0u : 1u;
                ch4tc_mma(d, ch4tc_desc(a_hi + ko), ch4tc_desc(b_hi + boff + ko), first_acc);
                ch4tc_mma(d, ch4tc_desc(a_hi + ko), ch4tc_desc(b_lo + boff + ko), 1u);
                ch4tc_mma(d, ch4tc_desc(a_lo + ko), ch4tc_desc(b_hi + boff + ko), 1u);
              }
            }
            ch4tc_commit(&bar_empty[s]);
            gm = g + 1;
            // the copy two chunks ahead, into the stage whose MMAs (chunk g - 1) are
            // queued ahead of this chunk's
            if (more) {
              const unsigned h = gl;  // == g + 2
              const int s2 = h % CH4TC_STAGES;
              if (h >= (unsigned)CH4TC_STAGES && !mbar_wait(&bar_empty[s2], ((h - CH4TC_STAGES) / CH4TC_STAGES) & 1)) {
                fail();
                break;
              }
              issue_load(ld, s2);
              ++gl;
              more = step(ld);
            }
          }
        }
      }
      // drain (bounded): the committed MMAs and the copies issued
      if (gm > 0) mbar_wait(&bar_empty[(gm - 1) % CH4TC_STAGES], ((gm - 1) / CH4TC_STAGES) & 1);
      for (unsigned h = gm; h < gl; ++h) mbar_wait(&bar_fb[h % CH4TC_STAGES], (h / CH4TC_STAGES) & 1);
    }
    __syncwarp();
  } else {
    // ---------------- producers: A chunks, epilogue ----------------
    const int row = t & (CH4TC_M - 1), qt = t / CH4TC_M;
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    // this quarter's Y2 values, indices CH4TC_QLEN qt .., start in the run of m = m_q,
    // d_q values into it
    int m_q = 0;
    while (m_q < CH4_L2 && ch4tc_y2_off(m_q + 1) <= CH4TC_QLEN * qt) ++m_q;
    const int d_q = CH4TC_QLEN * qt - ch4tc_y2_off(m_q);
    unsigned g = 0;
    bool stop = false;
    for (long long task = blockIdx.x; task < total && !stop; task += gridDim.x) {
      const long long w = task * a.task_step;
      const int seg = seg_of(w);
      // ---- this thread's record: geometry, powers of x ----
      const int first = a.sorted[w * CH4TC_M];
      const int mine = a.sorted[w * CH4TC_M + row];
      const int src = mine >= 0 ? mine : first;
      const float *rec = a.records + (size_t)src * HH_REC_WORDS;
      float M[3][3], n1[3], n2[3];
      {
        const float r[3] = {rec[0], rec[1], rec[2]};
        const float qt4[4] = {rec[3], rec[4], rec[5], rec[6]};
        const float u[3] = {rec[7], rec[8], rec[9]};
        quat_matrix<float>(qt4, M);
        const float R = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        const float iR = 1.f / R;
        const float iu = 1.f / sqrtf(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          n1[k] = (M[0][k] * r[0] + M[1][k] * r[1] + M[2][k] * r[2]) * iR;
          n2[k] = (M[0][k] * u[0] + M[1][k] * u[1] + M[2][k] * u[2]) * iu;
        }
      }
      const float R = sqrtf(rec[0] * rec[0] + rec[1] * rec[1] + rec[2] * rec[2]);
      const float x = R - float(a.centre[seg]);
      const float xp[4] = {1.f, x, x * x, x * x * x};
      float acc[3] = {0.f, 0.f, 0.f};
      for (int q = 0; q < 2; ++q) {
        Ch4TcY2Gen y2g;
        y2g.start(n2[0], n2[1], n2[2], m_q);
        for (int i = 0; i < d_q; ++i) (void)y2g.next();
        bool bad = bad_s != 0;
        for (int c = 0; c < CH4TC_NCHUNK; ++c, ++g) {
          const int s = g % CH4TC_STAGES;
          // this thread's Y2 of the chunk (column group qt): the quarter's next value
          const float y2 = ch4tc_k_of(c, qt) >= 0 ? y2g.next() : 0.f;
          // stage s is free once the MMAs of chunk g - 3 are done
          if (!bad && g >= (unsigned)CH4TC_STAGES &&
              !mbar_wait(&bar_empty[s], ((g - CH4TC_STAGES) / CH4TC_STAGES) & 1)) {
            bad = true;
            fail();
          }
          if (!bad) {
            float4 hi, lo;
            float *ph = &hi.x, *pl = &lo.x;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float v = y2 * xp[j];
              const float h = tf32_hi(v);
              ph[j] = h;
              pl[j] = v - h;
            }
            *reinterpret_cast<float4 *>(reinterpret_cast<float *>(stA(s, 0)) + ch4tc_img_off(row, 4 * qt)) = hi;
            *reinterpret_cast<float4 *>(reinterpret_cast<float *>(stA(s, 1)) + ch4tc_img_off(row, 4 * qt)) = lo;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          }
          __syncwarp();
          if (lane == 0 && !bad) mbar_arrive(&bar_fa[s]);
          if (!bad && bad_s) bad = true;
        }
        // ---- all MMAs of this pass done: the quarters' partial sums from TMEM ----
        if (!bad && !mbar_wait(&bar_empty[(g - 1) % CH4TC_STAGES], ((g - 1) / CH4TC_STAGES) & 1)) {
          bad = true;
          fail();
        }
        // tcgen05.ld is a warp-wide instruction: the warp reads TMEM or skips it as one
        bad = __any_sync(0xffffffffu, bad);
        tc_fence_after();
        if (!bad) {
          // the quarter's m range of the Y1 columns: components 0 and 1 in pass 0 (one
          // Y1 recurrence for both), component 2 in pass 1
          if (q == 0) {
            const uint32_t ta[2] = {lane_addr, lane_addr + CH4TC_COL1};
            float v[2];
            ch4tc_y1_dot<2>(ta, n1, CH4TC_Y1_M[qt], CH4TC_Y1_M[qt + 1], v);
            part_s[0][qt][row] = v[0];
            part_s[1][qt][row] = v[1];
          } else {
            const uint32_t ta[1] = {lane_addr};
            float v[1];
            ch4tc_y1_dot<1>(ta, n1, CH4TC_Y1_M[qt], CH4TC_Y1_M[qt + 1], v);
            part_s[2][qt][row] = v[0];
          }
        }
        // the accumulators may be rewritten by the next pass's MMAs
        tc_fence_before();
        __syncwarp();
        if (lane == 0 && !bad) mbar_arrive(&bar_tfree);
        if (ch4tc_producers_sync_or(bad || bad_s)) {
          stop = true;
          break;
        }
        if (qt == 0) {
#pragma unroll
          for (int cc = (q == 0 ? 0 : 2); cc < (q == 0 ? 2 : 3); ++cc)
            acc[cc] = (part_s[cc][0][row] + part_s[cc][1][row]) + (part_s[cc][2][row] + part_s[cc][3][row]);
        }
      }
      if (stop) break;
      if (seg == CH4_NSEG - 1) {
        const float i2 = 1.f / (R * R);
        const float i6 = i2 * i2 * i2;
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) acc[cc] *= i6;
      }
      if (qt == 0 && mine >= 0) {
        float *o = a.mu + (size_t)mine * 4;
#pragma unroll
        for (int i = 0; i < 3; ++i) o[i] = M[i][0] * acc[0] + M[i][1] * acc[1] + M[i][2] * acc[2];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CH4TC_TMEM_COLS)
                 : "memory");
}

}  // namespace hh
