// Batched CH4-CO2 dipole and the correlation step of the record path.
//
// The induced dipole of PES-IDS/ai_ids_ch4_co2.cpp:672-1067 is, per Cartesian
// component c of the CH4 body frame,
//   mu_c = sum_e  Y1_e(n1) Y2_e(n2) K_e(R)
// over 8,658 entries e = (c, Y1, Y2) (hh_ch4co2_host.cpp folds the 320 radial
// functions of each entry into one piecewise cubic on their common grid of 30
// pieces).  n1 and n2 are the directions of the intermolecular axis and of the
// CO2 axis in the CH4 body frame; Y1 (l <= 13) and Y2 (even l <= 12) are real
// spherical harmonics with the Legendre normalisation sqrt((l-m)!/(l+m)!) (the
// table carries the inverse factor), computed from the unit vectors by the
// three-term recurrence in l and (x + i y)^m, without angles.
//
// Inside a trajectory kernel the 32 lanes of a warp sit at different R, so each
// coefficient load would be a 32-way gather over pieces.  Instead the trajectory
// kernel writes each sample as a record and:
//   1. seg_count / seg_scan / seg_scatter sort the valid records by radial piece,
//      each piece padded to a multiple of the warp task (32 S records), so every
//      warp task has one piece;
//   2. dipole_kernel: a warp evaluates 32 S records of one piece, S per lane; the
//      coefficient stream of that piece is the same for all lanes (broadcast loads,
//      shared by a lane's S records) and is walked in batches of 4 entries, the next
//      batch loaded while one is summed; the S values of Y2 of each index sit side by
//      side in shared memory (one vector load); Y1 is generated in the order of the
//      stream;
//   3. corr_kernel applies the reference's per-sample tests in order (NaN dipole,
//      |C| > 1e100, |C_k / C_k-1| > 1e10: src/hawaii.c:2183-2243) and adds
//      w mu0.mu(t_k) of every trajectory that passes into C(t).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_ch4co2_tables.h"
#include "hh_traj.cuh"

namespace hh {

constexpr int CH4_NSEG = HH_CH4CO2_NSEG;
constexpr int CH4_L1 = HH_CH4CO2_L1MAX;
constexpr int CH4_L2 = HH_CH4CO2_L2MAX;
constexpr int CH4_NY2 = 91;  // even l2 <= 12, all m2 and cos/sin
constexpr int CH4_DIP_WARPS = 4;

// folded dipole table in device memory (built by ch4co2_build_fold): the entries in
// batches of 4, each group (one Y1, cos or sin, one component) padded with zero
// entries to whole batches
struct Ch4Co2Fold {
  int n_batch;
  const float4 *cf;             // [NSEG][4 n_batch] (c0, c1, c2, c3), FP32
  const double2 *cd;            // [NSEG][4 n_batch][2] (c0, c1), (c2, c3), FP64
  const unsigned int *y2;       // [n_batch] the batch's four Y2 indices, one byte each
  const unsigned int *meta;     // [n_batch] cs | comp << 1 | (ends its group) << 3 | lm << 8
  double seg_hi[CH4_NSEG - 1];
  double centre[CH4_NSEG];
};

struct Ch4SortArgs {
  const void *records;
  const int *rec_len;
  long long n_traj;           // trajectories of this chunk
  int stride, N;
  unsigned int *count;        // [NSEG]
  unsigned int *cursor;       // [NSEG]
  long long *warp0;           // [NSEG + 1] first warp task of each piece; [NSEG] = total
  int *sorted;                // record index per task slot, -1 for padding
  int task;                   // records per warp task (32 S)
  double seg_hi[CH4_NSEG - 1];
};

template <typename PHYS> __device__ __forceinline__ int ch4_seg(const double *hi, PHYS R) {
  int s = 0;
#pragma unroll 1
  while (s < CH4_NSEG - 1 && double(R) >= hi[s]) ++s;
  return s;
}

// slot sl of trajectory t holds a stored sample
__device__ __forceinline__ bool ch4_valid(const int *rec_len, long long t, int sl, int N) {
  if (sl == 0) return true;
  if (sl < N) return sl <= rec_len[2 * t];
  return sl - (N - 1) <= rec_len[2 * t + 1];
}

template <typename PHYS> __device__ __forceinline__ PHYS ch4_rec_R(const void *records, long long i) {
  const PHYS *r = static_cast<const PHYS *>(records) + i * HH_REC_WORDS;
  return sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

template <typename PHYS>
__global__ void __launch_bounds__(256) ch4_seg_count_kernel(Ch4SortArgs a) {
  __shared__ unsigned int h[CH4_NSEG];
  for (int i = threadIdx.x; i < CH4_NSEG; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const long long n = a.n_traj * a.stride;
  const int lane = threadIdx.x & 31;
  for (long long b0 = blockIdx.x * (long long)blockDim.x; b0 < n; b0 += (long long)gridDim.x * blockDim.x) {
    const long long i = b0 + threadIdx.x;
    int s = -1;
    if (i < n) {
      const long long t = i / a.stride;
      const int sl = (int)(i - t * a.stride);
      if (ch4_valid(a.rec_len, t, sl, a.N)) s = ch4_seg(a.seg_hi, ch4_rec_R<PHYS>(a.records, i));
    }
    // one shared-memory atomic per (warp, piece)
    const unsigned peers = __match_any_sync(0xffffffffu, s);
    if (s >= 0 && lane == __ffs(peers) - 1) atomicAdd(&h[s], (unsigned)__popc(peers));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < CH4_NSEG; i += blockDim.x)
    if (h[i]) atomicAdd(&a.count[i], h[i]);
}

// one warp: piece offsets in warp tasks, cursors reset
__global__ void ch4_seg_scan_kernel(Ch4SortArgs a) {
  if (threadIdx.x == 0) {
    long long w = 0;
    for (int s = 0; s < CH4_NSEG; ++s) {
      a.warp0[s] = w;
      w += (a.count[s] + a.task - 1) / a.task;
      a.cursor[s] = 0;
    }
    a.warp0[CH4_NSEG] = w;
  }
}

// one cursor atomic per (warp, piece): the lanes of a warp that land in the same piece
// (consecutive slots of a trajectory mostly do) take consecutive positions
template <typename PHYS>
__global__ void __launch_bounds__(256) ch4_seg_scatter_kernel(Ch4SortArgs a) {
  const long long n = a.n_traj * a.stride;
  const int lane = threadIdx.x & 31;
  for (long long b0 = blockIdx.x * (long long)blockDim.x; b0 < n; b0 += (long long)gridDim.x * blockDim.x) {
    const long long i = b0 + threadIdx.x;
    int s = -1;
    if (i < n) {
      const long long t = i / a.stride;
      const int sl = (int)(i - t * a.stride);
      if (ch4_valid(a.rec_len, t, sl, a.N)) s = ch4_seg(a.seg_hi, ch4_rec_R<PHYS>(a.records, i));
    }
    const unsigned peers = __match_any_sync(0xffffffffu, s);
    const int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (s >= 0 && lane == leader) base = atomicAdd(&a.cursor[s], (unsigned)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (s >= 0) a.sorted[a.warp0[s] * a.task + base + __popc(peers & ((1u << lane) - 1u))] = (int)i;
  }
}

struct Ch4DipArgs {
  Ch4Co2Fold f;
  const void *records;
  const int *sorted;
  const long long *warp0;
  void *mu;                   // [record][4] lab-frame dipole in the surface precision
  // tasks evaluated: 0, task_step, 2 task_step, ... below the total, at most max_tasks
  // of them (1 and all for a real run; a timing run takes a spread-out subset)
  long long max_tasks;
  long long task_step;
};

// S: records per lane of the dipole kernel (the S values of a Y2 index are one
// shared-memory vector).  More records per lane share each coefficient load among
// more samples; fewer leave room for more resident warps (the per-lane Y2 arrays
// take 91 x 32 x S values per warp).  The host picks S per precision by timing the
// candidates on the first chunk of records (hh_api.cu, ch4_tune_dipole).
constexpr int CH4_DIP_SMAX = 4;
template <typename PHYS, int S> __host__ __device__ constexpr size_t ch4_dip_smem() {
  return (size_t)CH4_DIP_WARPS * CH4_NY2 * 32 * S * sizeof(PHYS);
}

template <typename PHYS, int S> struct Vec;
template <> struct Vec<float, 4> { using T = float4; };
template <> struct Vec<float, 2> { using T = float2; };
template <> struct Vec<float, 1> { using T = float; };
template <> struct Vec<double, 2> { using T = double2; };
template <> struct Vec<double, 1> { using T = double; };
template <typename V> __device__ __forceinline__ auto vget(const V &v, int s);
__device__ __forceinline__ float vget(const float4 &v, int s) {
  return s == 0 ? v.x : s == 1 ? v.y : s == 2 ? v.z : v.w;
}
__device__ __forceinline__ double vget(const double2 &v, int s) { return s == 0 ? v.x : v.y; }
__device__ __forceinline__ float vget(const float2 &v, int s) { return s == 0 ? v.x : v.y; }
__device__ __forceinline__ float vget(const float &v, int) { return v; }
__device__ __forceinline__ double vget(const double &v, int) { return v; }

// Y2 of the CO2 axis n2 in the CH4 frame: even l <= 12, in the order
// m = 0..12, l = m..12 (even), cos then sin; Y[idx * 32 S + lane S + s]
template <typename T, int S>
__device__ __forceinline__ void ch4_y2(T x, T y, T z, T *Y, int lane, int s_) {
  T C = T(1), Sn = T(0), pm = T(1);
  int idx = 0;
  T *Yl = Y + lane * S + s_;
#pragma unroll 1
  for (int m = 0; m <= CH4_L2; ++m) {
    if (m > 0) {
      const T c = C * x - Sn * y;
      Sn = C * y + Sn * x;
      C = c;
      pm = -pm * sqrt(T(2 * m - 1) / T(2 * m));
    }
    T qa = T(1), qb = T(0);
#pragma unroll 1
    for (int l = m; l <= CH4_L2; ++l) {
      T q;
      if (l == m) q = T(1);
      else if (l == m + 1) q = sqrt(T(2 * m + 1)) * z;
      else q = (T(2 * l - 1) * z * qa - sqrt(T((l - 1) * (l - 1) - m * m)) * qb) / sqrt(T(l * l - m * m));
      if ((l & 1) == 0) {
        Yl[(idx++) * 32 * S] = pm * C * q;
        if (m > 0) Yl[(idx++) * 32 * S] = pm * Sn * q;
      }
      qb = qa;
      qa = q;
    }
  }
}

template <typename PHYS, int S>
__global__ void __launch_bounds__(32 * CH4_DIP_WARPS) ch4_dipole_kernel(Ch4DipArgs a) {
  using V = typename Vec<PHYS, S>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long w0[CH4_NSEG + 1];
  for (int i = threadIdx.x; i <= CH4_NSEG; i += blockDim.x) w0[i] = a.warp0[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  PHYS *Y2 = reinterpret_cast<PHYS *>(smem_raw) + (size_t)warp * CH4_NY2 * 32 * S;
  const V *Y2v = reinterpret_cast<const V *>(Y2) + lane;
  const long long total = min((w0[CH4_NSEG] + a.task_step - 1) / a.task_step, a.max_tasks);
  const long long nw = (long long)gridDim.x * CH4_DIP_WARPS;
  for (long long wi = (long long)blockIdx.x * CH4_DIP_WARPS + warp; wi < total; wi += nw) {
    const long long w = wi * a.task_step;
    int seg = 0;
    while (seg < CH4_NSEG - 1 && w0[seg + 1] <= w) ++seg;
    // record s of this lane: task slot s * 32 + lane; padding slots evaluate the
    // task's first record (always valid) and store nothing.  Shuffles run in every lane.
    int mine[S];
    PHYS x[S], M[S][3][3], n1[S][3], iR6[S];
    const int first = __shfl_sync(0xffffffffu, a.sorted[w * 32 * S + lane], 0);
#pragma unroll
    for (int s = 0; s < S; ++s) {
      mine[s] = a.sorted[w * 32 * S + s * 32 + lane];
      const int src = mine[s] >= 0 ? mine[s] : first;
      const PHYS *rec = static_cast<const PHYS *>(a.records) + (size_t)src * HH_REC_WORDS;
      const PHYS r[3] = {rec[0], rec[1], rec[2]};
      const PHYS qt[4] = {rec[3], rec[4], rec[5], rec[6]};
      const PHYS u[3] = {rec[7], rec[8], rec[9]};
      quat_matrix<PHYS>(qt, M[s]);
      const PHYS R = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      const PHYS iR = PHYS(1) / R;
      const PHYS iu = PHYS(1) / sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      PHYS n2[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        n1[s][k] = (M[s][0][k] * r[0] + M[s][1][k] * r[1] + M[s][2][k] * r[2]) * iR;
        n2[k] = (M[s][0][k] * u[0] + M[s][1][k] * u[1] + M[s][2][k] * u[2]) * iu;
      }
      ch4_y2<PHYS, S>(n2[0], n2[1], n2[2], Y2, lane, s);
      x[s] = R - PHYS(a.f.centre[seg]);
      const PHYS i2 = iR * iR;
      iR6[s] = i2 * i2 * i2;
    }
    __syncwarp();
    const float4 *cf = a.f.cf + (size_t)seg * 4 * a.f.n_batch;
    const double2 *cd = a.f.cd + (size_t)seg * 8 * a.f.n_batch;
    PHYS acc[S][3], C[S], Sn[S], qa[S], qb[S], Yc[S], Ys[S];
    // per-power sums A_j = sum_e Y2_e c_je of the current group, collapsed by Horner
    // at its end
    PHYS A0[S], A1[S], A2[S], A3[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      acc[s][0] = acc[s][1] = acc[s][2] = PHYS(0);
      C[s] = PHYS(1);
      Sn[s] = PHYS(0);
      qa[s] = qb[s] = Yc[s] = Ys[s] = PHYS(0);
      A0[s] = A1[s] = A2[s] = A3[s] = PHYS(0);
    }
    PHYS pm = PHYS(1);
    // Y1 position in the m-major order (l, m); "before (0, 0)" at the start
    int m = -1, l = CH4_L1, lm = -1;
    // one flat loop over the batches; the next batch's coefficients, indices and
    // descriptor are loaded while this one is summed
    PHYS cn[4][4];
    unsigned idn, dn;
    auto load = [&](int b) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if constexpr (sizeof(PHYS) == 4) {
          const float4 c4 = __ldg(&cf[4 * b + j]);
          cn[j][0] = c4.x; cn[j][1] = c4.y; cn[j][2] = c4.z; cn[j][3] = c4.w;
        } else {
          const double2 lo = __ldg(&cd[2 * (4 * b + j)]), hi = __ldg(&cd[2 * (4 * b + j) + 1]);
          cn[j][0] = lo.x; cn[j][1] = lo.y; cn[j][2] = hi.x; cn[j][3] = hi.y;
        }
      }
      idn = __ldg(&a.f.y2[b]);
      dn = __ldg(&a.f.meta[b]);
    };
    load(0);
    const int nb = a.f.n_batch;
#pragma unroll 1
    for (int b = 0; b < nb; ++b) {
      PHYS c[4][4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) c[j][k] = cn[j][k];
      const unsigned ids = idn, d = dn;
      if (b + 1 < nb) load(b + 1);
      V yv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) yv[j] = Y2v[int((ids >> (8 * j)) & 0xffu) * 32];
      // advance Y1 to this batch's (l, m) by the three-term recurrence in l and
      // (x + i y)^m (the same for every lane of the warp)
      const int want = int(d >> 8);
#pragma unroll 1
      while (lm < want) {
        ++lm;
        if (l == CH4_L1) {
          ++m;
          l = m;
          if (m > 0) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
              const PHYS cc = C[s] * n1[s][0] - Sn[s] * n1[s][1];
              Sn[s] = C[s] * n1[s][1] + Sn[s] * n1[s][0];
              C[s] = cc;
            }
            pm = -pm * sqrt(PHYS(2 * m - 1) / PHYS(2 * m));
          }
#pragma unroll
          for (int s = 0; s < S; ++s) {
            qa[s] = PHYS(1);
            qb[s] = PHYS(0);
          }
        } else {
          ++l;
          const PHYS ca = PHYS(2 * l - 1), cb = sqrt(PHYS((l - 1) * (l - 1) - m * m));
          const PHYS id = (l > m + 1) ? PHYS(1) / sqrt(PHYS(l * l - m * m)) : PHYS(0);
          const PHYS c1 = sqrt(PHYS(2 * m + 1));
#pragma unroll
          for (int s = 0; s < S; ++s) {
            const PHYS z = n1[s][2];
            const PHYS q = (l == m + 1) ? c1 * z : (ca * z * qa[s] - cb * qb[s]) * id;
            qb[s] = qa[s];
            qa[s] = q;
          }
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
          Yc[s] = pm * C[s] * qa[s];
          Ys[s] = pm * Sn[s] * qa[s];
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const PHYS y = vget(yv[j], s);
          A0[s] += y * c[j][0];
          A1[s] += y * c[j][1];
          A2[s] += y * c[j][2];
          A3[s] += y * c[j][3];
        }
      }
      if (d & 8u) {
        const unsigned comp = (d >> 1) & 3u;
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const PHYS sum = A0[s] + x[s] * (A1[s] + x[s] * (A2[s] + x[s] * A3[s]));
          const PHYS t = ((d & 1u) ? Ys[s] : Yc[s]) * sum;
          if (comp == 0) acc[s][0] += t;
          else if (comp == 1) acc[s][1] += t;
          else acc[s][2] += t;
          A0[s] = A1[s] = A2[s] = A3[s] = PHYS(0);
        }
      }
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
      if (seg == CH4_NSEG - 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[s][c] *= iR6[s];
      }
      if (mine[s] >= 0) {
        PHYS *o = static_cast<PHYS *>(a.mu) + (size_t)mine[s] * 4;
#pragma unroll
        for (int i = 0; i < 3; ++i) o[i] = M[s][i][0] * acc[s][0] + M[s][i][1] * acc[s][1] + M[s][i][2] * acc[s][2];
      }
    }
    __syncwarp();
  }
}

struct Ch4CorrArgs {
  const void *mu;
  const int *rec_len;
  const int *rec_status;
  long long n_traj;           // trajectories of this chunk
  long long traj_base;        // index of the chunk's first trajectory
  long long traj_per_iter;
  int stride;
  double *crln;
  const double *sat_w;        // [traj][n_sat] (global trajectory index) or nullptr
  int n_sat;
  unsigned int *status_hist;
  unsigned long long *n_failed;
  // check only (Zimmermann estimate): per trajectory 1 when dropped, and the stored
  // samples per item cut at a soft injected failure, instead of adding into crln
  int *fail_out;
  int *len_out;
};

template <typename PHYS>
__device__ __forceinline__ PHYS ch4_val(const PHYS *mu, long long slot, const PHYS *m0) {
  const PHYS *d = mu + slot * 4;
  return m0[0] * d[0] + m0[1] * d[1] + m0[2] * d[2];
}

// one thread per trajectory of the chunk
template <typename PHYS>
__global__ void __launch_bounds__(256) ch4_corr_kernel(TrajParams P, Ch4CorrArgs a) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool live = t < a.n_traj;
  const PHYS *mu = static_cast<const PHYS *>(a.mu);
  const long long base = (live ? t : 0) * a.stride;
  PHYS m0[3] = {PHYS(0), PHYS(0), PHYS(0)};
  int len[2] = {0, 0};
  bool failed = false;
  if (live) {
#pragma unroll
    for (int c = 0; c < 3; ++c) m0[c] = mu[base * 4 + c];
    for (int dir = 0; dir < 2; ++dir) {
      const long long item = 2 * (a.traj_base + t) + dir;
      int st = a.rec_status[2 * t + dir];
      len[dir] = a.rec_len[2 * t + dir];
      PHYS prev = PHYS(0);
      for (int k = 1; k <= len[dir]; ++k) {
        const long long slot = base + (dir ? P.N - 1 + k : k);
        const PHYS *d = mu + slot * 4;
        int code = -1;
        const PHYS val = m0[0] * d[0] + m0[1] * d[1] + m0[2] * d[2];
        if (isnan(d[0]) || isnan(d[1]) || isnan(d[2])) code = HH_ST_NAN_DIPOLE;
        else if (item == P.inject_item && k == P.inject_k) code = P.inject_status;
        else if (fabs(double(val)) > 1e100) code = HH_ST_OVERFLOW;
        else if (k > 1 && fabs(double(val) / double(prev)) > 1e10) code = HH_ST_JUMP;
        if (code >= 0) {
          st = code;
          if (code >= HH_ST_NAN_DIPOLE) failed = true;
          len[dir] = k - 1;
          break;
        }
        prev = val;
      }
      atomicAdd(&a.status_hist[st], 1u);
    }
    if (failed) atomicAdd(a.n_failed, 1ull);
    if (a.fail_out) {
      a.fail_out[t] = failed ? 1 : 0;
      a.len_out[2 * t] = len[0];
      a.len_out[2 * t + 1] = len[1];
    }
  }
  if (a.fail_out) return;
  const long long gt = a.traj_base + (live ? t : 0);
  const long long slice = (a.n_sat > 0) ? 0 : gt / a.traj_per_iter;
  const unsigned full = 0xffffffffu;
  const bool uniform = __all_sync(full, __shfl_sync(full, slice, 0) == slice);
  const bool add = live && !failed;
  const int nsl = a.n_sat > 0 ? a.n_sat : 1;
  for (int s = 0; s < nsl; ++s) {
    const double ws = P.weight * (a.n_sat > 0 ? (add ? a.sat_w[gt * a.n_sat + s] : 0.0) : 1.0);
    double *C = a.crln + (a.n_sat > 0 ? (long long)s * P.N : slice * P.N);
    const PHYS c0 = m0[0] * m0[0] + m0[1] * m0[1] + m0[2] * m0[2];
    // both branches add their t = 0 term
    double v0 = add ? 2.0 * ws * double(c0) : 0.0;
    if (uniform) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v0 += __shfl_down_sync(full, v0, o);
      if ((threadIdx.x & 31) == 0 && v0 != 0.0) atomicAdd(&C[0], v0);
    } else if (v0 != 0.0) {
      atomicAdd(&C[0], v0);
    }
    for (int dir = 0; dir < 2; ++dir) {
      const int my = add ? len[dir] : 0;
      int mx = my;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(full, mx, o));
      for (int k = 1; k <= mx; ++k) {
        double v = 0.0;
        if (k <= my) v = ws * double(ch4_val(mu, base + (dir ? P.N - 1 + k : k), m0));
        if (uniform) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
          if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&C[k], v);
        } else if (v != 0.0) {
          atomicAdd(&C[k], v);
        }
      }
    }
  }
}

// Zimmermann estimate (correlation_eval_zimmerman_trick, src/hawaii.c:1888-2114): per
// trajectory the dipole vectors d[c], c = 0..2N-2, with d[N-1] = mu0, d[N-1+k] = mu(t_k)
// and d[N-1-k] = mu(-t_k) (zero past a branch's stored samples), give
//   C(s) += w sum_{c < N} d[c] . d[c+s],   w = ppf ALU^3 / N,
// for trajectories that were not dropped.
struct ZimmArgs {
  const void *series;         // [traj][slot][4] in the surface precision
  const int *len;             // [2 traj] stored samples per branch
  const int *failed;          // [traj] 1 when dropped
  long long n_traj, traj_base, traj_per_iter;
  int stride, N;
  double w;
  double *crln;
};

template <typename PHYS>
__device__ __forceinline__ void zimm_d(const PHYS *sv, int N, int lf, int lb, int c, double d[3]) {
  int slot = -1;
  if (c == N - 1) slot = 0;
  else if (c > N - 1) { if (c - (N - 1) <= lf) slot = c - (N - 1); }
  else if ((N - 1) - c <= lb) slot = N - 1 + ((N - 1) - c);
  if (slot < 0) { d[0] = d[1] = d[2] = 0.0; return; }
  const PHYS *v = sv + (size_t)slot * 4;
  d[0] = double(v[0]); d[1] = double(v[1]); d[2] = double(v[2]);
}

// FFT form of the lagged sum (the O(N^2) loop of src/hawaii.c:2089-2094).  With
// a = d[0..N-1] and b = d[0..2N-2], zero-padded to L >= 2N - 1 (a power of two),
// C(s) = sum_c a[c] . b[c+s] is the circular cross-correlation of a and b for
// s < N (no term wraps), so with the transform F[k] = sum_j x_j e^{+2 pi i jk/L} of
// stockham_batch_kernel:
//   C(s) = (1/L) Re sum_k conj(P_k) e^{+2 pi i sk/L},  P_k = sum_comp conj(A_k) B_k.
//   1. zimm_pack: per trajectory and component the complex series a_j + i b_j
//      (zero for a dropped trajectory);
//   2. log2 L Stockham passes over 3 series per trajectory;
//   3. zimm_cross: A_k = (Z_k + conj Z_{L-k}) / 2, B_k = (Z_k - conj Z_{L-k}) / 2i, and
//      conj(P_k) per trajectory;
//   4. log2 L passes over one series per trajectory;
//   5. zimm_accum: C(s) += w Re(.)/L into each trajectory's C(t) slice.
// All transforms are FP64 on both precision paths.
template <typename PHYS>
__global__ void __launch_bounds__(256) zimm_pack_kernel(ZimmArgs a, int L, long long t0, long long m, double2 *z) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= 3 * m * L) return;
  const long long sr = i / L;
  const int j = (int)(i - sr * L);
  const long long t = t0 + sr / 3;
  const int comp = (int)(sr % 3);
  double av = 0.0, bv = 0.0;
  if (!a.failed[t] && j <= 2 * a.N - 2) {
    const PHYS *sv = static_cast<const PHYS *>(a.series) + (size_t)t * a.stride * 4;
    double d[3];
    zimm_d(sv, a.N, a.len[2 * t], a.len[2 * t + 1], j, d);
    bv = d[comp];
    if (j < a.N) av = d[comp];
  }
  z[i] = make_double2(av, bv);
}

__global__ void __launch_bounds__(256) zimm_cross_kernel(const double2 *Z, int L, long long m, double2 *pc) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m * L) return;
  const long long t = i / L;
  const int k = (int)(i - t * L);
  const int kr = (L - k) & (L - 1);
  double pr = 0.0, pi = 0.0;
  for (int c = 0; c < 3; ++c) {
    const double2 zk = Z[(3 * t + c) * L + k], zm = Z[(3 * t + c) * L + kr];
    const double ar = 0.5 * (zk.x + zm.x), ai = 0.5 * (zk.y - zm.y);
    const double br = 0.5 * (zk.y + zm.y), bi = -0.5 * (zk.x - zm.x);
    pr += ar * br + ai * bi;  // conj(A) B
    pi += ar * bi - ai * br;
  }
  pc[i] = make_double2(pr, -pi);
}

// grid: x over s < N, y over groups of 256 trajectories
__global__ void __launch_bounds__(256) zimm_accum_kernel(const double2 *R, int L, int N, long long m,
                                                         long long t_first, long long traj_per_iter, double w,
                                                         double *crln) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= N) return;
  const long long lo = (long long)blockIdx.y * 256, hi = min(m, lo + 256);
  long long slice = (t_first + lo) / traj_per_iter;
  double acc = 0.0;
  for (long long t = lo; t < hi; ++t) {
    const long long sl = (t_first + t) / traj_per_iter;
    if (sl != slice) {
      if (acc != 0.0) atomicAdd(&crln[slice * N + s], w * acc);
      acc = 0.0;
      slice = sl;
    }
    acc += R[t * L + s].x;
  }
  if (acc != 0.0) atomicAdd(&crln[slice * N + s], w * acc);
}

}  // namespace hh
