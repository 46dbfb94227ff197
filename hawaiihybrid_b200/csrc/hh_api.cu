// C ABI of libhh_cuda.so (include/hh_cuda.h): device context, buffers, the
// sampler rounds, the trajectory launch with its failure-compensation pass, the
// zeroth-moment integral and the CF->SF transform.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "../../include/hh_cuda.h"
#include "hh_ch4co2_dip.cuh"
#include "hh_ch4co2_tc.cuh"
#include "hh_ch4co2_fold.h"
#include "hh_co2ar_tables.h"
#include "hh_consts.h"
#include "hh_defer.cuh"
#include "hh_fft.cuh"
#include "hh_internal.h"
#include "hh_m0.cuh"
#include "hh_prmu.cuh"
#include "hh_traj.cuh"
#include "hh_vegas.cuh"

namespace hh {
// 8 independent FMA chains per thread; the loop body is 8 FMAs = 16 flops
template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *out, int iters, T a, T b) {
  T v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = T(threadIdx.x + i) * T(1e-3);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = v[i] * a + b;
  }
  T s = v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6] + v[7];
  if (s == T(-12345.678)) out[threadIdx.x] = s;  // keeps the chains alive
}
}  // namespace hh

namespace {

using namespace hh;

char g_errmsg[512] = "";

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      snprintf(g_errmsg, sizeof g_errmsg, "%s:%d %s: %s", __FILE__, __LINE__, #call, \
               cudaGetErrorString(e_));                                              \
      return HH_E_CUDA;                                                              \
    }                                                                                \
  } while (0)

template <typename T> struct DevBuf {
  T *p = nullptr;
  size_t cap = 0;
  // exactly n elements when it grows (several buffers hold gigabytes; callers that
  // expect growth ask for their own headroom)
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, n * sizeof(T));
    if (e == cudaSuccess) cap = n;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct TrajTune {
  int warps;        // bulk kernel warps per block
  int handoff_div;  // hand-off when at most (solo warp slots) / handoff_div items are open
};

struct Ctx {
  bool init = false;
  int device = -1;
  int sys = 0;
  double mu = 0.0, II = 0.0;
  int QP = 0, D = 0;
  cudaStream_t st = nullptr;
  // [0, 1]: call; [2, 3]: trajectory launches; [4, 5]: autotuner timing runs;
  // [6, 7]: per-kernel timer (hh_cuda_debug_kernel_ms)
  cudaEvent_t ev[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // side stream that generates the MT19937 words of the next call while this
  // call's trajectories run
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_sampled = nullptr, ev_pregen = nullptr;
  bool pregen_pending = false;
  // deferred samples: the contexts the bulk trajectory kernel wrote are evaluated on
  // st3 (lowest priority; st has the highest) while the solo kernel runs; ev_bulk
  // follows the snapshot of their count, ev_eval1 the first sample launch
  cudaStream_t st3 = nullptr;
  cudaEvent_t ev_bulk = nullptr, ev_eval1 = nullptr;
  bool bulk_snap = false;  // the last trajectory launch snapshotted its context count
  int num_sms = 0;
  Co2arTablesGlobal *d_tab = nullptr;
  N2arDipFold *d_n2ar_fold = nullptr;  // N2-Ar dipole models, folded (hh_n2ar_fold.h)
  N2arPesNet<double> *d_n2ar_pes_d = nullptr;  // N2-Ar PES network, FP64 and FP32
  N2arPesNet<float> *d_n2ar_pes_f = nullptr;
  float4 *d_n2ar_tab = nullptr;  // N2-Ar mixed-path dipole table (hh_n2ar.cuh), built on the device
  // CH4-CO2: rotor moments, stand-in surface constants, folded dipole table
  SamplerExtra sx{};
  double2 *d_ch4_cd = nullptr;
  float4 *d_ch4_cf = nullptr;
  unsigned int *d_ch4_y2 = nullptr;
  unsigned int *d_ch4_meta = nullptr;
  int ch4_B = 0;
  int ch4_groups = 0;  // (Y1, component, cos/sin) groups of the batch stream
  unsigned char *d_ch4_tc = nullptr;  // coefficient images of the tensor-core dipole kernel
  int *d_ch4_tc_err = nullptr;        // set by that kernel when an mbarrier wait gave up
  int ch4_dip_s[2] = {0, 0};  // records per lane of the dipole kernel [FP64, mixed]; 0: not tuned yet
  hh_requantization req{};  // PR_MU requantization of monomer 1 (hh_cuda_set_requantization)
  // trajectory launch picks per [system][FP64, mixed] (warps == 0: not tuned yet)
  TrajTune traj_tune[5][2] = {};
  DevBuf<double> tune_crln, tune_cnt;  // the autotuner's scratch C(t) and counters
  // MT19937 stream
  uint32_t *d_mt = nullptr;
  unsigned short *d_mt_jump_seg = nullptr, *d_mt_jump_coarse = nullptr;  // jump-ahead tables
  DevBuf<uint32_t> mt_seg_states;
  DevBuf<uint32_t> words[2];
  int cur = 0;
  long long wbase = 0, wvalid = 0, wpos = 0;
  double p_accept = 0.25;
  // sampler scratch
  DevBuf<unsigned char> accept, consumed;
  DevBuf<double> qp_cand, energy, qp0;
  DevBuf<unsigned int> block_counts;
  DevBuf<long long> cand_idx;
  DevBuf<unsigned long long> scal;  // [0] first_irregular, [1] total
  // trajectories
  DevBuf<double> crln;
  DevBuf<unsigned long long> counters;
  DevBuf<unsigned int> status_hist, queue;
  DevBuf<int> fail_flag, fail_list, fail_count, items;
  DevBuf<unsigned char> handoff;   // open items handed from the bulk to the solo kernel
  DevBuf<unsigned int> hcount;     // n_handoff, solo cursor, closed items
  DevBuf<uint4> trace;
  // deferred samples (hh_defer.cuh): contexts and their count (+ the largest count of a
  // call's launches), first/last sample value per context, per-item state
  DevBuf<unsigned char> dctx, dvals, item_mu0;
  DevBuf<unsigned long long> dcount;
  DevBuf<int> item_status;
  DevBuf<unsigned> item_fail;
  DevBuf<unsigned char> istart;  // precomputed item starts (ItemStart per item)
  double defer_est = 32.0;  // contexts per item, from the previous calls
  // CORRELATION_ARRAY weights [n][n_sat]: with ratios (C(t)) and without (nstar)
  DevBuf<double> sat_w, sat_wraw;
  // CH4-CO2 record path: sample records, their dipoles, the piece sort
  DevBuf<unsigned char> rec, rec_mu;
  DevBuf<int> rec_len, rec_status, rec_sorted;
  DevBuf<unsigned int> seg_cnt;
  DevBuf<long long> seg_w0;
  DevBuf<unsigned long long> rec_nfail;
  DevBuf<int> zim_fail;  // Zimmermann estimate on the record path: dropped trajectories
  // PR_MU: complex series (two buffers) and the spectrum
  DevBuf<double2> pm_a, pm_b;
  DevBuf<double2> zf_a, zf_b;   // Zimmermann FFT workspace
  DevBuf<double> pm_sf;
  // M0
  DevBuf<double> m0_partials, m0_out;
  // VEGAS: grid edges, block sums, per-bin sums of F^2
  DevBuf<double> vg_edges, vg_sums, vg_hist;
  // FFT, and the CUDA graph of its kernel sequence for the current (N, dt, buffers)
  DevBuf<double> f_cf, f_nu, f_sf;
  DevBuf<double2> f_a, f_b;
  cudaGraphExec_t idct_exec = nullptr;
  size_t idct_N = 0;
  double idct_dt = 0.0;
  const void *idct_bufs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

Ctx g;
unsigned long long g_launches = 0;  // kernel launches of the current call

// per-kernel-class device time (hh_cuda_debug_kernel_ms): when on, kt_begin /
// kt_end bracket a launch with events and wait for it
struct KernelTimer {
  bool on = false;
  double ms[HH_KT_COUNT] = {};
  unsigned long long n[HH_KT_COUNT] = {};
};
KernelTimer g_kt;
inline void kt_begin() {
  if (g_kt.on) cudaEventRecord(g.ev[6], g.st);
}
inline void kt_end(int cls) {
  if (!g_kt.on) return;
  cudaEventRecord(g.ev[7], g.st);
  cudaEventSynchronize(g.ev[7]);
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, g.ev[6], g.ev[7]) == cudaSuccess) {
    g_kt.ms[cls] += ms;
    g_kt.n[cls] += 1;
  }
}
int g_inject_item = -1, g_inject_k = -1, g_inject_status = 0;
uint32_t *g_trace_host = nullptr;  // registered by hh_cuda_debug_item_trace for the next call
uint64_t g_trace_cap = 0;

bool g_co2ar_dip_exp = false;  // a CO2-Ar dipole interval with exponential terms
void build_tables(Co2arTablesGlobal *t) {
  memcpy(t->pes, hh_co2ar_pes, sizeof(t->pes));
  memcpy(t->dipx, hh_co2ar_dipx, sizeof(t->dipx));
  memcpy(t->dipz, hh_co2ar_dipz, sizeof(t->dipz));
  for (int i = 0; i < CO2AR_NINT; ++i) {
    t->rbound[i] = (i < CO2AR_NINT - 1) ? hh_co2ar_rbound[i] : 1e300;
    t->rlo[i] = hh_co2ar_rlo[i];
    int fp = 0, fd = 0;
    for (int l = 0; l < CO2AR_NL; ++l) {
      const double *rp = hh_co2ar_pes[i][l];
      const double *rx = hh_co2ar_dipx[i][l];
      const double *rz = hh_co2ar_dipz[i][l];
      for (int k = 4; k < 8; ++k) {
        if (rp[k] != 0.0) fp |= 1;
        if (rx[k] != 0.0 || rz[k] != 0.0) fd |= 1;
      }
      if (rp[8] != 0.0) fp |= 2;
      if (rx[8] != 0.0 || rz[8] != 0.0) fd |= 2;
    }
    t->fpes[i] = fp;
    t->fdip[i] = fd;
    if (fd & 2) g_co2ar_dip_exp = true;
  }
}

int check_params(const hh_calc_params *p) {
  if (!p) return HH_E_INVALID_ARGUMENT;
  if (!(p->sampler_Rmin > 0) || !(p->sampler_Rmax > p->sampler_Rmin)) return HH_E_INVALID_ARGUMENT;
  if (!(p->sampling_time > 0) || p->MaxTrajectoryLength < 1) return HH_E_INVALID_ARGUMENT;
  if (!(p->Rcut > 0) || !(p->cvode_tolerance > 0)) return HH_E_INVALID_ARGUMENT;
  if (p->pair_state < 1 || p->pair_state > 3) return HH_E_INVALID_ARGUMENT;
  if (p->MaxTrajectoryLength > (size_t)INT32_MAX) return HH_E_INVALID_ARGUMENT;
  if (p->use_zimmermann_trick && p->pair_state != HH_PAIR_STATE_BOUND) return HH_E_INVALID_ARGUMENT;
  return HH_OK;
}

// blocks a request of nblk blocks generates: long requests go by whole segments
long long mt_round_blocks(long long nblk) {
  return nblk >= 2 * MT_SEG_BLOCKS ? (nblk + MT_SEG_BLOCKS - 1) / MT_SEG_BLOCKS * MT_SEG_BLOCKS : nblk;
}

// nblk (from mt_round_blocks) blocks of the stream into out, on stream s
int gen_blocks(uint32_t *out, long long nblk, cudaStream_t s) {
  if (nblk >= 2 * MT_SEG_BLOCKS) {
    const int nseg = (int)(nblk / MT_SEG_BLOCKS);
    CK(g.mt_seg_states.ensure((size_t)nseg * MT_N));
    CK(launch_mt_generate_segments(g.d_mt, out, nseg, g.mt_seg_states.p, g.d_mt_jump_seg, g.d_mt_jump_coarse, s));
    g_launches += 4;
  } else {
    CK(launch_mt_generate(g.d_mt, out, nblk, s));
    g_launches += 1;
  }
  return HH_OK;
}

// make words [wpos, need_end) resident in words[cur]
int ensure_words(long long need_end) {
  if (g.wbase <= g.wpos && g.wbase + g.wvalid >= need_end) return HH_OK;
  long long end_old = g.wbase + g.wvalid;
  long long left = std::max(0LL, end_old - g.wpos);
  long long gen = need_end - (g.wpos + left);
  long long nblk = mt_round_blocks((gen + MT_N - 1) / MT_N + 1);
  int nxt = 1 - g.cur;
  CK(g.words[nxt].ensure((size_t)(left + nblk * MT_N)));
  if (left) {
    CK(cudaMemcpyAsync(g.words[nxt].p, g.words[g.cur].p + (g.wpos - g.wbase),
                       (size_t)left * sizeof(uint32_t), cudaMemcpyDeviceToDevice, g.st));
  }
  int rc = gen_blocks(g.words[nxt].p + left, nblk, g.st);
  if (rc) return rc;
  g.cur = nxt;
  g.wbase = g.wpos;
  g.wvalid = left + nblk * MT_N;
  return HH_OK;
}

// the main stream waits for words generated ahead on the side stream (they and
// the generator state are read or rewritten next)
int join_pregen() {
  if (g.pregen_pending) {
    CK(cudaStreamWaitEvent(g.st, g.ev_pregen, 0));
    g.pregen_pending = false;
  }
  return HH_OK;
}

// After a call's sampling: generate, on the side stream, the next n words of the
// stream, the ones the next call of the same size will consume.  They are the
// words ensure_words would produce later; generating them now overlaps the
// sequential MT19937 refresh with this call's trajectories.
int pregen_words(long long n) {
  n = std::min(n, 1LL << 26);
  if (n <= 0 || g.pregen_pending) return HH_OK;
  const long long need_end = g.wpos + n;
  if (g.wbase <= g.wpos && g.wbase + g.wvalid >= need_end) return HH_OK;
  const long long end_old = g.wbase + g.wvalid;
  const long long left = std::max(0LL, end_old - g.wpos);
  const long long gen = need_end - (g.wpos + left);
  const long long nblk = mt_round_blocks((gen + MT_N - 1) / MT_N + 1);
  const int nxt = 1 - g.cur;
  CK(g.words[nxt].ensure((size_t)(left + nblk * MT_N)));
  CK(cudaEventRecord(g.ev_sampled, g.st));
  CK(cudaStreamWaitEvent(g.st2, g.ev_sampled, 0));
  if (left) {
    CK(cudaMemcpyAsync(g.words[nxt].p, g.words[g.cur].p + (g.wpos - g.wbase),
                       (size_t)left * sizeof(uint32_t), cudaMemcpyDeviceToDevice, g.st2));
  }
  int rc = gen_blocks(g.words[nxt].p + left, nblk, g.st2);
  if (rc) return rc;
  CK(cudaEventRecord(g.ev_pregen, g.st2));
  g.pregen_pending = true;
  g.cur = nxt;
  g.wbase = g.wpos;
  g.wvalid = left + nblk * MT_N;
  return HH_OK;
}

int reseed(uint32_t seed) {
  int rc = join_pregen();
  if (rc) return rc;
  CK(launch_mt_seed(seed, g.d_mt, g.st));
  g.wbase = g.wvalid = g.wpos = 0;
  return HH_OK;
}

// draw n accepted phase points into d_out (device), in the reference's order
int sample_into(const hh_calc_params *p, double T, uint64_t n, double *d_out, uint64_t *ncand_out) {
  uint64_t got = 0, ncand_total = 0;
  int jrc = join_pregen();
  if (jrc) return jrc;
  CK(g.cand_idx.ensure(std::max<uint64_t>(n, 1)));
  CK(g.scal.ensure(4));
  while (got < n) {
    long long remaining = (long long)(n - got);
    double pe = std::max(g.p_accept, 0.01);
    long long ncand = (long long)(remaining / pe * 1.15) + 4096;
    ncand = std::min(std::max(ncand, 65536LL), 1LL << 23);
    int rc = ensure_words(g.wpos + ncand * g.D + 4096);
    if (rc) return rc;
    CK(g.accept.ensure(ncand));
    CK(g.consumed.ensure(ncand));
    CK(g.qp_cand.ensure((size_t)ncand * g.QP));
    CK(g.energy.ensure(ncand));
    CK(g.block_counts.ensure((ncand + 1023) / 1024 + 1));
    CK(cudaMemsetAsync(g.scal.p, 0xff, sizeof(unsigned long long), g.st));
    CK(launch_candidates(g.sys, g.mu, g.II, T, p->sampler_Rmin, p->sampler_Rmax, p->pesmin,
                         p->pair_state, g.d_tab, g.words[g.cur].p, g.wvalid, g.wpos - g.wbase, g.D,
                         ncand, g.accept.p, g.consumed.p, g.qp_cand.p, g.energy.p, g.scal.p,
                         g.sx, g.st));
    g_launches += 1;
    unsigned long long first_irr = 0;
    CK(cudaMemcpyAsync(&first_irr, g.scal.p, sizeof first_irr, cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    long long limit = (first_irr == ~0ULL) ? ncand - 1 : (long long)first_irr;
    CK(launch_compact(g.accept.p, g.qp_cand.p, ncand, limit, g.QP, (long long)got, (long long)n,
                      d_out, g.cand_idx.p, g.block_counts.p, g.scal.p + 1, g.st));
    g_launches += 3;
    unsigned long long total = 0;
    CK(cudaMemcpyAsync(&total, g.scal.p + 1, sizeof total, cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    long long take = std::min<long long>((long long)total, remaining);
    long long E;
    if (take == remaining && take > 0) {
      long long last = 0;
      CK(cudaMemcpy(&last, g.cand_idx.p + got + take - 1, sizeof last, cudaMemcpyDeviceToHost));
      E = last;
    } else {
      E = limit;
    }
    int usedE = g.D;
    if (first_irr != ~0ULL && E == (long long)first_irr) {
      unsigned char cE = 0;
      CK(cudaMemcpy(&cE, g.consumed.p + E, 1, cudaMemcpyDeviceToHost));
      if (cE == 0) {
        snprintf(g_errmsg, sizeof g_errmsg, "sampler ran past the generated stream");
        return HH_E_SAMPLER;
      }
      usedE = cE;
    }
    g.wpos += E * g.D + usedE;
    ncand_total += (uint64_t)(E + 1);
    got += (uint64_t)take;
    if (got < n && ncand_total > 20000000000ULL) {
      snprintf(g_errmsg, sizeof g_errmsg,
               "sampler: %llu of %llu phase points accepted after %llu candidates (acceptance too low)",
               (unsigned long long)got, (unsigned long long)n, (unsigned long long)ncand_total);
      return HH_E_SAMPLER;
    }
    g.p_accept = std::max(1.0, (double)total) / double(limit + 1);
  }
  if (ncand_out) *ncand_out = ncand_total;
  return HH_OK;
}

// HH_DEFER_OVERLAP (default 1; 0 off): with deferred samples, the contexts of the bulk
// trajectory kernel are evaluated while the solo kernel runs
int g_defer_overlap = [] {
  const char *e = getenv("HH_DEFER_OVERLAP");
  return e ? atoi(e) : 1;
}();

// One trajectory launch: the bulk kernel (WARPS warps per block) until at most
// cap / handoff_div items are open, then the solo kernel for the rest, where cap is
// the solo kernel's warp slots.  With ev_split, events ev[4] (start), ev[5] (after the
// bulk kernel) and ev[7] (end) are recorded for the autotuner.
template <int SYS, typename PHYS, typename STG, bool COMP, int WARPS, bool REQ = false>
int launch_traj_w(const TrajParams &P, const TrajIO &io, int handoff_div, bool ev_split) {
  auto kern = traj_kernel<SYS, PHYS, STG, COMP, false, WARPS, REQ>;
  const size_t smem = traj_smem_bytes<SYS, PHYS, STG, WARPS>();
  if (smem > 48 * 1024) CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  constexpr int THREADS = 32 * WARPS;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem));
  int grid = std::max(1, per_sm) * g.num_sms;
  long long need = (io.n_items + THREADS - 1) / THREADS;
  if (need < grid) grid = (int)std::max(1LL, need);
  // the last open items (and all items of a launch that small) run one per warp
  // in the solo kernel, one state component per lane
  auto solo = traj_kernel<SYS, PHYS, STG, COMP, true, traj_warps<PHYS>(), REQ>;
  constexpr int SOLO_THREADS = traj_threads<PHYS>();
  const size_t smem_solo = traj_smem_bytes<SYS, PHYS, STG>();
  if (smem_solo > 48 * 1024)
    CK(cudaFuncSetAttribute(solo, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_solo));
  int per_sm_solo = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_solo, solo, SOLO_THREADS, smem_solo));
  const int solo_grid = std::max(1, per_sm_solo) * g.num_sms;
  const unsigned cap = (unsigned)solo_grid * (SOLO_THREADS / 32);
  constexpr int NS = SYS == SYS_HEAR ? 6 : SYS == SYS_CH4CO2 ? 19 : 12;
  CK(g.handoff.ensure((size_t)cap * sizeof(HandoffState<NS, PHYS, STG>)));
  CK(g.hcount.ensure(4));
  CK(cudaMemsetAsync(g.hcount.p, 0, 4 * sizeof(unsigned int), g.st));
  TrajIO io2 = io;
  io2.handoff = g.handoff.p;
  io2.n_handoff = g.hcount.p;
  io2.solo_cursor = g.hcount.p + 1;
  io2.done = g.hcount.p + 2;
  io2.handoff_at = std::max(1u, cap / (unsigned)std::max(1, handoff_div));
  if (ev_split) CK(cudaEventRecord(g.ev[4], g.st));
  g.bulk_snap = false;
  if ((unsigned)io.n_items > cap) {
    kt_begin();
    kern<<<grid, THREADS, smem, g.st>>>(P, io2, g.d_tab);
    CK(cudaGetLastError());
    kt_end(HH_KT_TRAJ_BULK);
    g_launches += 1;
    // deferred samples: the count of the contexts the bulk kernel wrote, for the first
    // sample launch beside the solo kernel (not while kernels are timed one by one)
    if (io.ctx && g_defer_overlap && !g_kt.on) {
      defer_snapshot_kernel<<<1, 1, 0, g.st>>>(io.ctx_count);
      CK(cudaGetLastError());
      CK(cudaEventRecord(g.ev_bulk, g.st));
      g.bulk_snap = true;
      g_launches += 1;
    }
  }
  if (ev_split) CK(cudaEventRecord(g.ev[5], g.st));
  kt_begin();
  solo<<<solo_grid, SOLO_THREADS, smem_solo, g.st>>>(P, io2, g.d_tab);
  CK(cudaGetLastError());
  kt_end(HH_KT_TRAJ_SOLO);
  g_launches += 1;
  if (ev_split) CK(cudaEventRecord(g.ev[7], g.st));
  return HH_OK;
}

template <int SYS, typename PHYS, typename STG, bool COMP>
int launch_traj_pick(const TrajParams &P, const TrajIO &io, int warps, int handoff_div, bool ev_split) {
  if (warps == TRAJ_WARPS_CANDIDATES[0])
    return launch_traj_w<SYS, PHYS, STG, COMP, TRAJ_WARPS_CANDIDATES[0]>(P, io, handoff_div, ev_split);
  return launch_traj_w<SYS, PHYS, STG, COMP, TRAJ_WARPS_CANDIDATES[1]>(P, io, handoff_div, ev_split);
}

// Autotuner of the trajectory launch (first large plain-C(t) call per system and
// precision): the bulk kernel's warps per block and the hand-off threshold (how many
// open items are left to the solo kernel, i.e. when the launch switches from 32
// trajectories per warp to one).  Timed on the launch's first items, into scratch
// C(t) and counters, so the call's own results are untouched:
//   1. each warps-per-block candidate with the full hand-off threshold: bulk kernel time;
//   2. with the faster shape, thresholds cap / 2 and cap / 4 against cap: launch time.
// HH_TRAJ_WARPS (4 or 8) and HH_TRAJ_HANDOFF_DIV (1, 2 or 4) fix a choice instead.
constexpr int TRAJ_TUNE_MIN_ITEMS = 16384;  // smaller launches use the defaults, untuned
constexpr int TRAJ_TUNE_ITEMS = 32768;      // items the timing runs integrate

template <int SYS, typename PHYS, typename STG, bool COMP>
int tune_traj(const TrajParams &P, const TrajIO &io, TrajTune *out) {
  const char *ew = getenv("HH_TRAJ_WARPS");
  const char *ed = getenv("HH_TRAJ_HANDOFF_DIV");
  int fixed_w = ew ? atoi(ew) : 0, fixed_d = ed ? atoi(ed) : 0;
  if (fixed_w != TRAJ_WARPS_CANDIDATES[0] && fixed_w != TRAJ_WARPS_CANDIDATES[1]) fixed_w = 0;
  if (fixed_d != 1 && fixed_d != 2 && fixed_d != 4) fixed_d = 0;
  const int n_s = std::min(io.n_items, TRAJ_TUNE_ITEMS);
  const int nsl = std::max(1, io.n_sat);
  CK(g.tune_crln.ensure((size_t)P.N * nsl));
  CK(g.tune_cnt.ensure(16 + 2 * HH_ST_COUNT + 1));
  TrajIO t = io;
  t.n_items = n_s;
  t.items = nullptr;
  t.crln = g.tune_crln.p;
  t.counters = reinterpret_cast<unsigned long long *>(g.tune_cnt.p);
  t.status_hist = reinterpret_cast<unsigned int *>(g.tune_cnt.p + 8);
  t.queue = reinterpret_cast<unsigned int *>(g.tune_cnt.p + 8 + HH_ST_COUNT);
  t.fail_flag = nullptr;
  t.fail_list = nullptr;
  t.fail_count = nullptr;
  t.traj_per_iter = LLONG_MAX / 4;  // every sampled item into the one scratch slice
  t.item_trace = nullptr;
  TrajParams Pt = P;
  Pt.inject_item = -1;
  auto run = [&](int w, int d, float *bulk_ms, float *all_ms) -> int {
    CK(cudaMemsetAsync(g.tune_cnt.p, 0, (16 + 2 * HH_ST_COUNT + 1) * sizeof(double), g.st));
    if (t.ctx_count) CK(cudaMemsetAsync(t.ctx_count, 0, sizeof(unsigned long long), g.st));
    CK(cudaMemsetAsync(g.tune_crln.p, 0, (size_t)P.N * nsl * sizeof(double), g.st));
    int rc = launch_traj_pick<SYS, PHYS, STG, COMP>(Pt, t, w, d, true);
    if (rc) return rc;
    CK(cudaEventSynchronize(g.ev[7]));
    CK(cudaEventElapsedTime(bulk_ms, g.ev[4], g.ev[5]));
    CK(cudaEventElapsedTime(all_ms, g.ev[4], g.ev[7]));
    return HH_OK;
  };
  float bulk, all;
  int w_best = fixed_w ? fixed_w : traj_warps<PHYS>();
  if (!fixed_w) {
    float best = 0.f;
    for (int c = 0; c < 2; ++c) {
      const int w = TRAJ_WARPS_CANDIDATES[c];
      int rc = run(w, 1, &bulk, &all);
      if (rc) return rc;
      if (c == 0 || bulk < best) {
        best = bulk;
        w_best = w;
      }
    }
  }
  int d_best = fixed_d ? fixed_d : 1;
  if (!fixed_d) {
    float best = 0.f;
    for (int d : {1, 2, 4}) {
      int rc = run(w_best, d, &bulk, &all);
      if (rc) return rc;
      if (d == 1 || all < best) {
        best = all;
        d_best = d;
      }
    }
  }
  // the timing runs' sample contexts are scratch
  if (t.ctx_count) CK(cudaMemsetAsync(t.ctx_count, 0, sizeof(unsigned long long), g.st));
  out->warps = w_best;
  out->handoff_div = d_best;
  return HH_OK;
}

template <int SYS, typename PHYS, typename STG, bool COMP>
int launch_traj(const TrajParams &P, const TrajIO &io, int *grid_out) {
  (void)grid_out;
  TrajTune &tt = g.traj_tune[SYS][sizeof(PHYS) == 4 ? 1 : 0];
  const bool plain = !io.records && !io.series;
  if (tt.warps == 0 && plain && io.n_items >= TRAJ_TUNE_MIN_ITEMS) {
    int rc = tune_traj<SYS, PHYS, STG, COMP>(P, io, &tt);
    if (rc) return rc;
  }
  const int w = tt.warps ? tt.warps : traj_warps<PHYS>();
  const int d = tt.handoff_div ? tt.handoff_div : 1;
  return launch_traj_pick<SYS, PHYS, STG, COMP>(P, io, w, d, false);
}

// PR_MU with requantization: the REQ kernels of the linear-monomer systems
int run_traj_dispatch_req(int precision, const TrajParams &P, const TrajIO &io) {
  const bool mixed = precision == HH_PRECISION_MIXED;
  if (g.sys == SYS_N2AR) {
    TrajIO io2 = io;
    io2.dipnet = g.d_n2ar_fold;
    io2.pesnet = mixed ? (const void *)g.d_n2ar_pes_f : (const void *)g.d_n2ar_pes_d;
    io2.diptab = mixed ? g.d_n2ar_tab : nullptr;
    return mixed ? launch_traj_w<SYS_N2AR, float, float, false, traj_warps<float>(), true>(P, io2, 1, false)
                 : launch_traj_w<SYS_N2AR, double, double, false, traj_warps<double>(), true>(P, io2, 1, false);
  }
  if (g.sys == SYS_CO2AR)
    return mixed ? launch_traj_w<SYS_CO2AR, float, float, false, traj_warps<float>(), true>(P, io, 1, false)
                 : launch_traj_w<SYS_CO2AR, double, double, false, traj_warps<double>(), true>(P, io, 1, false);
  return HH_E_UNSUPPORTED_SYSTEM;
}

int run_traj_dispatch(int precision, const TrajParams &P, const TrajIO &io) {
  if (g.sys == SYS_HEAR) {
    if (precision == HH_PRECISION_MIXED) return launch_traj<SYS_HEAR, float, float, false>(P, io, nullptr);
    return launch_traj<SYS_HEAR, double, double, false>(P, io, nullptr);
  }
  if (g.sys == SYS_N2AR) {
    TrajIO io2 = io;
    io2.dipnet = g.d_n2ar_fold;
    if (precision == HH_PRECISION_MIXED) {
      io2.pesnet = g.d_n2ar_pes_f;
      io2.diptab = g.d_n2ar_tab;
      return launch_traj<SYS_N2AR, float, float, false>(P, io2, nullptr);
    }
    io2.pesnet = g.d_n2ar_pes_d;
    io2.diptab = nullptr;
    return launch_traj<SYS_N2AR, double, double, false>(P, io2, nullptr);
  }
  // plain FP32 sums: compensation does not reduce the FP32 error of the surfaces,
  // which comes from the radial rows, and cost 12 % of the kernel's time
  if (precision == HH_PRECISION_MIXED) return launch_traj<SYS_CO2AR, float, float, false>(P, io, nullptr);
  return launch_traj<SYS_CO2AR, double, double, false>(P, io, nullptr);
}

// ---------------------------------------------------------------------------
// deferred samples (hh_defer.cuh)
// ---------------------------------------------------------------------------
// the mixed path's plain C(t) of the systems with a surface dipole; records, series,
// satellite temperatures, PR_MU and a failure injection with a soft status keep
// in-kernel samples.  g_defer (hh_cuda_debug_set_defer; environment HH_DEFER_SAMPLES,
// default 1): 0 in-kernel samples for every call, 1 deferred for CO2-Ar, 2 also N2-Ar.
using DeferCtx = SampleCtx<float, 6>;
constexpr size_t DEFER_CTX_BYTES = sizeof(DeferCtx) + 2 * sizeof(float);  // + first/last value
int g_defer = [] {
  const char *e = getenv("HH_DEFER_SAMPLES");
  return e ? atoi(e) : 1;
}();
bool defer_eligible(int precision, const TrajParams &P, const TrajIO &io) {
  // the CO2-Ar sample kernel evaluates dipole intervals without exponential terms
  const bool sys_ok = g.sys == SYS_CO2AR ? g_defer >= 1 && !g_co2ar_dip_exp : (g.sys == SYS_N2AR && g_defer >= 2);
  return sys_ok && precision == HH_PRECISION_MIXED && io.n_sat == 0 && !io.series && !io.records && !P.prmu &&
         (P.inject_item < 0 || P.inject_status >= HH_ST_NAN_DIPOLE);
}

// the sample kernels for the contexts of the launch just made with io; n_items and
// items as io's; traj_base: io.ic's first trajectory in the call (for the fail list)
template <int SYS>
int run_deferred_sys(const TrajParams &P, const TrajIO &io, long long traj_base) {
  DeferArgs a;
  memset(&a, 0, sizeof a);
  a.ctx = io.ctx;
  a.ctx_count = io.ctx_count;
  a.ctx_cap = io.ctx_cap;
  a.items = io.items;
  a.n_items = io.n_items;
  a.item_status = io.item_status;
  a.item_mu0 = io.item_mu0;
  a.item_fail = g.item_fail.p + 2 * traj_base;
  a.first_v = g.dvals.p;
  a.last_v = g.dvals.p + io.ctx_cap * sizeof(float);
  a.crln = io.crln;
  a.traj_per_iter = io.traj_per_iter;
  a.inv_traj_per_iter = 1.0 / double(io.traj_per_iter);
  a.status_hist = io.status_hist;
  a.fail_flag = io.fail_flag;
  a.fail_list = io.fail_list;
  a.fail_count = io.fail_count;
  a.traj_base = traj_base;
  a.peak = g.dcount.p + DEFER_PEAK;
  auto eval = SYS == SYS_CO2AR ? defer_eval_co2ar_kernel<float, float> : defer_eval_kernel<SYS_N2AR, float, float>;
  const size_t smem = DeferSys<SYS, float, float>::smem();
  if (smem > 48 * 1024) CK(cudaFuncSetAttribute(eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  constexpr int threads = defer_eval_threads<SYS>();
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eval, threads, smem));
  const int grid = std::max(1, per_sm) * g.num_sms;
  unsigned long long *cnt = io.ctx_count;
  kt_begin();
  if (g.bulk_snap) {
    // the bulk kernel's contexts on st3 beside the solo kernel (whose blocks st's
    // priority places first), the solo kernel's after it on st
    DeferArgs a1 = a;
    a1.ctx_hi = cnt + DEFER_SNAP;
    CK(cudaStreamWaitEvent(g.st3, g.ev_bulk, 0));
    eval<<<grid, threads, smem, g.st3>>>(a1, P, io, g.d_tab);
    CK(cudaGetLastError());
    CK(cudaEventRecord(g.ev_eval1, g.st3));
    DeferArgs a2 = a;
    a2.ctx_lo = cnt + DEFER_SNAP;
    eval<<<grid, threads, smem, g.st>>>(a2, P, io, g.d_tab);
    CK(cudaGetLastError());
    CK(cudaStreamWaitEvent(g.st, g.ev_eval1, 0));
    g.bulk_snap = false;
    g_launches += 1;
  } else {
    eval<<<grid, threads, smem, g.st>>>(a, P, io, g.d_tab);
    CK(cudaGetLastError());
  }
  defer_jump_kernel<float, float, 6><<<8 * g.num_sms, DEFER_THREADS, 0, g.st>>>(a, P);
  CK(cudaGetLastError());
  defer_items_kernel<float><<<(unsigned)std::max(1, (io.n_items + DEFER_THREADS - 1) / DEFER_THREADS),
                              DEFER_THREADS, 0, g.st>>>(a, P);
  CK(cudaGetLastError());
  kt_end(HH_KT_SAMPLES);
  g_launches += 3;
  return HH_OK;
}

// the launch's item starts (mixed path: CO2-Ar, CH4-CO2) into buf, which then backs
// io.setup
using DeferStart = ItemStart<12, float, float>;
using Ch4Start = ItemStart<19, float, float>;
int run_item_starts(const TrajParams &P, TrajIO &io, unsigned char *buf) {
  if (g.sys != SYS_CO2AR && g.sys != SYS_N2AR && g.sys != SYS_CH4CO2) return HH_OK;
  TrajIO is = io;
  auto k = item_start_kernel<SYS_CH4CO2, float, float>;
  size_t smem = 0;
  if (g.sys == SYS_CO2AR) {
    k = item_start_kernel<SYS_CO2AR, float, float>;
    smem = smem_tables_bytes<float>();
  } else if (g.sys == SYS_N2AR) {
    // the mixed path's networks, as run_traj_dispatch gives them
    k = item_start_kernel<SYS_N2AR, float, float>;
    smem = sizeof(N2arDipFold) + sizeof(N2arPesNet<float>);
    is.dipnet = g.d_n2ar_fold;
    is.pesnet = g.d_n2ar_pes_f;
    is.diptab = g.d_n2ar_tab;
  }
  if (smem > 48 * 1024) CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, smem));
  const int grid = std::max(1, std::min(per_sm * g.num_sms, (io.n_items + 255) / 256));
  kt_begin();
  k<<<grid, 256, smem, g.st>>>(P, is, g.d_tab, buf);
  CK(cudaGetLastError());
  kt_end(HH_KT_ITEM_START);
  g_launches += 1;
  io.setup = buf;
  return HH_OK;
}

int run_deferred(const TrajParams &P, const TrajIO &io, long long traj_base) {
  if (g.sys == SYS_N2AR) {
    TrajIO io2 = io;
    io2.dipnet = g.d_n2ar_fold;
    io2.diptab = g.d_n2ar_tab;
    return run_deferred_sys<SYS_N2AR>(P, io2, traj_base);
  }
  return run_deferred_sys<SYS_CO2AR>(P, io, traj_base);
}

// device memory the CH4-CO2 record path may hold for one chunk of trajectories
constexpr size_t CH4_RECORD_BUDGET = size_t(24) << 30;
// FFT workspace of the Zimmermann estimate (two buffers)
constexpr size_t ZIMM_FFT_BUDGET = size_t(2) << 30;

// Zimmermann lagged sums of the za.n_traj trajectories whose dipole series are in
// za.series, by batched FFT cross-correlation (hh_ch4co2_dip.cuh), in sub-chunks
// whose transforms fit ZIMM_FFT_BUDGET
template <typename PHYS>
int zimm_fft(const ZimmArgs &za) {
  const int N = za.N;
  int L = 1;
  while (L < 2 * N - 1) L <<= 1;
  const size_t per = 3 * (size_t)L * sizeof(double2);
  const long long m = std::max<long long>(1, std::min<long long>(za.n_traj, (long long)(ZIMM_FFT_BUDGET / (2 * per))));
  CK(g.zf_a.ensure(3 * (size_t)m * L));
  CK(g.zf_b.ensure(3 * (size_t)m * L));
  const int passes = __builtin_ctz((unsigned)L);
  for (long long t0 = 0; t0 < za.n_traj; t0 += m) {
    const long long mm = std::min<long long>(m, za.n_traj - t0);
    zimm_pack_kernel<PHYS><<<(unsigned)((3 * mm * L + 255) / 256), 256, 0, g.st>>>(za, L, t0, mm, g.zf_a.p);
    CK(cudaGetLastError());
    double2 *x = g.zf_a.p, *y = g.zf_b.p;
    for (long long s = 1; s < L; s *= 2) {
      stockham_batch_kernel<<<(unsigned)((3 * mm * (L / 2) + 255) / 256), 256, 0, g.st>>>(x, y, L, s, 3 * mm);
      std::swap(x, y);
    }
    zimm_cross_kernel<<<(unsigned)((mm * L + 255) / 256), 256, 0, g.st>>>(x, L, mm, y);
    CK(cudaGetLastError());
    std::swap(x, y);
    for (long long s = 1; s < L; s *= 2) {
      stockham_batch_kernel<<<(unsigned)((mm * (L / 2) + 255) / 256), 256, 0, g.st>>>(x, y, L, s, mm);
      std::swap(x, y);
    }
    const dim3 agrid((unsigned)((N + 255) / 256), (unsigned)((mm + 255) / 256));
    zimm_accum_kernel<<<agrid, 256, 0, g.st>>>(x, L, N, mm, za.traj_base + t0, za.traj_per_iter, za.w / L, za.crln);
    CK(cudaGetLastError());
    g_launches += 3 + 2 * (unsigned long long)passes;
  }
  return HH_OK;
}

// one launchable variant of the CH4-CO2 dipole kernel (S records per lane)
// S: records per lane of ch4_dipole_kernel, or CH4_DIP_TC for the tensor-core kernel
// (hh_ch4co2_tc.cuh: tasks of 128 records, one CTA per SM)
constexpr int CH4_DIP_TC = -1;
struct Ch4DipVariant {
  void (*kern)(Ch4DipArgs);
  int S;
  size_t smem;
  int grid;
  int task() const { return S == CH4_DIP_TC ? CH4TC_M : 32 * S; }
};

int ch4_dip_tc_variant(Ch4DipVariant *v) {
  v->kern = nullptr;
  v->S = CH4_DIP_TC;
  v->smem = CH4TC_SMEM;
  CK(cudaFuncSetAttribute(ch4_dipole_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v->smem));
  v->grid = g.num_sms;  // the kernel holds all 512 TMEM columns of its SM
  return HH_OK;
}

template <typename PHYS, int S> int ch4_dip_variant(Ch4DipVariant *v) {
  v->kern = ch4_dipole_kernel<PHYS, S>;
  v->S = S;
  v->smem = ch4_dip_smem<PHYS, S>();
  if (v->smem > 48 * 1024)
    CK(cudaFuncSetAttribute(v->kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v->smem));
  int per = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, v->kern, 32 * CH4_DIP_WARPS, v->smem));
  v->grid = std::max(1, per) * g.num_sms;
  return HH_OK;
}

// the dipole kernel's candidates per precision: S = 1, 2, 4 and the tensor-core
// kernel (FP32), S = 1, 2 (FP64)
template <typename PHYS> int ch4_dip_candidates(Ch4DipVariant *v, int *n) {
  int rc = ch4_dip_variant<PHYS, 1>(&v[0]);
  if (!rc) rc = ch4_dip_variant<PHYS, 2>(&v[1]);
  *n = 2;
  if constexpr (sizeof(PHYS) == 4) {
    if (!rc) rc = ch4_dip_variant<PHYS, 4>(&v[2]);
    if (!rc) rc = ch4_dip_tc_variant(&v[3]);
    *n = 4;
  }
  return rc;
}

// CH4-CO2: the trajectory kernel writes every sample as a record, then the
// records are sorted by radial piece, their dipoles evaluated in batches and
// C(t) accumulated with the reference's per-sample tests (hh_ch4co2_dip.cuh).
// Trajectories go through in chunks whose records fit CH4_RECORD_BUDGET.
template <typename PHYS>
int run_records_t(const TrajParams &P, const double *d_ic, uint64_t n, uint64_t per_iter,
                  int precision, const double *d_satw, int n_sat, unsigned long long *cnt_dev, bool zimm, uint4 *trace = nullptr) {
  const int N = P.N;
  const int stride = 2 * N - 1;
  const size_t rec_b = HH_REC_WORDS * sizeof(PHYS), mu_b = 4 * sizeof(PHYS);
  const size_t per_traj = (size_t)stride * (rec_b + mu_b + sizeof(int)) + 4 * sizeof(int);
  uint64_t chunk = std::max<uint64_t>(1, CH4_RECORD_BUDGET / per_traj);
  chunk = std::min<uint64_t>(chunk, (uint64_t)((INT32_MAX - 128 * CH4_NSEG) / stride));
  chunk = std::min<uint64_t>(chunk, n);
  const size_t slots = (size_t)chunk * stride;
  CK(g.rec.ensure(slots * rec_b));
  CK(g.rec_mu.ensure(slots * mu_b));
  CK(g.rec_sorted.ensure(slots + (size_t)32 * CH4_DIP_SMAX * CH4_NSEG));
  CK(g.rec_len.ensure(2 * chunk));
  CK(g.rec_status.ensure(2 * chunk));
  CK(g.seg_cnt.ensure(2 * CH4_NSEG));
  CK(g.seg_w0.ensure(CH4_NSEG + 1));
  CK(g.rec_nfail.ensure(1));
  CK(cudaMemsetAsync(g.rec_nfail.p, 0, sizeof(unsigned long long), g.st));
  if (zimm) CK(g.zim_fail.ensure(chunk));
  Ch4Co2Fold fold;
  fold.n_batch = g.ch4_B;
  fold.cf = g.d_ch4_cf;
  fold.cd = g.d_ch4_cd;
  fold.y2 = g.d_ch4_y2;
  fold.meta = g.d_ch4_meta;
  for (int i = 0; i < CH4_NSEG - 1; ++i) fold.seg_hi[i] = hh_ch4co2_seg_hi[i];
  for (int i = 0; i < CH4_NSEG; ++i) fold.centre[i] = hh_ch4co2_centre[i];
  // dipole kernel variants; the records per lane are picked per precision by timing
  // every candidate on the first chunk of records (a dipole depends only on its
  // record, so every variant writes the same values)
  Ch4DipVariant cand[4];
  int ncand = 0;
  int rc0 = ch4_dip_candidates<PHYS>(cand, &ncand);
  if (rc0) return rc0;
  int &tuned_s = g.ch4_dip_s[sizeof(PHYS) == 4 ? 1 : 0];
  if (tuned_s == 0) {
    // HH_CH4_DIP_S fixes the records per lane (when it names a candidate; "tc" the
    // tensor-core kernel) instead of timing
    const char *env = getenv("HH_CH4_DIP_S");
    const int want = env ? (strcmp(env, "tc") == 0 ? CH4_DIP_TC : atoi(env)) : 0;
    for (int c = 0; c < ncand; ++c)
      if (cand[c].S == want) tuned_s = want;
  }
  for (uint64_t base = 0; base < n; base += chunk) {
    const uint64_t nc = std::min<uint64_t>(chunk, n - base);
    CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
    TrajIO io;
    memset(&io, 0, sizeof io);
    io.ic = d_ic + base * g.QP;
    io.n_items = (int)(2 * nc);
    io.queue = g.queue.p;
    io.crln = g.crln.p;
    io.counters = cnt_dev;
    io.status_hist = g.status_hist.p;
    io.traj_per_iter = (long long)per_iter;
    io.records = g.rec.p;
    io.rec_stride = stride;
    io.rec_len = g.rec_len.p;
    io.rec_status = g.rec_status.p;
    for (int k = 0; k < 3; ++k) io.inv_I1[k] = 1.0 / g.sx.II1[k];
    io.lj = g.sx.lj;
    io.item_trace = trace ? trace + 2 * base : nullptr;
    if (precision == HH_PRECISION_MIXED) {
      // item starts precomputed, one thread per item (the refills then load them)
      CK(g.istart.ensure(2 * chunk * sizeof(Ch4Start)));
      int rc1 = run_item_starts(P, io, g.istart.p);
      if (rc1) return rc1;
    }
    int rc = (precision == HH_PRECISION_MIXED) ? launch_traj<SYS_CH4CO2, float, float, false>(P, io, nullptr)
                                               : launch_traj<SYS_CH4CO2, double, double, false>(P, io, nullptr);
    if (rc) return rc;
    Ch4SortArgs sa;
    sa.records = g.rec.p;
    sa.rec_len = g.rec_len.p;
    sa.n_traj = (long long)nc;
    sa.stride = stride;
    sa.N = N;
    sa.count = g.seg_cnt.p;
    sa.cursor = g.seg_cnt.p + CH4_NSEG;
    sa.warp0 = g.seg_w0.p;
    sa.sorted = g.rec_sorted.p;
    for (int i = 0; i < CH4_NSEG - 1; ++i) sa.seg_hi[i] = hh_ch4co2_seg_hi[i];
    const long long nslots = (long long)nc * stride;
    const int sgrid = (int)std::min<long long>((nslots + 255) / 256, 8LL * g.num_sms);
    Ch4DipArgs da;
    da.f = fold;
    da.records = g.rec.p;
    da.sorted = g.rec_sorted.p;
    da.warp0 = g.seg_w0.p;
    da.mu = g.rec_mu.p;
    // sort the records into the tasks of variant v (32 S records, 128 for tensor cores)
    auto sort_for = [&](const Ch4DipVariant &v) -> int {
      sa.task = v.task();
      CK(cudaMemsetAsync(g.seg_cnt.p, 0, 2 * CH4_NSEG * sizeof(unsigned int), g.st));
      CK(cudaMemsetAsync(g.rec_sorted.p, 0xff, (nc * stride + (size_t)sa.task * CH4_NSEG) * sizeof(int), g.st));
      ch4_seg_count_kernel<PHYS><<<sgrid, 256, 0, g.st>>>(sa);
      ch4_seg_scan_kernel<<<1, 32, 0, g.st>>>(sa);
      ch4_seg_scatter_kernel<PHYS><<<sgrid, 256, 0, g.st>>>(sa);
      CK(cudaGetLastError());
      return HH_OK;
    };
    // the dipoles of the first max_tasks warp tasks with variant v
    auto dipole_with = [&](const Ch4DipVariant &v, long long max_tasks, long long step) -> int {
      if (v.S == CH4_DIP_TC) {
        if constexpr (sizeof(PHYS) == 4) {
          Ch4TcArgs ta;
          ta.records = static_cast<const float *>(g.rec.p ? (const void *)g.rec.p : nullptr);
          ta.sorted = g.rec_sorted.p;
          ta.warp0 = g.seg_w0.p;
          ta.blob = g.d_ch4_tc;
          ta.mu = reinterpret_cast<float *>(g.rec_mu.p);
          for (int i = 0; i < CH4_NSEG; ++i) ta.centre[i] = hh_ch4co2_centre[i];
          ta.max_tasks = max_tasks;
          ta.task_step = step;
          ta.err = g.d_ch4_tc_err;
          ch4_dipole_tc_kernel<<<v.grid, CH4TC_THREADS, v.smem, g.st>>>(ta);
        }
      } else {
        da.max_tasks = max_tasks;
        da.task_step = step;
        v.kern<<<v.grid, 32 * CH4_DIP_WARPS, v.smem, g.st>>>(da);
      }
      CK(cudaGetLastError());
      return HH_OK;
    };
    if (tuned_s == 0) {
      float best = 0.0f;
      for (int c = 0; c < ncand; ++c) {
        int rcs = sort_for(cand[c]);
        if (rcs) return rcs;
        // about 2^20 records for every variant, in tasks spread over all radial
        // pieces: one untimed run (the variant's first launch), then the timed one
        const long long step = std::max<long long>(1, nslots >> 20);
        rcs = dipole_with(cand[c], (1LL << 20) / cand[c].task(), step);
        if (rcs) return rcs;
        CK(cudaEventRecord(g.ev[4], g.st));
        rcs = dipole_with(cand[c], (1LL << 20) / cand[c].task(), step);
        if (rcs) return rcs;
        CK(cudaEventRecord(g.ev[5], g.st));
        CK(cudaEventSynchronize(g.ev[5]));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, g.ev[4], g.ev[5]));
        if (tuned_s == 0 || ms < best) {
          best = ms;
          tuned_s = cand[c].S;
        }
      }
      g_launches += 5 * (unsigned long long)ncand;
    }
    const Ch4DipVariant *use = &cand[0];
    for (int c = 0; c < ncand; ++c)
      if (cand[c].S == tuned_s) use = &cand[c];
    kt_begin();
    int rcd = sort_for(*use);
    kt_end(HH_KT_CH4_SORT);
    if (rcd) return rcd;
    kt_begin();
    rcd = dipole_with(*use, LLONG_MAX, 1);
    kt_end(HH_KT_CH4_DIPOLE);
    if (rcd) return rcd;
    Ch4CorrArgs ca;
    ca.mu = g.rec_mu.p;
    ca.rec_len = g.rec_len.p;
    ca.rec_status = g.rec_status.p;
    ca.n_traj = (long long)nc;
    ca.traj_base = (long long)base;
    ca.traj_per_iter = (long long)per_iter;
    ca.stride = stride;
    ca.crln = g.crln.p;
    ca.sat_w = d_satw;
    ca.n_sat = n_sat;
    ca.status_hist = g.status_hist.p;
    ca.n_failed = g.rec_nfail.p;
    ca.fail_out = zimm ? g.zim_fail.p : nullptr;
    ca.len_out = zimm ? g.rec_len.p : nullptr;
    kt_begin();
    ch4_corr_kernel<PHYS><<<(unsigned)((nc + 255) / 256), 256, 0, g.st>>>(P, ca);
    CK(cudaGetLastError());
    kt_end(HH_KT_CH4_CORR);
    g_launches += 5;
    if (zimm) {
      ZimmArgs za;
      za.series = g.rec_mu.p;
      za.len = g.rec_len.p;
      za.failed = g.zim_fail.p;
      za.n_traj = (long long)nc;
      za.traj_base = (long long)base;
      za.traj_per_iter = (long long)per_iter;
      za.stride = stride;
      za.N = N;
      za.w = 2.0 * P.weight / N;  // ppf ALU^3 / N
      za.crln = g.crln.p;
      const int rc = zimm_fft<PHYS>(za);
      if (rc) return rc;
    }
  }
  return HH_OK;
}

// Zimmermann estimate for the systems with an inline dipole: the trajectory kernel
// writes the dipole vector of every stored sample, then zimm_fft forms each
// trajectory's lagged products.  Trajectories go through in chunks whose series fit
// CH4_RECORD_BUDGET.  Dropped trajectories are skipped (no compensation pass).
template <typename PHYS>
int run_series_t(const TrajParams &P, const TrajIO &io0, const double *d_ic, uint64_t n, uint64_t per_iter,
                 int precision) {
  const int N = P.N;
  const int stride = 2 * N - 1;
  const size_t per_traj = (size_t)stride * 4 * sizeof(PHYS) + 2 * sizeof(int);
  uint64_t chunk = std::max<uint64_t>(1, CH4_RECORD_BUDGET / per_traj);
  chunk = std::min<uint64_t>(chunk, n);
  CK(g.rec_mu.ensure((size_t)chunk * stride * 4 * sizeof(PHYS)));
  CK(g.rec_len.ensure(2 * chunk));
  for (uint64_t base = 0; base < n; base += chunk) {
    const uint64_t nc = std::min<uint64_t>(chunk, n - base);
    CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
    CK(cudaMemsetAsync(g.fail_flag.p, 0, nc * sizeof(int), g.st));
    TrajIO io = io0;
    io.ic = d_ic + base * g.QP;
    io.n_items = (int)(2 * nc);
    io.series = g.rec_mu.p;
    io.rec_stride = stride;
    io.rec_len = g.rec_len.p;
    int rc = run_traj_dispatch(precision, P, io);
    if (rc) return rc;
    ZimmArgs za;
    za.series = g.rec_mu.p;
    za.len = g.rec_len.p;
    za.failed = g.fail_flag.p;
    za.n_traj = (long long)nc;
    za.traj_base = (long long)base;
    za.traj_per_iter = (long long)per_iter;
    za.stride = stride;
    za.N = N;
    za.w = 2.0 * P.weight / N;  // ppf ALU^3 / N
    za.crln = g.crln.p;
    rc = zimm_fft<PHYS>(za);
    if (rc) return rc;
  }
  return HH_OK;
}

// The bulk trajectory kernel's warps start each round together (TrajParams::block_sync):
// they then fetch the same step code at the same time, where unsynchronised warps at
// different phases of the loop thrash the instruction cache (CO2-Ar mixed, deferred
// samples: 22.0 -> 8.9 ms per iteration).  HH_TRAJ_BLOCK_SYNC=n puts the barrier on every
// n-th round instead, 0 switches it off.
int traj_block_sync() {
  const char *e = getenv("HH_TRAJ_BLOCK_SYNC");
  return e ? std::max(0, atoi(e)) : 1;
}

// The plain C(t) launches of run_trajectories, then the replay of failed trajectories
// (the reference drops a trajectory whose correlation_eval returns 1 while still
// counting it: both branches are replayed with the opposite weight).  With deferred
// samples the iterations go in launches whose sample contexts fit the buffer (at most
// 32 GiB and 40 % of the free memory, or HH_DEFER_BUDGET_MB); a launch that wrote
// more contexts than the buffer holds repeats the call with a larger estimate of
// contexts per item (HH_DEFER_EST sets the first one), and a second overflow with
// in-kernel samples.
int run_plain(int precision, const TrajParams &P, const TrajIO &io0, uint64_t n, uint64_t per_iter,
              uint64_t n_iter, int *nfail_out) {
  const size_t N = (size_t)P.N;
  const bool eligible = defer_eligible(precision, P, io0);
  for (int attempt = 0;; ++attempt) {
    const bool defer = eligible && attempt < 2;
    if (attempt > 0) {
      CK(cudaMemsetAsync(g.crln.p, 0, N * n_iter * sizeof(double), g.st));
      CK(cudaMemsetAsync(g.counters.p, 0, 16 * sizeof(unsigned long long), g.st));
      CK(cudaMemsetAsync(g.status_hist.p, 0, 2 * HH_ST_COUNT * sizeof(unsigned int), g.st));
      CK(cudaMemsetAsync(g.fail_flag.p, 0, n * sizeof(int), g.st));
      CK(cudaMemsetAsync(g.fail_count.p, 0, sizeof(int), g.st));
    }
    CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
    TrajIO io = io0;
    unsigned long long cap = 0;
    uint64_t it_launch = n_iter, items_launch = 2 * n;
    if (defer) {
      size_t free_b = 0, total_b = 0;
      CK(cudaMemGetInfo(&free_b, &total_b));
      double budget = std::min(32.0 * double(1ull << 30), 0.4 * double(free_b + g.dctx.cap + g.dvals.cap));
      if (const char *eb = getenv("HH_DEFER_BUDGET_MB")) budget = std::max(1.0, atof(eb)) * double(1 << 20);
      if (attempt == 0)
        if (const char *ee = getenv("HH_DEFER_EST")) g.defer_est = std::max(0.01, atof(ee));
      const double per_item = g.defer_est * double(DEFER_CTX_BYTES);
      const uint64_t max_items = (uint64_t)std::max(1.0, budget / per_item);
      it_launch = std::min<uint64_t>(n_iter, std::max<uint64_t>(1, max_items / (2 * per_iter)));
      items_launch = 2 * std::min<uint64_t>(n, it_launch * per_iter);
      cap = (unsigned long long)(g.defer_est * double(items_launch)) + 4096ull;
      if (getenv("HH_DEFER_TRACE"))
        fprintf(stderr, "[defer] attempt %d est %.3f items %llu cap %llu (buffer %llu) launches of %llu iterations, "
                "budget %.2f GB, free %.2f GB\n", attempt, g.defer_est, (unsigned long long)items_launch, cap,
                (unsigned long long)(g.dctx.cap / sizeof(DeferCtx)), (unsigned long long)it_launch, budget / 1e9,
                free_b / 1e9);
      // 10 % headroom: the estimate moves a little from call to call, and a larger
      // buffer would otherwise be reallocated (cudaFree and cudaMalloc of gigabytes)
      // inside a call
      const size_t alloc = (size_t)(1.1 * double(cap));
      if (g.dctx.cap < cap * sizeof(DeferCtx)) CK(g.dctx.ensure(alloc * sizeof(DeferCtx)));
      if (g.dvals.cap < cap * 2 * sizeof(float)) CK(g.dvals.ensure(alloc * 2 * sizeof(float)));
      CK(g.dcount.ensure(DEFER_WORDS));
      CK(g.item_status.ensure(2 * n));
      CK(g.item_mu0.ensure(2 * n * 4 * sizeof(float)));
      CK(g.item_fail.ensure(2 * n));
      if (g.sys == SYS_CO2AR) CK(g.istart.ensure(2 * n * sizeof(DeferStart)));
      CK(cudaMemsetAsync(g.item_fail.p, 0xff, 2 * n * sizeof(unsigned), g.st));
      CK(cudaMemsetAsync(g.dcount.p, 0, 2 * sizeof(unsigned long long), g.st));
      io.ctx = g.dctx.p;
      io.ctx_count = g.dcount.p;
      io.ctx_cap = cap;
      io.item_status = g.item_status.p;
      io.item_mu0 = g.item_mu0.p;
    }
    // item starts precomputed for the mixed N2-Ar path (its refill set-up evaluates the
    // PIP-NN surface twice and the dipole once on one lane)
    const bool starts = !defer && precision == HH_PRECISION_MIXED && g.sys == SYS_N2AR && io.n_sat == 0 &&
                        !io.series && !io.records;
    if (!defer) {
      if (starts) {
        CK(g.istart.ensure(2 * n * sizeof(DeferStart)));
        int rc = run_item_starts(P, io, g.istart.p);
        if (rc) return rc;
      }
      int rc = run_traj_dispatch(precision, P, io);
      if (rc) return rc;
    } else {
      for (uint64_t i0 = 0; i0 < n_iter; i0 += it_launch) {
        const uint64_t t0 = i0 * per_iter, t1 = std::min(n, (i0 + it_launch) * per_iter);
        TrajIO il = io;
        il.ic = io.ic + t0 * (uint64_t)g.QP;
        il.n_items = (int)(2 * (t1 - t0));
        il.crln = io.crln + i0 * N;
        il.fail_flag = io.fail_flag + t0;
        il.item_status = g.item_status.p + 2 * t0;
        il.item_mu0 = g.item_mu0.p + 2 * t0 * 4 * sizeof(float);
        il.item_trace = io.item_trace ? io.item_trace + 2 * t0 : nullptr;
        if (i0 > 0) {
          CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
          CK(cudaMemsetAsync(g.dcount.p, 0, sizeof(unsigned long long), g.st));
        }
        int rc = run_item_starts(P, il, g.istart.p + 2 * t0 * sizeof(DeferStart));
        if (rc) return rc;
        rc = run_traj_dispatch(precision, P, il);
        if (rc) return rc;
        rc = run_deferred(P, il, (long long)t0);
        if (rc) return rc;
      }
    }
    int nfail = 0;
    unsigned long long peak = 0;
    CK(cudaMemcpyAsync(&nfail, g.fail_count.p, sizeof nfail, cudaMemcpyDeviceToHost, g.st));
    if (defer) CK(cudaMemcpyAsync(&peak, g.dcount.p + DEFER_PEAK, sizeof peak, cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    if (defer) {
      const double per = double(peak) / double(std::max<uint64_t>(1, items_launch));
      if (peak > cap) {
        g.defer_est = std::max(2.0 * g.defer_est, 1.25 * per);
        continue;
      }
      g.defer_est = std::max(8.0, 1.25 * per);
    }
    if (nfail > 0) {
      std::vector<int> fl(nfail), it(2 * (size_t)nfail);
      CK(cudaMemcpy(fl.data(), g.fail_list.p, nfail * sizeof(int), cudaMemcpyDeviceToHost));
      for (int i = 0; i < nfail; ++i) {
        it[2 * i] = 2 * fl[i];
        it[2 * i + 1] = 2 * fl[i] + 1;
      }
      CK(g.items.ensure(it.size()));
      CK(cudaMemcpyAsync(g.items.p, it.data(), it.size() * sizeof(int), cudaMemcpyHostToDevice, g.st));
      CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
      TrajParams P2 = P;
      P2.weight = -P.weight;
      TrajIO io2 = io;
      io2.items = g.items.p;
      io2.n_items = (int)it.size();
      io2.fail_flag = nullptr;
      io2.counters = g.counters.p + 8;  // replay work is not counted twice
      io2.status_hist = g.status_hist.p + HH_ST_COUNT;
      io2.item_trace = nullptr;
      if (defer) {
        io2.ctx_cap = g.dctx.cap / sizeof(DeferCtx);
        if (io2.ctx_cap > g.dvals.cap / (2 * sizeof(float))) io2.ctx_cap = g.dvals.cap / (2 * sizeof(float));
        CK(cudaMemsetAsync(g.dcount.p, 0, 2 * sizeof(unsigned long long), g.st));
      }
      if (defer || starts) {
        int rc = run_item_starts(P2, io2, g.istart.p);
        if (rc) return rc;
      }
      int rc = run_traj_dispatch(precision, P2, io2);
      if (rc) return rc;
      if (defer) {
        rc = run_deferred(P2, io2, 0);
        if (rc) return rc;
        CK(cudaMemcpyAsync(&peak, g.dcount.p + DEFER_PEAK, sizeof peak, cudaMemcpyDeviceToHost, g.st));
        CK(cudaStreamSynchronize(g.st));
        if (peak > io2.ctx_cap) {
          g.defer_est *= 2.0;
          continue;
        }
      }
    }
    *nfail_out = nfail;
    return HH_OK;
  }
}

// integrate both branches of n trajectories whose phase points are in d_ic;
// trajectories [i*per_iter, (i+1)*per_iter) accumulate into C(t) slice i
int run_trajectories(const hh_calc_params *p, const double *d_ic, uint64_t n, uint64_t per_iter,
                     int precision, double *crln_host, hh_stats *stats, const double *d_satw = nullptr,
                     int n_sat = 0) {
  const size_t N = p->MaxTrajectoryLength;
  // C(t) slices: one per iteration, or one per satellite temperature
  const uint64_t n_iter = (n_sat > 0) ? (uint64_t)n_sat : (n + per_iter - 1) / per_iter;
  TrajParams P;
  memset(&P, 0, sizeof P);
  P.mu = g.mu;
  P.II = g.II;
  P.dt = p->sampling_time;
  P.N = (int)N;
  P.Rcut = p->Rcut;
  double tol = (precision == HH_PRECISION_MIXED)
                   ? (p->mixed_tolerance > 0 ? p->mixed_tolerance : 1e-8)
                   : p->cvode_tolerance;
  P.rtol = P.atol = tol;
  P.max_steps = p->max_steps > 0 ? p->max_steps : 50000;
  P.max_total_steps = 4000000;
  P.weight = p->partial_partition_function_ratio * 0.5 * HH_ALU * HH_ALU * HH_ALU;
  P.noise_floor = 16.0 * 5.96e-8;  // 16 FP32 half-ulps
  P.inject_item = g_inject_item;
  P.inject_k = g_inject_k;
  P.inject_status = g_inject_status;
  P.block_sync = traj_block_sync();
  CK(g.crln.ensure(N * n_iter));
  CK(g.counters.ensure(16));
  CK(g.status_hist.ensure(2 * HH_ST_COUNT));
  CK(g.queue.ensure(1));
  CK(g.fail_flag.ensure(std::max<uint64_t>(n, 1)));
  CK(g.fail_list.ensure(std::max<uint64_t>(n, 1)));
  CK(g.fail_count.ensure(1));
  CK(cudaMemsetAsync(g.crln.p, 0, N * n_iter * sizeof(double), g.st));
  CK(cudaMemsetAsync(g.counters.p, 0, 16 * sizeof(unsigned long long), g.st));
  CK(cudaMemsetAsync(g.status_hist.p, 0, 2 * HH_ST_COUNT * sizeof(unsigned int), g.st));
  CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
  CK(cudaMemsetAsync(g.fail_flag.p, 0, n * sizeof(int), g.st));
  CK(cudaMemsetAsync(g.fail_count.p, 0, sizeof(int), g.st));
  TrajIO io;
  memset(&io, 0, sizeof io);
  io.ic = d_ic;
  io.items = nullptr;
  io.n_items = (int)(2 * n);
  io.queue = g.queue.p;
  io.crln = g.crln.p;
  io.counters = g.counters.p;
  io.status_hist = g.status_hist.p;
  io.fail_flag = g.fail_flag.p;
  io.fail_list = g.fail_list.p;
  io.fail_count = g.fail_count.p;
  io.traj_per_iter = (long long)per_iter;
  io.item_trace = nullptr;
  io.dipnet = nullptr;
  io.pesnet = nullptr;
  io.diptab = nullptr;
  io.sat_w = d_satw;
  io.n_sat = n_sat;
  uint32_t *trace_host = g_trace_host;
  g_trace_host = nullptr;
  if (trace_host && g_trace_cap >= 4 * 2 * n) {
    CK(g.trace.ensure(2 * n));
    CK(cudaMemsetAsync(g.trace.p, 0, 2 * n * sizeof(uint4), g.st));
    io.item_trace = g.trace.p;
  }
  CK(cudaEventRecord(g.ev[2], g.st));
  int nfail = 0;
  const bool zimm = p->use_zimmermann_trick != 0;
  if (g.sys == SYS_CH4CO2) {
    int rc = (precision == HH_PRECISION_MIXED)
                 ? run_records_t<float>(P, d_ic, n, per_iter, precision, d_satw, n_sat, g.counters.p, zimm,
                                        io.item_trace)
                 : run_records_t<double>(P, d_ic, n, per_iter, precision, d_satw, n_sat, g.counters.p, zimm,
                                         io.item_trace);
    if (rc) return rc;
    unsigned long long nf = 0;
    int tc_err = 0;
    CK(cudaMemcpyAsync(&nf, g.rec_nfail.p, sizeof nf, cudaMemcpyDeviceToHost, g.st));
    CK(cudaMemcpyAsync(&tc_err, g.d_ch4_tc_err, sizeof tc_err, cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    if (tc_err) {
      CK(cudaMemsetAsync(g.d_ch4_tc_err, 0, sizeof(int), g.st));
      snprintf(g_errmsg, sizeof g_errmsg, "tensor-core dipole kernel: an mbarrier wait timed out");
      return HH_E_CUDA;
    }
    nfail = (int)nf;
  } else if (zimm) {
    if (n_sat > 0) return HH_E_INVALID_ARGUMENT;
    int rc = (precision == HH_PRECISION_MIXED) ? run_series_t<float>(P, io, d_ic, n, per_iter, precision)
                                               : run_series_t<double>(P, io, d_ic, n, per_iter, precision);
    if (rc) return rc;
    CK(cudaMemcpyAsync(&nfail, g.fail_count.p, sizeof nfail, cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
  } else {
    int rc = run_plain(precision, P, io, n, per_iter, n_iter, &nfail);
    if (rc) return rc;
  }
  CK(cudaEventRecord(g.ev[3], g.st));
  CK(cudaMemcpyAsync(crln_host, g.crln.p, N * n_iter * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  if (io.item_trace)
    CK(cudaMemcpyAsync(trace_host, g.trace.p, 2 * n * sizeof(uint4), cudaMemcpyDeviceToHost, g.st));
  unsigned long long cnt[8];
  unsigned int hist[HH_ST_COUNT];
  CK(cudaMemcpyAsync(cnt, g.counters.p, sizeof cnt, cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(hist, g.status_hist.p, sizeof hist, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  if (stats) {
    stats->n_steps = cnt[0];
    stats->n_rejected_steps = cnt[1];
    stats->n_rhs = cnt[2];
    stats->n_samples = cnt[3];
    stats->n_dense = cnt[4];
    stats->n_failed = (uint64_t)nfail;
    for (int i = 0; i < 8; ++i) stats->status[i] = (i < HH_ST_COUNT) ? hist[i] : 0;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, g.ev[2], g.ev[3]));
    stats->traj_ms = ms;
  }
  return HH_OK;
}

// launches the M0 kernel of the bound system over `grid` blocks; allocates nothing
int launch_m0(const M0Args &a, int grid, bool mixed, double *partials) {
  const int block = 256;
  kt_begin();
  if (g.sys == SYS_HEAR) {
    if (mixed) m0_kernel<SYS_HEAR, float, true><<<grid, block, 0, g.st>>>(a, g.d_tab, nullptr, partials);
    else m0_kernel<SYS_HEAR, double, false><<<grid, block, 0, g.st>>>(a, g.d_tab, nullptr, partials);
  } else if (g.sys == SYS_N2AR) {
    const size_t smem = sizeof(N2arDipFold);
    if (mixed) {
      auto k = m0_kernel<SYS_N2AR, float, true>;
      CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k<<<grid, block, smem, g.st>>>(a, g.d_tab, g.d_n2ar_fold, partials);
    } else {
      auto k = m0_kernel<SYS_N2AR, double, false>;
      CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k<<<grid, block, smem, g.st>>>(a, g.d_tab, g.d_n2ar_fold, partials);
    }
  } else {
    if (mixed)
      m0_kernel<SYS_CO2AR, float, true><<<grid, block, sizeof(Co2arTables<float>), g.st>>>(
          a, g.d_tab, nullptr, partials);
    else
      m0_kernel<SYS_CO2AR, double, false><<<grid, block, sizeof(Co2arTables<double>), g.st>>>(
          a, g.d_tab, nullptr, partials);
  }
  CK(cudaGetLastError());
  kt_end(HH_KT_MOMENT);
  return HH_OK;
}

// the second-moment kernels (FP64)
int launch_m2(const M0Args &a, int grid, double *partials) {
  const int block = 256;
  kt_begin();
  if (g.sys == SYS_HEAR) {
    m0_kernel<SYS_HEAR, double, false, 2><<<grid, block, 0, g.st>>>(a, g.d_tab, nullptr, partials);
  } else if (g.sys == SYS_N2AR) {
    const size_t smem = sizeof(N2arDipFold);
    auto k = m0_kernel<SYS_N2AR, double, false, 2>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, block, smem, g.st>>>(a, g.d_tab, g.d_n2ar_fold, partials);
  } else {
    m0_kernel<SYS_CO2AR, double, false, 2><<<grid, block, sizeof(Co2arTables<double>), g.st>>>(
        a, g.d_tab, nullptr, partials);
  }
  CK(cudaGetLastError());
  kt_end(HH_KT_MOMENT);
  return HH_OK;
}

// ---------------------------------------------------------------------------
// Scratch of hh_cuda_m0_noalloc: a fixed array compiled into the library, so
// that M0 can run in a process that must not allocate device memory once its
// run has started.  Layout: block partials [M0_NOALLOC_MAX_BLOCKS][M0_MAXT][2]
// (sum of w, sum of w^2), then results [HH_M0_NOALLOC_MAX_T][2].  One copy per
// device; calls whose GPU work overlaps share it and race.
constexpr int M0_NOALLOC_MAX_BLOCKS = 1024;
constexpr size_t M0_NOALLOC_PARTIALS = (size_t)M0_NOALLOC_MAX_BLOCKS * M0_MAXT * 2;
constexpr size_t M0_NOALLOC_WORDS = M0_NOALLOC_PARTIALS + 2 * (size_t)HH_M0_NOALLOC_MAX_T;
static_assert(HH_M0_NOALLOC_MAX_T % M0_MAXT == 0, "result slots come in whole temperature chunks");
static_assert(M0_NOALLOC_WORDS * sizeof(double) == HH_M0_NOALLOC_SCRATCH_BYTES,
              "header size of the allocation-free M0 scratch");
static __device__ __align__(256) double g_m0_noalloc_scratch[M0_NOALLOC_WORDS];

constexpr int NOALLOC_MAX_DEVICES = 64;
double *g_m0_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};  // device address per device, set on first use

// Device address of the scratch on the current device `dev`.  The first call
// per device after the library is brought up asks the runtime for it; bringing
// the library up (hh_cuda_init on a fresh context) and hh_cuda_shutdown forget the
// cached addresses, because a context torn down and created again may place the
// array elsewhere.
int m0_noalloc_scratch(int dev, double **out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return HH_E_INVALID_ARGUMENT;
  if (!g_m0_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_m0_noalloc_scratch));
    g_m0_noalloc_ptr[dev] = static_cast<double *>(ptr);
  }
  *out = g_m0_noalloc_ptr[dev];
  return HH_OK;
}

void m0_noalloc_forget() {
  for (auto &ptr : g_m0_noalloc_ptr) ptr = nullptr;
}

// Lepage's grid refinement (J. Comput. Phys. 27 (1978) 192) of one VEGAS iteration:
// per dimension, the per-bin sums d_i of F^2 are smoothed with their neighbours,
// normalised, compressed to m_i = ((1 - r_i) / -ln r_i)^alpha (r_i = d_i / sum d), and
// the new edges split the cumulative m into NB equal parts, interpolating linearly
// inside the old bins.  A dimension without any non-zero d keeps its grid.
void vegas_refine(std::vector<double> &edges, const std::vector<double> &hist, int D, double alpha) {
  const int NB = VEGAS_NB;
  std::vector<double> sm(NB), m(NB), cum(NB + 1), ne(NB + 1);
  for (int d = 0; d < D; ++d) {
    const double *h = hist.data() + (size_t)d * NB;
    double *e = edges.data() + (size_t)d * (NB + 1);
    sm[0] = 0.5 * (h[0] + h[1]);
    for (int i = 1; i < NB - 1; ++i) sm[i] = (h[i - 1] + h[i] + h[i + 1]) / 3.0;
    sm[NB - 1] = 0.5 * (h[NB - 2] + h[NB - 1]);
    double tot = 0.0;
    for (int i = 0; i < NB; ++i) tot += sm[i];
    if (!(tot > 0.0)) continue;
    double M = 0.0;
    for (int i = 0; i < NB; ++i) {
      const double r = sm[i] / tot;
      m[i] = (r > 0.0 && r < 1.0) ? pow((1.0 - r) / -log(r), alpha) : (r >= 1.0 ? 1.0 : 0.0);
      M += m[i];
    }
    if (!(M > 0.0)) continue;
    cum[0] = 0.0;
    for (int i = 0; i < NB; ++i) cum[i + 1] = cum[i] + m[i];
    ne[0] = e[0];
    ne[NB] = e[NB];
    int j = 0;
    for (int k = 1; k < NB; ++k) {
      const double target = M * double(k) / double(NB);
      while (j < NB - 1 && cum[j + 1] < target) ++j;
      const double frac = m[j] > 0.0 ? (target - cum[j]) / m[j] : 0.0;
      ne[k] = e[j] + std::min(1.0, std::max(0.0, frac)) * (e[j + 1] - e[j]);
    }
    for (int k = 0; k <= NB; ++k) e[k] = ne[k];
  }
}

template <int SYS> int launch_vegas(const VegasArgs &a, int grid) {
  const size_t smem = vegas_smem<SYS>();
  CK(cudaFuncSetAttribute(vegas_kernel<SYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kt_begin();
  vegas_kernel<SYS><<<grid, VEGAS_THREADS, smem, g.st>>>(a, g.d_tab, g.d_n2ar_fold);
  CK(cudaGetLastError());
  kt_end(HH_KT_MOMENT);
  return HH_OK;
}

}  // namespace

extern "C" {

const char *hh_cuda_strerror(int code) {
  switch (code) {
    case HH_OK: return "ok";
    case HH_E_NOT_INITIALIZED: return "hh_cuda_init has not been called";
    case HH_E_INVALID_ARGUMENT: return "invalid argument";
    case HH_E_CUDA: return g_errmsg[0] ? g_errmsg : "CUDA error";
    case HH_E_UNSUPPORTED_SYSTEM: return "unsupported system";
    case HH_E_OUT_OF_MEMORY: return "out of device memory";
    case HH_E_NOT_POWER_OF_TWO: return "length of the input array should be a power of 2";
    case HH_E_SAMPLER: return g_errmsg[0] ? g_errmsg : "sampler error";
    case HH_E_NO_DEVICE: return "no CUDA device";
    case HH_E_SCRATCH_LIMIT:
      return "request exceeds the fixed scratch of an allocation-free entry point "
             "(hh_cuda_m0_noalloc: nT > HH_M0_NOALLOC_MAX_T)";
    default: return "unknown error";
  }
}

int hh_cuda_init(int device, const hh_system_desc *sys) {
  if (!sys) return HH_E_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return HH_E_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return HH_E_INVALID_ARGUMENT;
  int sid = sys->system_id;
  if (sid == HH_SYSTEM_HE_AR) {
    if (sys->monomer1_type != HH_MONOMER_ATOM || sys->monomer2_type != HH_MONOMER_ATOM)
      return HH_E_UNSUPPORTED_SYSTEM;
  } else if (sid == HH_SYSTEM_CO2_AR || sid == HH_SYSTEM_N2_AR) {
    if (sys->monomer1_type != HH_MONOMER_LINEAR_MOLECULE || sys->monomer2_type != HH_MONOMER_ATOM)
      return HH_E_UNSUPPORTED_SYSTEM;
    if (!(sys->II1[0] > 0) || sys->II1[0] != sys->II1[1]) return HH_E_INVALID_ARGUMENT;
  } else if (sid == HH_SYSTEM_CH4_CO2) {
    if (sys->monomer1_type != HH_MONOMER_ROTOR || sys->monomer2_type != HH_MONOMER_LINEAR_MOLECULE)
      return HH_E_UNSUPPORTED_SYSTEM;
    if (!(sys->II1[0] > 0) || !(sys->II1[1] > 0) || !(sys->II1[2] > 0) || !(sys->II2[0] > 0) ||
        sys->II2[0] != sys->II2[1])
      return HH_E_INVALID_ARGUMENT;
  } else {
    return HH_E_UNSUPPORTED_SYSTEM;
  }
  if (!(sys->mu > 0)) return HH_E_INVALID_ARGUMENT;
  if (g.init && g.device != device) hh_cuda_shutdown();
  CK(cudaSetDevice(device));
  if (!g.init) {
    m0_noalloc_forget();
    int prio_low = 0, prio_high = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    CK(cudaStreamCreateWithPriority(&g.st, cudaStreamNonBlocking, prio_high));
    CK(cudaStreamCreateWithFlags(&g.st2, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithPriority(&g.st3, cudaStreamNonBlocking, prio_low));
    CK(cudaEventCreateWithFlags(&g.ev_bulk, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&g.ev_eval1, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&g.ev_sampled, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&g.ev_pregen, cudaEventDisableTiming));
    for (auto &e : g.ev) CK(cudaEventCreate(&e));
    CK(cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, device));
    CK(cudaMalloc(&g.d_tab, sizeof(Co2arTablesGlobal)));
    CK(cudaMalloc(&g.d_mt, MT_N * sizeof(uint32_t)));
    CK(upload_mt_jump_tables(&g.d_mt_jump_seg, &g.d_mt_jump_coarse));
    static Co2arTablesGlobal host_tab;
    build_tables(&host_tab);
    CK(cudaMemcpy(g.d_tab, &host_tab, sizeof host_tab, cudaMemcpyHostToDevice));
    g.device = device;
    g.init = true;
    int rc = reseed(0);
    if (rc) return rc;
  }
  if (sid == HH_SYSTEM_N2_AR && !g.d_n2ar_fold) {
    static N2arDipFold host_fold;
    if (n2ar_build_fold(&host_fold) != 0) return HH_E_UNSUPPORTED_SYSTEM;
    CK(cudaMalloc(&g.d_n2ar_fold, sizeof(N2arDipFold)));
    CK(cudaMemcpy(g.d_n2ar_fold, &host_fold, sizeof host_fold, cudaMemcpyHostToDevice));
    static N2arPesNet<double> pes_d;
    static N2arPesNet<float> pes_f;
    n2ar_build_pes(&pes_d, &pes_f);
    CK(cudaMalloc(&g.d_n2ar_pes_d, sizeof pes_d));
    CK(cudaMalloc(&g.d_n2ar_pes_f, sizeof pes_f));
    CK(cudaMemcpy(g.d_n2ar_pes_d, &pes_d, sizeof pes_d, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.d_n2ar_pes_f, &pes_f, sizeof pes_f, cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g.d_n2ar_tab, (size_t)N2T_CELLS * N2T_CELL_F4 * sizeof(float4)));
    n2ar_tab_build_kernel<<<N2T_CELLS, 128>>>(g.d_n2ar_fold, g.d_n2ar_tab);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
  }
  if (sid == HH_SYSTEM_CH4_CO2 && !g.d_ch4_cd) {
    Ch4Co2FoldHost f;
    if (ch4co2_build_fold(&f) != 0) return HH_E_UNSUPPORTED_SYSTEM;
    // the padded batch stream (whole batches of 4 entries per group)
    const size_t B = (size_t)f.n_batch;
    std::vector<float4> cf(HH_CH4CO2_NSEG * 4 * B);
    for (size_t i = 0; i < cf.size(); ++i)
      cf[i] = make_float4((float)f.bcoef[4 * i], (float)f.bcoef[4 * i + 1], (float)f.bcoef[4 * i + 2],
                          (float)f.bcoef[4 * i + 3]);
    CK(cudaMalloc(&g.d_ch4_cd, f.bcoef.size() * sizeof(double)));
    CK(cudaMalloc(&g.d_ch4_cf, cf.size() * sizeof(float4)));
    CK(cudaMalloc(&g.d_ch4_y2, 4 * B));
    CK(cudaMalloc(&g.d_ch4_meta, B * sizeof(unsigned int)));
    CK(cudaMemcpy(g.d_ch4_cd, f.bcoef.data(), f.bcoef.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.d_ch4_cf, cf.data(), cf.size() * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.d_ch4_y2, f.by2.data(), 4 * B, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.d_ch4_meta, f.bmeta.data(), B * sizeof(unsigned int), cudaMemcpyHostToDevice));
    std::vector<float> tc_blob;
    if (ch4co2_build_tc_blob(f, &tc_blob) != 0) return HH_E_UNSUPPORTED_SYSTEM;
    CK(cudaMalloc(&g.d_ch4_tc, tc_blob.size() * sizeof(float)));
    CK(cudaMemcpy(g.d_ch4_tc, tc_blob.data(), tc_blob.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g.d_ch4_tc_err, sizeof(int)));
    CK(cudaMemset(g.d_ch4_tc_err, 0, sizeof(int)));
    // the harmonics' recurrence coefficients by (m, l) (hh_ch4co2_tc.cuh)
    {
      float alpha[CH4_L1 + 1][CH4_L1 + 1] = {}, beta[CH4_L1 + 1][CH4_L1 + 1] = {}, pmv[CH4_L1 + 1];
      double pm = 1.0;
      for (int m = 0; m <= CH4_L1; ++m) {
        if (m > 0) pm = -pm * sqrt(double(2 * m - 1) / double(2 * m));
        pmv[m] = (float)pm;
        for (int l = m + 1; l <= CH4_L1; ++l) {
          if (l == m + 1) {
            alpha[m][l] = (float)sqrt(double(2 * m + 1));
          } else {
            const double id = 1.0 / sqrt(double(l * l - m * m));
            alpha[m][l] = (float)(double(2 * l - 1) * id);
            beta[m][l] = (float)(sqrt(double((l - 1) * (l - 1) - m * m)) * id);
          }
        }
      }
      CK(cudaMemcpyToSymbol(c_ch4tc_alpha, alpha, sizeof alpha));
      CK(cudaMemcpyToSymbol(c_ch4tc_beta, beta, sizeof beta));
      CK(cudaMemcpyToSymbol(c_ch4tc_pm, pmv, sizeof pmv));
    }
    g.ch4_B = f.n_batch;
    g.ch4_groups = 0;
    for (size_t b = 0; b < B; ++b) g.ch4_groups += (f.bmeta[b] & 8u) ? 1 : 0;
  }
  g.sys = (sid == HH_SYSTEM_HE_AR)    ? SYS_HEAR
          : (sid == HH_SYSTEM_N2_AR)  ? SYS_N2AR
          : (sid == HH_SYSTEM_CH4_CO2) ? SYS_CH4CO2
                                      : SYS_CO2AR;
  g.mu = sys->mu;
  // the linear monomer's moment: monomer 1, or CO2 as monomer 2 of CH4-CO2
  g.II = (sid == HH_SYSTEM_HE_AR) ? 0.0 : (sid == HH_SYSTEM_CH4_CO2 ? sys->II2[0] : sys->II1[0]);
  g.QP = (sid == HH_SYSTEM_HE_AR) ? 6 : (sid == HH_SYSTEM_CH4_CO2 ? 16 : 10);
  g.D = (sid == HH_SYSTEM_HE_AR) ? 10 : (sid == HH_SYSTEM_CH4_CO2 ? 25 : 16);
  memset(&g.sx, 0, sizeof g.sx);
  if (sid == HH_SYSTEM_CH4_CO2) {
    for (int k = 0; k < 3; ++k) g.sx.II1[k] = sys->II1[k];
    hh_ch4co2_lj_pairs(g.sx.lj.A, g.sx.lj.B);
  }
  g.p_accept = 0.25;
  return HH_OK;
}

int hh_cuda_seed(uint32_t seed) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  CK(cudaSetDevice(g.device));
  int rc = reseed(seed);
  if (rc) return rc;
  CK(cudaStreamSynchronize(g.st));
  return HH_OK;
}

int hh_cuda_sample(const hh_calc_params *p, double T, uint32_t seed, uint64_t n, double *qp_out,
                   uint64_t *n_candidates) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  int rc = check_params(p);
  if (rc) return rc;
  if (!(T > 0) || (n > 0 && !qp_out)) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  if (seed > 0) {
    rc = reseed(seed);
    if (rc) return rc;
  }
  if (n == 0) return HH_OK;
  CK(g.qp0.ensure(n * g.QP));
  rc = sample_into(p, T, n, g.qp0.p, n_candidates);
  if (rc) return rc;
  CK(cudaMemcpyAsync(qp_out, g.qp0.p, n * g.QP * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return HH_OK;
}

int hh_cuda_correlation_multi(const hh_calc_params *p, double T, uint32_t seed,
                              uint64_t n_per_iteration, uint32_t n_iterations, int precision_mode,
                              double *crln_sums, double *ntraj, hh_stats *stats) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  int rc = check_params(p);
  if (rc) return rc;
  const uint64_t n_accept = n_per_iteration * (uint64_t)n_iterations;
  if (!(T > 0) || !crln_sums || n_per_iteration == 0 || n_iterations == 0 ||
      n_accept > (uint64_t)(INT32_MAX / 2))
    return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  if (seed > 0) {
    rc = reseed(seed);
    if (rc) return rc;
  }
  hh_stats local;
  memset(&local, 0, sizeof local);
  g_launches = 0;
  CK(g.qp0.ensure(n_accept * g.QP));
  CK(cudaEventRecord(g.ev[0], g.st));
  uint64_t ncand = 0;
  const long long wpos0 = g.wpos;
  rc = sample_into(p, T, n_accept, g.qp0.p, &ncand);
  if (rc) return rc;
  CK(cudaEventRecord(g.ev[1], g.st));
  rc = pregen_words(g.wpos - wpos0);
  if (rc) return rc;
  rc = run_trajectories(p, g.qp0.p, n_accept, n_per_iteration, precision_mode, crln_sums, &local);
  if (rc) return rc;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[1]));
  local.sample_ms = ms;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[3]));
  local.total_ms = ms;
  local.n_candidates = ncand;
  local.n_accepted = n_accept;
  local.n_kernel_launches = g_launches;
  if (ntraj)
    for (uint32_t i = 0; i < n_iterations; ++i) ntraj[i] = (double)n_per_iteration;
  if (stats) *stats = local;
  return HH_OK;
}

int hh_cuda_correlation_temperatures(const hh_calc_params *p, const double *T, int nT, uint32_t seed,
                                     uint64_t n_per_T, int precision_mode, double *crln_sums,
                                     double *ntraj, hh_stats *stats) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  int rc = check_params(p);
  if (rc) return rc;
  if (!T || nT < 1 || !crln_sums || n_per_T == 0 || n_per_T * (uint64_t)nT > (uint64_t)(INT32_MAX / 2))
    return HH_E_INVALID_ARGUMENT;
  for (int i = 0; i < nT; ++i)
    if (!(T[i] > 0)) return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  if (seed > 0) {
    rc = reseed(seed);
    if (rc) return rc;
  }
  hh_stats local;
  memset(&local, 0, sizeof local);
  g_launches = 0;
  const uint64_t n = n_per_T * (uint64_t)nT;
  CK(g.qp0.ensure(n * g.QP));
  CK(cudaEventRecord(g.ev[0], g.st));
  const long long wpos0 = g.wpos;
  uint64_t ncand = 0;
  for (int i = 0; i < nT; ++i) {
    uint64_t nc = 0;
    rc = sample_into(p, T[i], n_per_T, g.qp0.p + (size_t)i * n_per_T * g.QP, &nc);
    if (rc) return rc;
    ncand += nc;
  }
  CK(cudaEventRecord(g.ev[1], g.st));
  rc = pregen_words(g.wpos - wpos0);
  if (rc) return rc;
  rc = run_trajectories(p, g.qp0.p, n, n_per_T, precision_mode, crln_sums, &local);
  if (rc) return rc;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[1]));
  local.sample_ms = ms;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[3]));
  local.total_ms = ms;
  local.n_candidates = ncand;
  local.n_accepted = n;
  local.n_kernel_launches = g_launches;
  if (ntraj)
    for (int i = 0; i < nT; ++i) ntraj[i] = (double)n_per_T;
  if (stats) *stats = local;
  return HH_OK;
}

int hh_cuda_prmu(const hh_calc_params *p, double T, double R0, double approx_freq_max, int allow_truncating,
                 uint32_t seed, uint64_t n_traj, int precision_mode, double *nu, double *sf, size_t sf_len,
                 size_t *n_freq, double *ntraj, hh_stats *stats) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (g.sys == SYS_CH4CO2) return HH_E_UNSUPPORTED_SYSTEM;
  if (g.req.mode != HH_REQ_NONE && g.sys == SYS_HEAR) return HH_E_UNSUPPORTED_SYSTEM;
  int rc = check_params(p);
  if (rc) return rc;
  if (!(T > 0) || !(R0 > 0) || !(approx_freq_max > 0) || !nu || !sf || !n_freq || n_traj == 0 ||
      n_traj > (uint64_t)(INT32_MAX / 2))
    return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  const size_t N = p->MaxTrajectoryLength;
  if (N < 2 || (N & (N - 1))) return HH_E_NOT_POWER_OF_TWO;  // gsl_fft_real_radix2_transform
  const double dt = p->sampling_time;
  // frequency grid (src/hawaii.c:3189-3200)
  const double step = 1.0 / (dt * HH_ATU) / HH_LIGHTSPEED_CM / (double)N;
  const double fmax_theory = 1.0 / (HH_LIGHTSPEED_CM * dt * HH_ATU) / 2.0;
  if (approx_freq_max > fmax_theory) return HH_E_INVALID_ARGUMENT;
  const size_t L = (size_t)(int)(approx_freq_max / step) + 1;
  *n_freq = L;
  if (sf_len < L) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  if (seed > 0) {
    rc = reseed(seed);
    if (rc) return rc;
  }
  hh_stats local;
  memset(&local, 0, sizeof local);
  g_launches = 0;
  // draws: q_generator, R := R0, p_generator, inward pR; one word fewer than a candidate
  CK(g.qp0.ensure(n_traj * g.QP));
  CK(cudaEventRecord(g.ev[0], g.st));
  const int D0 = g.D;
  const double pa0 = g.p_accept;
  g.D = D0 - 1;
  g.sx.prmu_R0 = R0;
  g.p_accept = 1.0;
  uint64_t ncand = 0;
  rc = sample_into(p, T, n_traj, g.qp0.p, &ncand);
  g.D = D0;
  g.sx.prmu_R0 = 0.0;
  g.p_accept = pa0;
  if (rc) return rc;
  CK(cudaEventRecord(g.ev[1], g.st));
  // forward branches with samples k = 1..N at t = k dt, ending after R > R0
  TrajParams P;
  memset(&P, 0, sizeof P);
  P.mu = g.mu;
  P.II = g.II;
  P.dt = dt;
  P.N = (int)N + 1;
  P.Rcut = R0;
  const double tol = (precision_mode == HH_PRECISION_MIXED)
                         ? (p->mixed_tolerance > 0 ? p->mixed_tolerance : 1e-8)
                         : p->cvode_tolerance;
  P.rtol = P.atol = tol;
  P.max_steps = p->max_steps > 0 ? p->max_steps : 50000;
  P.max_total_steps = 4000000;
  P.noise_floor = 16.0 * 5.96e-8;
  P.inject_item = P.inject_k = -1;
  P.prmu = 1;
  P.block_sync = traj_block_sync();
  const bool req = g.req.mode != HH_REQ_NONE;
  if (req) {
    P.req_mode = g.req.mode;
    P.req_len = (int)g.req.torque_cache_len;
    P.req_limit = g.req.torque_limit;
  }
  const int stride = (int)N + 1;
  const size_t ps = (precision_mode == HH_PRECISION_MIXED) ? sizeof(float) : sizeof(double);
  const size_t per_traj = (size_t)stride * 4 * ps + 2 * 2 * N * sizeof(double2) + 4 * sizeof(int);
  const uint64_t chunk = std::min<uint64_t>(n_traj, std::max<uint64_t>(1, CH4_RECORD_BUDGET / per_traj));
  CK(g.rec_mu.ensure((size_t)chunk * stride * 4 * ps));
  CK(g.rec_len.ensure(2 * chunk));
  CK(g.rec_status.ensure(2 * chunk));
  CK(g.pm_a.ensure(2 * chunk * N));
  CK(g.pm_b.ensure(2 * chunk * N));
  CK(g.pm_sf.ensure(L));
  CK(g.counters.ensure(16));
  CK(g.status_hist.ensure(2 * HH_ST_COUNT));
  CK(g.queue.ensure(1));
  CK(g.rec_nfail.ensure(1));
  CK(cudaMemsetAsync(g.pm_sf.p, 0, L * sizeof(double), g.st));
  CK(cudaMemsetAsync(g.counters.p, 0, 16 * sizeof(unsigned long long), g.st));
  CK(cudaMemsetAsync(g.rec_nfail.p, 0, sizeof(unsigned long long), g.st));
  CK(cudaEventRecord(g.ev[2], g.st));
  const double sf_coeff = HH_HARTREE * pow(HH_ALU, 6) * HH_ATU * R0 * R0 * dt * dt;
  for (uint64_t base = 0; base < n_traj; base += chunk) {
    const uint64_t nc = std::min<uint64_t>(chunk, n_traj - base);
    CK(cudaMemsetAsync(g.queue.p, 0, sizeof(unsigned int), g.st));
    TrajIO io;
    memset(&io, 0, sizeof io);
    io.ic = g.qp0.p + base * g.QP;
    io.n_items = (int)nc;
    io.fwd_only = 1;
    io.queue = g.queue.p;
    io.crln = g.pm_sf.p;
    io.counters = g.counters.p;
    io.status_hist = g.status_hist.p + HH_ST_COUNT;  // the records' statuses are counted below
    io.traj_per_iter = (long long)n_traj;
    io.series = g.rec_mu.p;
    io.rec_stride = stride;
    io.rec_len = g.rec_len.p;
    io.rec_status = g.rec_status.p;
    io.dipnet = g.d_n2ar_fold;
    io.pesnet = (precision_mode == HH_PRECISION_MIXED) ? (const void *)g.d_n2ar_pes_f : (const void *)g.d_n2ar_pes_d;
    rc = req ? run_traj_dispatch_req(precision_mode, P, io) : run_traj_dispatch(precision_mode, P, io);
    if (rc) return rc;
    PrmuPackArgs pa;
    pa.req_mode = g.req.mode;
    pa.even_w = g.req.even_j_spin_weight;
    pa.odd_w = g.req.odd_j_spin_weight;
    pa.series = g.rec_mu.p;
    pa.len = g.rec_len.p;
    pa.status = g.rec_status.p;
    pa.qp = g.qp0.p + base * g.QP;
    pa.QP = g.QP;
    pa.n_traj = (long long)nc;
    pa.N = (int)N;
    pa.stride = stride;
    pa.allow_trunc = allow_truncating ? 1 : 0;
    pa.coeff = sf_coeff / g.mu;
    pa.z = g.pm_a.p;
    pa.counted = g.rec_nfail.p;
    const long long tot = (long long)nc * (long long)N;
    if (precision_mode == HH_PRECISION_MIXED)
      prmu_pack_kernel<float><<<(unsigned)((tot + 255) / 256), 256, 0, g.st>>>(pa);
    else
      prmu_pack_kernel<double><<<(unsigned)((tot + 255) / 256), 256, 0, g.st>>>(pa);
    CK(cudaGetLastError());
    const long long B = 2 * (long long)nc;
    double2 *x = g.pm_a.p, *y = g.pm_b.p;
    for (long long s = 1; s < (long long)N; s *= 2) {
      stockham_batch_kernel<<<(unsigned)((B * ((long long)N / 2) + 255) / 256), 256, 0, g.st>>>(x, y, (long long)N, s, B);
      std::swap(x, y);
    }
    prmu_accum_kernel<<<(unsigned)((L + 255) / 256), 256, 0, g.st>>>(x, B, (int)N, (int)L, g.pm_sf.p);
    CK(cudaGetLastError());
    g_launches += 2 + (unsigned long long)__builtin_ctzll((unsigned long long)N);  // pack, accumulate, passes
  }
  CK(cudaEventRecord(g.ev[3], g.st));
  unsigned long long counted = 0;
  unsigned long long cnt[8];
  CK(cudaMemcpyAsync(sf, g.pm_sf.p, L * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(&counted, g.rec_nfail.p, sizeof counted, cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(cnt, g.counters.p, sizeof cnt, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  for (size_t i = 0; i < L; ++i) nu[i] = step * (double)i;
  if (ntraj) *ntraj = (double)counted;
  float ms = 0.f;
  local.n_candidates = ncand;
  local.n_accepted = n_traj;
  local.n_steps = cnt[0];
  local.n_rejected_steps = cnt[1];
  local.n_rhs = cnt[2];
  local.n_samples = cnt[3];
  local.n_failed = n_traj - counted;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[1]));
  local.sample_ms = ms;
  CK(cudaEventElapsedTime(&ms, g.ev[2], g.ev[3]));
  local.traj_ms = ms;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[3]));
  local.total_ms = ms;
  local.n_kernel_launches = g_launches;
  if (stats) *stats = local;
  return HH_OK;
}

int hh_cuda_correlation_array(const hh_calc_params *p, double base_T, const double *sat_T,
                              const double *ppf_ratios, int n_sat, uint32_t seed, uint64_t n_accept,
                              int precision_mode, double *crln_sums, double *nstar, double *ntraj,
                              hh_stats *stats) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  int rc = check_params(p);
  if (rc) return rc;
  if (!(base_T > 0) || !sat_T || !ppf_ratios || !crln_sums || !nstar || n_sat < 1 || n_sat > SAT_MAX ||
      n_accept == 0 || n_accept > (uint64_t)(INT32_MAX / 2))
    return HH_E_INVALID_ARGUMENT;
  for (int s = 0; s < n_sat; ++s)
    if (!(sat_T[s] > 0)) return HH_E_INVALID_ARGUMENT;
  // the reference has no weights for PAIR_STATE_ALL (hawaii.c:2652)
  if (p->pair_state != HH_PAIR_STATE_FREE_AND_METASTABLE && p->pair_state != HH_PAIR_STATE_BOUND)
    return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  if (seed > 0) {
    rc = reseed(seed);
    if (rc) return rc;
  }
  hh_stats local;
  memset(&local, 0, sizeof local);
  g_launches = 0;
  CK(g.qp0.ensure(n_accept * g.QP));
  CK(g.sat_w.ensure(n_accept * n_sat));
  CK(g.sat_wraw.ensure(n_accept * n_sat));
  CK(cudaEventRecord(g.ev[0], g.st));
  uint64_t ncand = 0;
  const long long wpos0 = g.wpos;
  rc = sample_into(p, base_T, n_accept, g.qp0.p, &ncand);
  if (rc) return rc;
  rc = pregen_words(g.wpos - wpos0);
  if (rc) return rc;
  CK(launch_sat_weights(g.sys, g.mu, g.II, p->pesmin, p->pair_state, g.d_tab, g.qp0.p, (long long)n_accept,
                        base_T, sat_T, ppf_ratios, n_sat, g.sat_w.p, g.sat_wraw.p, g.sx, g.st));
  g_launches += 1;
  CK(cudaEventRecord(g.ev[1], g.st));
  hh_calc_params p1 = *p;
  p1.partial_partition_function_ratio = 1.0;  // the ratios are in the weights
  rc = run_trajectories(&p1, g.qp0.p, n_accept, n_accept, precision_mode, crln_sums, &local, g.sat_w.p, n_sat);
  if (rc) return rc;
  std::vector<double> wraw(n_accept * (size_t)n_sat);
  CK(cudaMemcpy(wraw.data(), g.sat_wraw.p, wraw.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int s = 0; s < n_sat; ++s) nstar[s] = 0.0;
  for (uint64_t i = 0; i < n_accept; ++i)
    for (int s = 0; s < n_sat; ++s) nstar[s] += wraw[i * n_sat + s];
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[1]));
  local.sample_ms = ms;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[3]));
  local.total_ms = ms;
  local.n_candidates = ncand;
  local.n_accepted = n_accept;
  local.n_kernel_launches = g_launches;
  if (ntraj) *ntraj = (double)n_accept;
  if (stats) *stats = local;
  return HH_OK;
}

int hh_cuda_correlation(const hh_calc_params *p, double T, uint32_t seed, uint64_t n_accept,
                        int precision_mode, double *crln_sum, double *ntraj, hh_stats *stats) {
  return hh_cuda_correlation_multi(p, T, seed, n_accept, 1, precision_mode, crln_sum, ntraj, stats);
}

int hh_cuda_correlation_ic(const hh_calc_params *p, const double *qp0, uint64_t n,
                           int precision_mode, double *crln_sum, hh_stats *stats) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  int rc = check_params(p);
  if (rc) return rc;
  if (!qp0 || !crln_sum || n == 0 || n > (uint64_t)(INT32_MAX / 2)) return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  hh_stats local;
  memset(&local, 0, sizeof local);
  g_launches = 0;
  CK(g.qp0.ensure(n * g.QP));
  CK(cudaEventRecord(g.ev[0], g.st));
  CK(cudaMemcpyAsync(g.qp0.p, qp0, n * g.QP * sizeof(double), cudaMemcpyHostToDevice, g.st));
  CK(cudaEventRecord(g.ev[1], g.st));
  rc = run_trajectories(p, g.qp0.p, n, n, precision_mode, crln_sum, &local);
  if (rc) return rc;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[3]));
  local.total_ms = ms;
  local.n_accepted = n;
  local.n_kernel_launches = g_launches;
  if (stats) *stats = local;
  return HH_OK;
}

int hh_cuda_moment_sums(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
                        uint64_t sample_offset, uint64_t seed, int moment, int precision_mode,
                        double *sum_w, double *sum_w2) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (g.sys == SYS_CH4CO2) return HH_E_UNSUPPORTED_SYSTEM;  // no CH4-CO2 moment integrand
  if (!p || !T || nT < 1 || !sum_w || n_samples == 0) return HH_E_INVALID_ARGUMENT;
  if (moment != 0 && moment != 2) return HH_E_INVALID_ARGUMENT;
  if (!(p->sampler_Rmin > 0) || !(p->sampler_Rmax > p->sampler_Rmin)) return HH_E_INVALID_ARGUMENT;
  if (p->pair_state < 1 || p->pair_state > 3) return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  if (moment == 2 && precision_mode != HH_PRECISION_FP64) return HH_E_INVALID_ARGUMENT;
  if (sample_offset > UINT64_MAX - n_samples) return HH_E_INVALID_ARGUMENT;
  for (int t = 0; t < nT; ++t)
    if (!(T[t] > 0)) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  const int grid = g.num_sms * 4;
  CK(g.m0_partials.ensure((size_t)grid * M0_MAXT * 2));
  CK(g.m0_out.ensure(M0_MAXT * 2));
  for (int t0 = 0; t0 < nT; t0 += M0_MAXT) {
    M0Args a;
    memset(&a, 0, sizeof a);
    a.sys = g.sys;
    a.moment = moment;
    a.inv_mu = 1.0 / g.mu;
    a.inv_II = g.sys == SYS_HEAR ? 0.0 : 1.0 / g.II;
    a.Rmin = p->sampler_Rmin;
    a.Rmax = p->sampler_Rmax;
    a.pair_state = p->pair_state;
    m0_set_temperatures(a, T + t0, std::min(M0_MAXT, nT - t0));
    a.n_samples = n_samples;
    a.offset = sample_offset;
    a.seed = seed;
    int rc = (moment == 2) ? launch_m2(a, grid, g.m0_partials.p)
                           : launch_m0(a, grid, precision_mode == HH_PRECISION_MIXED, g.m0_partials.p);
    if (rc) return rc;
    m0_finalize_kernel<<<1, 32, 0, g.st>>>(g.m0_partials.p, grid, g.m0_out.p);
    CK(cudaGetLastError());
    double out[M0_MAXT * 2];
    CK(cudaMemcpyAsync(out, g.m0_out.p, sizeof out, cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    for (int t = 0; t < a.nT; ++t) {
      sum_w[t0 + t] = out[2 * t];
      if (sum_w2) sum_w2[t0 + t] = out[2 * t + 1];
    }
  }
  return HH_OK;
}

// moment m[t] = scale <w> and its one-sigma error from the sums over n samples
static void moment_from_sums(const double *sw, const double *sw2, int nT, uint64_t n, double scale, double *m,
                             double *err) {
  for (int t = 0; t < nT; ++t) {
    const double mean = sw[t] / double(n);
    const double var = sw2[t] / double(n) - mean * mean;
    m[t] = scale * mean;
    if (err) err[t] = scale * sqrt(std::max(var, 0.0) / double(n));
  }
}

int hh_cuda_m0(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
               uint64_t seed, int precision_mode, double *m, double *err) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (!m || nT < 1) return HH_E_INVALID_ARGUMENT;
  std::vector<double> sw(nT), sw2(nT);
  int rc = hh_cuda_moment_sums(p, T, nT, n_samples, 0, seed, 0, precision_mode, sw.data(), sw2.data());
  if (rc) return rc;
  const double scale = HH_ZEROCOEFF * 4.0 * HH_PI * (p->sampler_Rmax - p->sampler_Rmin);
  moment_from_sums(sw.data(), sw2.data(), nT, n_samples, scale, m, err);
  return HH_OK;
}

int hh_cuda_m2(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples, uint64_t seed,
               double *m, double *err) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (!m || nT < 1) return HH_E_INVALID_ARGUMENT;
  std::vector<double> sw(nT), sw2(nT);
  int rc = hh_cuda_moment_sums(p, T, nT, n_samples, 0, seed, 2, HH_PRECISION_FP64, sw.data(), sw2.data());
  if (rc) return rc;
  const double scale = HH_SECONDCOEFF * 4.0 * HH_PI * (p->sampler_Rmax - p->sampler_Rmin);
  moment_from_sums(sw.data(), sw2.data(), nT, n_samples, scale, m, err);
  return HH_OK;
}

int hh_cuda_vegas(const hh_calc_params *p, int integrand, double T, uint64_t niterations, uint64_t npoints,
                  uint64_t seed, double *m, double *q) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (g.sys == SYS_CH4CO2) return HH_E_UNSUPPORTED_SYSTEM;  // no CH4-CO2 moment integrand
  if (!p || !m || !(T > 0) || niterations == 0 || npoints < 2) return HH_E_INVALID_ARGUMENT;
  if (integrand != VEGAS_INTEGRAND_M0 && integrand != VEGAS_INTEGRAND_PF) return HH_E_INVALID_ARGUMENT;
  if (!(p->sampler_Rmin > 0) || !(p->sampler_Rmax > p->sampler_Rmin)) return HH_E_INVALID_ARGUMENT;
  if (p->pair_state < 1 || p->pair_state > 3) return HH_E_INVALID_ARGUMENT;
  if (niterations > (uint64_t)1 << 20 || npoints > ((uint64_t)1 << 62) / niterations) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  const int D = g.QP;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)g.num_sms * 4,
                                                                  (npoints + VEGAS_THREADS - 1) / VEGAS_THREADS));
  CK(g.vg_edges.ensure((size_t)D * (VEGAS_NB + 1)));
  CK(g.vg_sums.ensure(2 * (size_t)grid));
  CK(g.vg_hist.ensure((size_t)D * VEGAS_NB));
  std::vector<double> edges((size_t)D * (VEGAS_NB + 1)), hist((size_t)D * VEGAS_NB), sums(2 * (size_t)grid);
  for (int d = 0; d < D; ++d)
    for (int k = 0; k <= VEGAS_NB; ++k) edges[(size_t)d * (VEGAS_NB + 1) + k] = double(k) / VEGAS_NB;
  VegasArgs a;
  memset(&a, 0, sizeof a);
  a.s.sys = g.sys;
  a.s.mu = g.mu;
  a.s.II = g.II;
  a.s.Rmin = p->sampler_Rmin;
  a.s.Rmax = p->sampler_Rmax;
  a.s.pair_state = p->pair_state;
  a.D = D;
  a.integrand = integrand;
  a.inv_kT = HH_HKT / T;
  a.n = npoints;
  a.seed = seed;
  a.edges = g.vg_edges.p;
  a.sums = g.vg_sums.p;
  a.hist = g.vg_hist.p;
  // weighted average of the iterations after the first (hep::accumulate of results
  // begin() + 1 .. end(), src/hep_hawaii.cpp:352), weights 1 / variance
  double wsum = 0.0, wv = 0.0, first_v = 0.0, first_e = 0.0;
  for (uint64_t it = 0; it < niterations; ++it) {
    CK(cudaMemcpyAsync(g.vg_edges.p, edges.data(), edges.size() * sizeof(double), cudaMemcpyHostToDevice, g.st));
    CK(cudaMemsetAsync(g.vg_hist.p, 0, hist.size() * sizeof(double), g.st));
    a.id0 = it * npoints;
    int rc = g.sys == SYS_HEAR ? launch_vegas<SYS_HEAR>(a, grid)
             : g.sys == SYS_N2AR ? launch_vegas<SYS_N2AR>(a, grid)
                                 : launch_vegas<SYS_CO2AR>(a, grid);
    if (rc) return rc;
    CK(cudaMemcpyAsync(sums.data(), g.vg_sums.p, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, g.st));
    CK(cudaMemcpyAsync(hist.data(), g.vg_hist.p, hist.size() * sizeof(double), cudaMemcpyDeviceToHost, g.st));
    CK(cudaStreamSynchronize(g.st));
    double S = 0.0, S2 = 0.0;
    for (int b = 0; b < grid; ++b) {
      S += sums[2 * b];
      S2 += sums[2 * b + 1];
    }
    const double n = double(npoints);
    const double mean = S / n;
    const double var = std::max(S2 / n - mean * mean, 0.0) / (n - 1.0);  // variance of the mean
    if (it == 0) {
      first_v = mean;
      first_e = sqrt(var);
    } else if (var > 0.0) {
      wsum += 1.0 / var;
      wv += mean / var;
    }
    if (it + 1 < niterations) vegas_refine(edges, hist, D, 1.5);
  }
  if (niterations == 1 || !(wsum > 0.0)) {
    *m = first_v;
    if (q) *q = first_e;
  } else {
    *m = wv / wsum;
    if (q) *q = sqrt(1.0 / wsum);
  }
  return HH_OK;
}

// the transform's kernels on g.st: pack, log2(2N) Stockham passes, finish
void idct_enqueue(size_t N, double dt) {
  const long long L = 2 * (long long)N;
  const int tb = 256;
  idct_pack_kernel<<<(unsigned)((L + tb - 1) / tb), tb, 0, g.st>>>(g.f_cf.p, (long long)N, dt, g.f_a.p);
  idct_pack2_kernel<<<(unsigned)((N + tb - 1) / tb), tb, 0, g.st>>>(g.f_cf.p, (long long)N, g.f_a.p);
  double2 *x = g.f_a.p, *y = g.f_b.p;
  for (long long s = 1; s < L; s *= 2) {
    stockham_pass_kernel<<<(unsigned)((L / 2 + tb - 1) / tb), tb, 0, g.st>>>(x, y, L, s);
    std::swap(x, y);
  }
  idct_finish_kernel<<<(unsigned)((N + tb - 1) / tb), tb, 0, g.st>>>(x, (long long)N, dt, g.f_nu.p,
                                                                      g.f_sf.p);
}

int hh_cuda_idct_cf_to_sf(double *cf, size_t N, double dt, double *nu, double *sf) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (!cf || !nu || !sf || !(dt > 0)) return HH_E_INVALID_ARGUMENT;
  if (N == 0 || (N & (N - 1))) return HH_E_NOT_POWER_OF_TWO;
  for (size_t i = 0; i < N; ++i)
    if (cf[i] != cf[i]) return HH_E_INVALID_ARGUMENT;  // the reference exits on NaN input
  CK(cudaSetDevice(g.device));
  long long L = 2 * (long long)N;
  CK(g.f_cf.ensure(N));
  CK(g.f_nu.ensure(N));
  CK(g.f_sf.ensure(N));
  CK(g.f_a.ensure(L));
  CK(g.f_b.ensure(L));
  // the ~log2(2N) + 3 small kernels are launch-bound: they are captured once per
  // (N, dt, buffers) into a CUDA graph and replayed
  const void *bufs[5] = {g.f_cf.p, g.f_nu.p, g.f_sf.p, g.f_a.p, g.f_b.p};
  bool same = g.idct_exec && g.idct_N == N && g.idct_dt == dt;
  for (int i = 0; i < 5; ++i) same = same && (g.idct_bufs[i] == bufs[i]);
  if (!same) {
    if (g.idct_exec) cudaGraphExecDestroy(g.idct_exec);
    g.idct_exec = nullptr;
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(g.st, cudaStreamCaptureModeThreadLocal));
    idct_enqueue(N, dt);
    CK(cudaStreamEndCapture(g.st, &graph));
    const cudaError_t e = cudaGraphInstantiate(&g.idct_exec, graph, 0);
    cudaGraphDestroy(graph);
    CK(e);
    g.idct_N = N;
    g.idct_dt = dt;
    for (int i = 0; i < 5; ++i) g.idct_bufs[i] = bufs[i];
  }
  (void)L;
  CK(cudaMemcpyAsync(g.f_cf.p, cf, N * sizeof(double), cudaMemcpyHostToDevice, g.st));
  CK(cudaGraphLaunch(g.idct_exec, g.st));
  CK(cudaMemcpyAsync(nu, g.f_nu.p, N * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(sf, g.f_sf.p, N * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  CK(cudaMemcpyAsync(cf, g.f_cf.p, N * sizeof(double), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return HH_OK;
}

int hh_cuda_mt_stream(uint32_t seed, uint64_t n, uint32_t *out) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (!out && n) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  int rc = reseed(seed);
  if (rc) return rc;
  rc = ensure_words((long long)n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(out, g.words[g.cur].p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  return reseed(seed);
}

namespace {
// body-frame N2-Ar dipole at (R, T) as each precision path evaluates it
__global__ void n2ar_dip_probe_kernel(const N2arDipFold *F, const float4 *tab, const double *R, const double *T,
                                      long long n, int mixed, double *out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double c = cos(T[i]), s = sin(T[i]);
  const N2arDipBody<double> d = mixed ? n2ar_dip_body_mixed(tab, F, R[i], c, fabs(s)) : n2ar_dip_body(F, R[i], c);
  out[2 * i] = d.dx;
  out[2 * i + 1] = d.dz;
}
}  // namespace

int hh_cuda_debug_n2ar_dipole(int precision, const double *R, const double *T, uint64_t n, double *out) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (g.sys != SYS_N2AR || !g.d_n2ar_tab) return HH_E_UNSUPPORTED_SYSTEM;
  if ((n && (!R || !T || !out)) || (precision != HH_PRECISION_FP64 && precision != HH_PRECISION_MIXED))
    return HH_E_INVALID_ARGUMENT;
  if (!n) return HH_OK;
  CK(cudaSetDevice(g.device));
  double *dR = nullptr, *dT = nullptr, *dO = nullptr;
  int rc = HH_OK;
  cudaError_t e = cudaMalloc(&dR, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dT, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dO, 2 * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(dR, R, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dT, T, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    n2ar_dip_probe_kernel<<<(unsigned)((n + 127) / 128), 128, 0, g.st>>>(
        g.d_n2ar_fold, g.d_n2ar_tab, dR, dT, (long long)n, precision == HH_PRECISION_MIXED, dO);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.st);
  if (e == cudaSuccess) e = cudaMemcpy(out, dO, 2 * n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    snprintf(g_errmsg, sizeof g_errmsg, "hh_cuda_debug_n2ar_dipole: %s", cudaGetErrorString(e));
    rc = HH_E_CUDA;
  }
  if (dR) cudaFree(dR);
  if (dT) cudaFree(dT);
  if (dO) cudaFree(dO);
  return rc;
}

int hh_cuda_debug_tuning(int *ch4_dip_s_fp64, int *ch4_dip_s_mixed) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (ch4_dip_s_fp64) *ch4_dip_s_fp64 = g.ch4_dip_s[0];
  if (ch4_dip_s_mixed) *ch4_dip_s_mixed = g.ch4_dip_s[1];
  return HH_OK;
}

int hh_cuda_debug_item_trace(uint32_t *out, uint64_t capacity_words) {
  g_trace_host = out;
  g_trace_cap = out ? capacity_words : 0;
  return HH_OK;
}

int hh_cuda_debug_inject(int traj, int dir, int k, int status) {
  if (status < 0 || status >= HH_ST_COUNT || dir < 0 || dir > 1) return HH_E_INVALID_ARGUMENT;
  if (traj < 0) {
    g_inject_item = g_inject_k = -1;
    g_inject_status = 0;
    return HH_OK;
  }
  g_inject_item = 2 * traj + dir;
  g_inject_k = k;
  g_inject_status = status;
  return HH_OK;
}

int hh_cuda_debug_traj_tuning(int precision, int set_warps, int set_handoff_div, int *warps, int *handoff_div) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (precision != HH_PRECISION_FP64 && precision != HH_PRECISION_MIXED) return HH_E_INVALID_ARGUMENT;
  TrajTune &tt = g.traj_tune[g.sys][precision == HH_PRECISION_MIXED ? 1 : 0];
  if (set_warps < 0 || set_handoff_div < 0) {
    tt.warps = tt.handoff_div = 0;
  } else if (set_warps > 0 || set_handoff_div > 0) {
    if (set_warps > 0 && set_warps != TRAJ_WARPS_CANDIDATES[0] && set_warps != TRAJ_WARPS_CANDIDATES[1])
      return HH_E_INVALID_ARGUMENT;
    if (set_handoff_div > 0 && set_handoff_div != 1 && set_handoff_div != 2 && set_handoff_div != 4)
      return HH_E_INVALID_ARGUMENT;
    const int dw = precision == HH_PRECISION_MIXED ? traj_warps<float>() : traj_warps<double>();
    tt.warps = set_warps > 0 ? set_warps : (tt.warps ? tt.warps : dw);
    tt.handoff_div = set_handoff_div > 0 ? set_handoff_div : (tt.handoff_div ? tt.handoff_div : 1);
  }
  if (warps) *warps = tt.warps;
  if (handoff_div) *handoff_div = tt.handoff_div;
  return HH_OK;
}

int hh_cuda_set_requantization(const hh_requantization *r) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (!r || r->mode == HH_REQ_NONE) {
    memset(&g.req, 0, sizeof g.req);
    return HH_OK;
  }
  if (r->mode != HH_REQ_INTEGER && r->mode != HH_REQ_HALFINTEGER) return HH_E_INVALID_ARGUMENT;
  if (r->torque_cache_len < 1 || r->torque_cache_len > 16383 || !(r->torque_limit > 0)) return HH_E_INVALID_ARGUMENT;
  // spin weights only for half-integer requantization (src/hawaii.c:3579-3593)
  if (r->mode == HH_REQ_INTEGER && (r->even_j_spin_weight > 0 || r->odd_j_spin_weight > 0))
    return HH_E_INVALID_ARGUMENT;
  g.req = *r;
  return HH_OK;
}

int hh_cuda_debug_set_ch4_dipole(int precision, int variant) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (precision != HH_PRECISION_FP64 && precision != HH_PRECISION_MIXED) return HH_E_INVALID_ARGUMENT;
  const bool mixed = precision == HH_PRECISION_MIXED;
  const bool ok = variant == 0 || variant == 1 || variant == 2 || (mixed && (variant == 4 || variant == CH4_DIP_TC));
  if (!ok) return HH_E_INVALID_ARGUMENT;
  g.ch4_dip_s[mixed ? 1 : 0] = variant;
  return HH_OK;
}

int hh_cuda_debug_set_defer(int mode, int *previous) {
  if (mode < -1 || mode > 2) return HH_E_INVALID_ARGUMENT;
  if (previous) *previous = g_defer;
  if (mode >= 0) g_defer = mode;
  return HH_OK;
}

int hh_cuda_debug_set_defer_overlap(int on, int *previous) {
  if (on < -1 || on > 1) return HH_E_INVALID_ARGUMENT;
  if (previous) *previous = g_defer_overlap;
  if (on >= 0) g_defer_overlap = on;
  return HH_OK;
}

int hh_cuda_debug_ch4co2_fold(int *n_batch, int *n_groups) {
  if (!g.init || !g.d_ch4_cd) return HH_E_NOT_INITIALIZED;
  if (n_batch) *n_batch = g.ch4_B;
  if (n_groups) *n_groups = g.ch4_groups;
  return HH_OK;
}

int hh_cuda_debug_kernel_ms(int enable, double *ms, uint64_t *launches, int n) {
  if (n < 0) return HH_E_INVALID_ARGUMENT;
  for (int i = 0; i < std::min(n, (int)HH_KT_COUNT); ++i) {
    if (ms) ms[i] = g_kt.ms[i];
    if (launches) launches[i] = g_kt.n[i];
  }
  g_kt = KernelTimer();
  g_kt.on = enable != 0;
  return HH_OK;
}

int hh_cuda_fma_peak(int precision, double *tflops) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (!tflops) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  const int iters = 1 << 15;
  double best = 0.0;
  CK(g.m0_out.ensure(M0_MAXT * 2));
  for (int rep = 0; rep < 4; ++rep) {
    int per_sm = 0;
    if (precision == HH_PRECISION_FP64)
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fma_peak_kernel<double>, 256, 0));
    else
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fma_peak_kernel<float>, 256, 0));
    int grid = per_sm * g.num_sms;
    CK(cudaEventRecord(g.ev[0], g.st));
    if (precision == HH_PRECISION_FP64)
      fma_peak_kernel<double><<<grid, 256, 0, g.st>>>(g.m0_out.p, iters, 0.999999, 1e-7);
    else
      fma_peak_kernel<float><<<grid, 256, 0, g.st>>>((float *)g.m0_out.p, iters, 0.999999f, 1e-7f);
    CK(cudaGetLastError());
    CK(cudaEventRecord(g.ev[1], g.st));
    CK(cudaEventSynchronize(g.ev[1]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, g.ev[0], g.ev[1]));
    double flops = double(grid) * 256.0 * iters * 16.0;
    best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  *tflops = best;
  return HH_OK;
}

// Allocation-free M0: the samples, kernels and result of hh_cuda_m0, with the
// block partials and results kept in g_m0_noalloc_scratch instead of buffers
// that grow on demand.  Every partial a launch reads was written by that
// launch, so only the result slots are cleared; a failed launch then cannot
// hand back an earlier call's numbers.
int hh_cuda_m0_noalloc(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
                       uint64_t seed, int precision_mode, double *m, double *err) {
  if (!g.init) return HH_E_NOT_INITIALIZED;
  if (g.sys == SYS_CH4CO2) return HH_E_UNSUPPORTED_SYSTEM;
  if (!p || !T || nT < 1 || !m || n_samples == 0) return HH_E_INVALID_ARGUMENT;
  if (nT > HH_M0_NOALLOC_MAX_T) return HH_E_SCRATCH_LIMIT;
  if (!(p->sampler_Rmin > 0) || !(p->sampler_Rmax > p->sampler_Rmin)) return HH_E_INVALID_ARGUMENT;
  if (p->pair_state < 1 || p->pair_state > 3) return HH_E_INVALID_ARGUMENT;
  if (precision_mode != HH_PRECISION_FP64 && precision_mode != HH_PRECISION_MIXED)
    return HH_E_INVALID_ARGUMENT;
  for (int t = 0; t < nT; ++t)
    if (!(T[t] > 0)) return HH_E_INVALID_ARGUMENT;
  CK(cudaSetDevice(g.device));
  double *scratch = nullptr;
  int rc = m0_noalloc_scratch(g.device, &scratch);
  if (rc) return rc;
  double *partials = scratch, *res = scratch + M0_NOALLOC_PARTIALS;
  const int grid = std::min(g.num_sms * 4, M0_NOALLOC_MAX_BLOCKS);
  const int n_chunks = (nT + M0_MAXT - 1) / M0_MAXT;
  CK(cudaMemsetAsync(res, 0, sizeof(double) * 2 * M0_MAXT * n_chunks, g.st));
  for (int c = 0; c < n_chunks; ++c) {
    const int t0 = c * M0_MAXT;
    M0Args a;
    memset(&a, 0, sizeof a);
    a.sys = g.sys;
    a.Rmin = p->sampler_Rmin;
    a.Rmax = p->sampler_Rmax;
    a.pair_state = p->pair_state;
    m0_set_temperatures(a, T + t0, std::min(M0_MAXT, nT - t0));
    a.n_samples = n_samples;
    a.offset = 0;
    a.seed = seed;
    rc = launch_m0(a, grid, precision_mode == HH_PRECISION_MIXED, partials);
    if (rc) return rc;
    m0_finalize_kernel<<<1, 32, 0, g.st>>>(partials, grid, res + 2 * (size_t)t0);
    CK(cudaGetLastError());
  }
  double out[2 * HH_M0_NOALLOC_MAX_T];
  CK(cudaMemcpyAsync(out, res, sizeof(double) * 2 * nT, cudaMemcpyDeviceToHost, g.st));
  CK(cudaStreamSynchronize(g.st));
  const double scale = HH_ZEROCOEFF * 4.0 * HH_PI * (p->sampler_Rmax - p->sampler_Rmin);
  for (int t = 0; t < nT; ++t) {
    double mean = out[2 * t] / double(n_samples);
    double var = out[2 * t + 1] / double(n_samples) - mean * mean;
    m[t] = scale * mean;
    if (err) err[t] = scale * sqrt(std::max(var, 0.0) / double(n_samples));
  }
  return HH_OK;
}

void hh_cuda_shutdown(void) {
  if (!g.init) return;
  cudaSetDevice(g.device);
  cudaStreamSynchronize(g.st);
  if (g.st2) cudaStreamSynchronize(g.st2);
  g.words[0].release();
  g.words[1].release();
  g.accept.release();
  g.consumed.release();
  g.qp_cand.release();
  g.energy.release();
  g.qp0.release();
  g.block_counts.release();
  g.cand_idx.release();
  g.scal.release();
  g.crln.release();
  g.counters.release();
  g.status_hist.release();
  g.queue.release();
  g.fail_flag.release();
  g.fail_list.release();
  g.fail_count.release();
  g.items.release();
  g.handoff.release();
  g.zf_a.release();
  g.zf_b.release();
  g.hcount.release();
  g.trace.release();
  g.sat_w.release();
  g.sat_wraw.release();
  g.rec.release();
  g.rec_mu.release();
  g.rec_len.release();
  g.rec_status.release();
  g.rec_sorted.release();
  g.seg_cnt.release();
  g.seg_w0.release();
  g.rec_nfail.release();
  g.zim_fail.release();
  g.pm_a.release();
  g.pm_b.release();
  g.pm_sf.release();
  g.m0_partials.release();
  g.m0_out.release();
  g.tune_crln.release();
  g.tune_cnt.release();
  g.vg_edges.release();
  g.vg_sums.release();
  g.vg_hist.release();
  g.f_cf.release();
  g.f_nu.release();
  g.f_sf.release();
  g.f_a.release();
  g.f_b.release();
  if (g.idct_exec) cudaGraphExecDestroy(g.idct_exec);
  if (g.d_tab) cudaFree(g.d_tab);
  if (g.d_n2ar_fold) cudaFree(g.d_n2ar_fold);
  if (g.d_n2ar_pes_d) cudaFree(g.d_n2ar_pes_d);
  if (g.d_n2ar_pes_f) cudaFree(g.d_n2ar_pes_f);
  if (g.d_n2ar_tab) cudaFree(g.d_n2ar_tab);
  if (g.d_ch4_cd) cudaFree(g.d_ch4_cd);
  if (g.d_ch4_cf) cudaFree(g.d_ch4_cf);
  if (g.d_ch4_y2) cudaFree(g.d_ch4_y2);
  if (g.d_ch4_meta) cudaFree(g.d_ch4_meta);
  if (g.d_ch4_tc) cudaFree(g.d_ch4_tc);
  if (g.d_ch4_tc_err) cudaFree(g.d_ch4_tc_err);
  if (g.d_mt) cudaFree(g.d_mt);
  if (g.d_mt_jump_seg) cudaFree(g.d_mt_jump_seg);
  if (g.d_mt_jump_coarse) cudaFree(g.d_mt_jump_coarse);
  g.mt_seg_states.release();
  for (auto &e : g.ev)
    if (e) cudaEventDestroy(e);
  if (g.st) cudaStreamDestroy(g.st);
  if (g.st2) cudaStreamDestroy(g.st2);
  if (g.st3) cudaStreamDestroy(g.st3);
  if (g.ev_bulk) cudaEventDestroy(g.ev_bulk);
  if (g.ev_eval1) cudaEventDestroy(g.ev_eval1);
  if (g.ev_sampled) cudaEventDestroy(g.ev_sampled);
  if (g.ev_pregen) cudaEventDestroy(g.ev_pregen);
  g = Ctx();
  m0_noalloc_forget();
}

}  // extern "C"
