// Initial-condition sampler on the GPU.
//
// The reference draws every candidate phase point from one MT19937 stream
// (thirdparty/mtwist.c, seeded by mt_seed32 in init_ms, src/hawaii.c:157-163)
// and consumes a fixed number of words per candidate (src/hawaii.c:1206-1421):
//   q_generator: R, Phi, Theta (+ phi1, theta1 for a linear monomer; + phi1,
//                theta1, psi1 of a rotor and phi2, theta2 of a second, linear monomer)
//   p_generator: 3 (+2, or +3+2) Box-Muller normals, 2 words each
//   reject:      1 word
// i.e. D = 10 (atom-atom), 16 (linear-atom) or 25 (rotor-linear) words.  A Box-Muller draw only
// retries when its first word is exactly 0 (log(0) = -inf).
//
// GPU mapping:
//  1. mt_generate: one CTA advances the MT state 624 words at a time with a
//     three-phase parallel refresh and writes the tempered words to HBM;
//  2. candidates: one thread per candidate c reads the words [c*D, (c+1)*D),
//     restates q_generator/p_generator/Hamiltonian/reject/pair-state filter in
//     FP64 with the reference's operation order, and flags acceptance;
//  3. count/scan/scatter: accepted candidates are compacted in candidate order,
//     which is the order the reference's while-loop accepts them.
// A zero word at a Box-Muller position shifts every later candidate's window:
// the candidate kernel reports the first such candidate and the host restarts
// the following round right after it.
//
// Long requests of the stream (the 100 K rejection step of CH4-CO2 takes about
// 1.5e9 words per call) are generated in segments of HH_MT_SEG_BLOCKS blocks, one
// CTA each, from segment start states found by jumping ahead (hh_mt_jump.h):
// a chain of coarse jumps (HH_MT_COARSE segments each) on one CTA, then the fine
// jumps of every coarse interval in parallel.  The words are the same as those of
// the sequential generator.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_consts.h"
#include "hh_internal.h"
#include "hh_mt_jump.h"
#include "hh_phase.cuh"
#include "hh_physics.cuh"
#include "hh_traj.cuh"

namespace hh {

__device__ __forceinline__ uint32_t mt_twist(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t y = (a & 0x80000000u) | (b & 0x7fffffffu);
  return c ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

// state[0..623] <- Knuth-69069 seeding (mts_seed32, thirdparty/mtwist.c:372-400):
// mt[0] = seed, mt[i] = 69069 * mt[i-1] (mod 2^32), i.e. 69069^i * seed
__global__ void mt_seed_kernel(uint32_t seed, uint32_t *state) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= MT_N) return;
  if (seed == 0) seed = 4357u;
  uint32_t p = 1u, b = 69069u;
  for (int e = i; e; e >>= 1) {
    if (e & 1) p *= b;
    b *= b;
  }
  state[i] = p * seed;
}

// Advance the generator by n_blocks refreshes, writing 624 tempered words per
// refresh to out.  One CTA of 256 threads; the state lives in shared memory.
// one refresh of the 624 words in shared memory, in place (three dependency
// phases); every thread of the CTA (>= 227 threads) calls it
__device__ __forceinline__ void mt_refresh_smem(uint32_t *mt) {
  const int tid = threadIdx.x;
  uint32_t v;
  if (tid < MT_N - MT_M) v = mt_twist(mt[tid], mt[tid + 1], mt[tid + MT_M]);
  __syncthreads();
  if (tid < MT_N - MT_M) mt[tid] = v;
  __syncthreads();
  {
    int i = tid + (MT_N - MT_M);
    if (tid < MT_N - MT_M) v = mt_twist(mt[i], mt[i + 1], mt[i - (MT_N - MT_M)]);
    __syncthreads();
    if (tid < MT_N - MT_M) mt[i] = v;
    __syncthreads();
  }
  {
    int i = tid + 2 * (MT_N - MT_M);
    if (i < MT_N) v = mt_twist(mt[i], mt[(i + 1) % MT_N], mt[i - (MT_N - MT_M)]);
    __syncthreads();
    if (i < MT_N) mt[i] = v;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) mt_generate_kernel(uint32_t *state, uint32_t *out,
                                                          long long n_blocks) {
  __shared__ uint32_t mt[MT_N];
  for (int i = threadIdx.x; i < MT_N; i += blockDim.x) mt[i] = state[i];
  __syncthreads();
  const int tid = threadIdx.x;
  for (long long b = 0; b < n_blocks; ++b) {
    uint32_t v;
    // phase A: i in [0, 227) depends on old words only
    if (tid < MT_N - MT_M) v = mt_twist(mt[tid], mt[tid + 1], mt[tid + MT_M]);
    __syncthreads();
    if (tid < MT_N - MT_M) mt[tid] = v;
    __syncthreads();
    // phase B: i in [227, 454) uses new words i-227 from phase A
    {
      int i = tid + (MT_N - MT_M);
      if (tid < MT_N - MT_M) v = mt_twist(mt[i], mt[i + 1], mt[i - (MT_N - MT_M)]);
      __syncthreads();
      if (tid < MT_N - MT_M) mt[i] = v;
      __syncthreads();
    }
    // phase C: i in [454, 624); the last word wraps to the new mt[0]
    {
      int i = tid + 2 * (MT_N - MT_M);
      if (i < MT_N) v = mt_twist(mt[i], mt[(i + 1) % MT_N], mt[i - (MT_N - MT_M)]);
      __syncthreads();
      if (i < MT_N) mt[i] = v;
      __syncthreads();
    }
    uint32_t *o = out + b * MT_N;
    for (int i = tid; i < MT_N; i += blockDim.x) o[i] = mt_temper(mt[i]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < MT_N; i += blockDim.x) state[i] = mt[i];
}

// Chains of jumps: CTA c starts from states[c * chain_stride] (a 624-word block
// state) and writes the states `step`, 2 step, ... n_jumps * step segments later to
// states[c * chain_stride + k * step], k = 1..n_jumps, stopping before index n_states.
// One jump of J words (bits: set-bit positions of x^J mod phi) XORs windows of the
// 19,937 + 623 stream words after the state, which are generated in shared memory.
constexpr int MT_JUMP_WIN = 33 * MT_N;  // the state and the 32 blocks after it
constexpr int MT_JUMP_THREADS = 640;
__global__ void __launch_bounds__(MT_JUMP_THREADS) mt_jump_chain_kernel(uint32_t *states, int chain_stride,
                                                                       int step, int n_jumps, int n_states,
                                                                       const unsigned short *bits, int n_bits) {
  extern __shared__ uint32_t jsm[];
  uint32_t *win = jsm;                                         // MT_JUMP_WIN words
  unsigned short *bs = reinterpret_cast<unsigned short *>(jsm + MT_JUMP_WIN);
  for (int i = threadIdx.x; i < n_bits; i += blockDim.x) bs[i] = bits[i];
  const long long base = (long long)blockIdx.x * chain_stride;
  for (int i = threadIdx.x; i < MT_N; i += blockDim.x) win[i] = states[base * MT_N + i];
  __syncthreads();
  for (int k = 1; k <= n_jumps; ++k) {
    const long long dst = base + (long long)k * step;
    if (dst >= n_states) break;
    // the 32 blocks after the state: block b + 1 from block b, refreshed in place in
    // a copy at its own position
    for (int b = 0; b < 32; ++b) {
      uint32_t *cur = win + (b + 1) * MT_N;
      for (int i = threadIdx.x; i < MT_N; i += blockDim.x) cur[i] = win[b * MT_N + i];
      __syncthreads();
      mt_refresh_smem(cur);
    }
    uint32_t acc = 0;
    if (threadIdx.x < MT_N) {
      const int j = threadIdx.x;
#pragma unroll 4
      for (int t = 0; t < n_bits; ++t) acc ^= win[bs[t] + j];
    }
    __syncthreads();
    if (threadIdx.x < MT_N) {
      win[threadIdx.x] = acc;
      states[dst * MT_N + threadIdx.x] = acc;
    }
    __syncthreads();
  }
}

// Fine jumps: CTA b computes segment s = (b / 31) * 32 + b % 31 + 1 (skipping the
// coarse states, which the chain made) by one jump of k = s % 32 segments from
// states[s - k] with the table of x^(k J) mod phi, so every segment state of a round
// is one jump deep instead of a chain of up to 31.
constexpr size_t MT_FINE_OFFSET = 10240;  // the fine tables' offset in the segment-table buffer
static_assert(HH_MT_JUMP_FINE_MAX <= 10240, "fine jump table exceeds the buffer");
__global__ void __launch_bounds__(MT_JUMP_THREADS) mt_jump_fine_kernel(uint32_t *states, int n_seg,
                                                                      const unsigned short *fine,
                                                                      const unsigned short *fine_n) {
  extern __shared__ uint32_t jsm[];
  uint32_t *win = jsm;                                         // MT_JUMP_WIN words
  unsigned short *bs = reinterpret_cast<unsigned short *>(jsm + MT_JUMP_WIN);
  constexpr int PER = HH_MT_COARSE - 1;
  const long long s = (long long)(blockIdx.x / PER) * HH_MT_COARSE + (blockIdx.x % PER) + 1;
  if (s >= n_seg) return;  // the whole block
  const int k = (int)(s % HH_MT_COARSE);
  const int n_bits = fine_n[k - 1];
  for (int i = threadIdx.x; i < n_bits; i += blockDim.x) bs[i] = fine[(size_t)(k - 1) * HH_MT_JUMP_FINE_MAX + i];
  const long long base = s - k;
  for (int i = threadIdx.x; i < MT_N; i += blockDim.x) win[i] = states[base * MT_N + i];
  __syncthreads();
  for (int b = 0; b < 32; ++b) {
    uint32_t *cur = win + (b + 1) * MT_N;
    for (int i = threadIdx.x; i < MT_N; i += blockDim.x) cur[i] = win[b * MT_N + i];
    __syncthreads();
    mt_refresh_smem(cur);
  }
  if (threadIdx.x < MT_N) {
    const int j = threadIdx.x;
    uint32_t acc = 0;
#pragma unroll 4
    for (int t = 0; t < n_bits; ++t) acc ^= win[bs[t] + j];
    states[s * MT_N + j] = acc;
  }
}

// Segment s: HH_MT_SEG_BLOCKS blocks from states[s], tempered words to
// out + s * HH_MT_SEG_BLOCKS * 624; the last segment's final block becomes the
// generator state.
__global__ void __launch_bounds__(256) mt_generate_segments_kernel(const uint32_t *states, uint32_t *out,
                                                                   int n_seg, uint32_t *final_state) {
  __shared__ uint32_t mt[MT_N];
  const int s = blockIdx.x;
  for (int i = threadIdx.x; i < MT_N; i += blockDim.x) mt[i] = states[(size_t)s * MT_N + i];
  __syncthreads();
  uint32_t *o = out + (size_t)s * HH_MT_SEG_BLOCKS * MT_N;
  for (int b = 0; b < HH_MT_SEG_BLOCKS; ++b) {
    mt_refresh_smem(mt);
    for (int i = threadIdx.x; i < MT_N; i += blockDim.x) o[(size_t)b * MT_N + i] = mt_temper(mt[i]);
  }
  __syncthreads();
  if (s == n_seg - 1)
    for (int i = threadIdx.x; i < MT_N; i += blockDim.x) final_state[i] = mt[i];
}

// reference operation order is kept; FP contraction is disabled for this code
// by building with -fmad=false on the sampler translation unit
__device__ __forceinline__ double mt_d(const uint32_t *w, long long &pos) {
  return double(w[pos++]) * (1.0 / 4294967296.0);
}

__device__ __forceinline__ double bm_normal(const uint32_t *w, long long &pos, long long limit,
                                            int &retries, bool &overrun) {
  for (;;) {
    if (pos + 2 > limit) { overrun = true; return 0.0; }
    double U = mt_d(w, pos);
    double V = mt_d(w, pos);
    double logU = log(U);
    if (isnan(logU) || isinf(logU)) { ++retries; continue; }
    return 1.0 * sqrt(-2 * logU) * cos(2.0 * HH_PI * V);
  }
}

// one thread per candidate; words of candidate c start at word_base + c*D
__global__ void __launch_bounds__(256) candidate_kernel(
    SamplerArgs a, const Co2arTablesGlobal *gtab, const uint32_t *words, long long n_words,
    long long word_base, int D, long long n_cand, unsigned char *accept, unsigned char *consumed,
    double *qp_out, double *energy_out, unsigned long long *first_irregular) {
  extern __shared__ unsigned char smem_raw[];
  Co2arTables<double> *tb = reinterpret_cast<Co2arTables<double> *>(smem_raw);
  if (a.sys == SYS_CO2AR) load_tables<double>(tb, gtab);
  __syncthreads();
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= n_cand) return;
  long long pos = word_base + c * D;
  const long long limit = n_words;
  int retries = 0;
  bool overrun = false;
  const int QP = (a.sys == SYS_HEAR) ? 6 : (a.sys == SYS_CH4CO2 ? 16 : 10);
  double qp[16];
  double RMIN = a.Rmin, RMAX = a.Rmax, T = a.T;
  // q_generator (src/hawaii.c:1232-1290)
  double R3 = mt_d(words, pos) * (RMAX * RMAX * RMAX - RMIN * RMIN * RMIN) + RMIN * RMIN * RMIN;
  qp[4] = pow(R3, 1.0 / 3.0);
  qp[0] = mt_d(words, pos) * 2.0 * HH_PI;
  qp[2] = acos(2.0 * mt_d(words, pos) - 1.0);
  if (a.sys == SYS_CH4CO2) {
    qp[6] = mt_d(words, pos) * 2.0 * HH_PI;
    qp[8] = acos(2.0 * mt_d(words, pos) - 1.0);
    qp[10] = mt_d(words, pos) * 2.0 * HH_PI;
    qp[12] = mt_d(words, pos) * 2.0 * HH_PI;
    qp[14] = acos(2.0 * mt_d(words, pos) - 1.0);
  } else if (a.sys != SYS_HEAR) {
    qp[6] = mt_d(words, pos) * 2.0 * HH_PI;
    qp[8] = acos(2.0 * mt_d(words, pos) - 1.0);
  }
  const bool prmu = a.x.prmu_R0 > 0.0;
  if (prmu) qp[4] = a.x.prmu_R0;
  // p_generator (src/hawaii.c:1292-1380)
  double sqrt_MUKT = sqrt(a.mu / HH_HKT * T);
  double sinTheta = sin(qp[2]);
  double x0 = bm_normal(words, pos, limit, retries, overrun);
  double x1 = bm_normal(words, pos, limit, retries, overrun);
  double x2 = bm_normal(words, pos, limit, retries, overrun);
  qp[1] = sqrt_MUKT * qp[4] * sinTheta * x0;
  qp[3] = sqrt_MUKT * qp[4] * x1;
  qp[5] = sqrt_MUKT * x2;
  if (a.sys == SYS_CH4CO2) {
    // p_generator_rotor (src/hawaii.c:1305-1327)
    double sqrt_IIx = sqrt(a.x.II1[0] / HH_HKT * T);
    double sqrt_IIy = sqrt(a.x.II1[1] / HH_HKT * T);
    double sqrt_IIz = sqrt(a.x.II1[2] / HH_HKT * T);
    double sin_theta = sin(qp[8]), cos_theta = cos(qp[8]);
    double sin_psi = sin(qp[10]), cos_psi = cos(qp[10]);
    double r0 = bm_normal(words, pos, limit, retries, overrun);
    double r1 = bm_normal(words, pos, limit, retries, overrun);
    double r2 = bm_normal(words, pos, limit, retries, overrun);
    qp[7] = sqrt_IIx * sin_theta * sin_psi * r0 + sqrt_IIy * sin_theta * cos_psi * r1 + sqrt_IIz * cos_theta * r2;
    qp[9] = sqrt_IIx * cos_psi * r0 - sqrt_IIy * sin_psi * r1;
    qp[11] = sqrt_IIz * r2;
    // p_generator_linear_molecule of the second monomer (src/hawaii.c:1292-1303)
    double sqrt_IIKT = sqrt(a.II / HH_HKT * T);
    double sin_t2 = sin(qp[14]);
    double m0 = bm_normal(words, pos, limit, retries, overrun);
    double m1 = bm_normal(words, pos, limit, retries, overrun);
    qp[13] = sqrt_IIKT * sin_t2 * m1;
    qp[15] = sqrt_IIKT * m0;
  } else if (a.sys != SYS_HEAR) {
    double sqrt_IIKT = sqrt(a.II / HH_HKT * T);
    double sin_theta = sin(qp[8]);
    double m0 = bm_normal(words, pos, limit, retries, overrun);
    double m1 = bm_normal(words, pos, limit, retries, overrun);
    qp[7] = sqrt_IIKT * sin_theta * m1;
    qp[9] = sqrt_IIKT * m0;
  }
  if (!prmu && pos + 1 > limit) overrun = true;
  bool acc = false;
  double E = 0.0;
  if (prmu) {
    if (qp[5] > 0.0) qp[5] = -qp[5];
    acc = !overrun;
  } else if (!overrun) {
    // Hamiltonian, then reject() (src/hawaii.c:1382-1421), then the filter (2981-2994)
    double kin = kinetic(a, qp);
    double pot = potential(a, tb, qp);
    E = kin + pot;
    double u = mt_d(words, pos);
    double Mval = exp(-a.pesmin * HH_HKT / T);
    double M = 1.5 * Mval;
    double proposal = exp(-kin * HH_HKT / T);
    double desired = exp(-(kin + pot) * HH_HKT / T);
    double weight = desired / proposal / M;
    acc = !(weight < u);
    if (a.pair_state == 1 && E < 0.0) acc = false;
    if (a.pair_state == 2 && E > 0.0) acc = false;
  }
  if (retries || overrun) atomicMin(first_irregular, (unsigned long long)c);
  accept[c] = acc ? 1 : 0;
  consumed[c] = overrun ? 0 : (unsigned char)(pos - (word_base + c * D));
  for (int i = 0; i < QP; ++i) qp_out[c * QP + i] = qp[i];
  energy_out[c] = E;
}

// ---- CORRELATION_ARRAY reweighting (src/hawaii.c:2640-2676) ----
// One thread per trajectory: its energy at the base temperature T0 (the same
// Hamiltonian the sampler's filter used) and, per satellite temperature Ts,
//   weight = exp(-E HkT / T0 / Ts (T0 - Ts)) / WTT,
// with WTT = exp(-pesmin HkT / T0 / Ts (T0 - Ts)) for bound pairs below T0 and 1
// otherwise, and weight = 0 for free pairs above T0.  w[i][s] = weight * ratio_s
// feeds C(t); wraw[i][s] = weight feeds nstar.
struct SatArgs {
  int n_sat;
  double T0;
  double Ts[SAT_MAX];
  double ratio[SAT_MAX];
};

__global__ void __launch_bounds__(256) sat_weight_kernel(SamplerArgs a, SatArgs s,
                                                         const Co2arTablesGlobal *gtab,
                                                         const double *qp, long long n, double *w,
                                                         double *wraw) {
  extern __shared__ unsigned char smem_raw[];
  Co2arTables<double> *tb = reinterpret_cast<Co2arTables<double> *>(smem_raw);
  if (a.sys == SYS_CO2AR) load_tables<double>(tb, gtab);
  __syncthreads();
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int QP = (a.sys == SYS_HEAR) ? 6 : (a.sys == SYS_CH4CO2 ? 16 : 10);
  double q[16];
  for (int c = 0; c < QP; ++c) q[c] = qp[i * QP + c];
  const double E = kinetic(a, q) + potential(a, tb, q);
  const double T0 = s.T0;
  for (int k = 0; k < s.n_sat; ++k) {
    const double T = s.Ts[k];
    double WTT = 1.0;
    if (a.pair_state == 2 && T < T0) WTT = exp(-a.pesmin * HH_HKT / T0 / T * (T0 - T));
    double weight = exp(-E * HH_HKT / T0 / T * (T0 - T)) / WTT;
    if (a.pair_state == 1 && T > T0) weight = 0.0;
    w[i * s.n_sat + k] = weight * s.ratio[k];
    wraw[i * s.n_sat + k] = weight;
  }
}

// ---- ordered compaction of accepted candidates ----
__global__ void __launch_bounds__(1024) count_kernel(const unsigned char *accept, long long n,
                                                     long long limit, unsigned int *block_counts) {
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int v = (c < n && c <= limit) ? accept[c] : 0;
  int cnt = __syncthreads_count(v);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = cnt;
}

// exclusive scan of block counts in one CTA (n_blocks is small)
__global__ void __launch_bounds__(1024) scan_kernel(unsigned int *counts, int n_blocks,
                                                    unsigned long long *total) {
  __shared__ unsigned int partial[1024];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n_blocks; base += 1024) {
    int i = base + threadIdx.x;
    unsigned int v = (i < n_blocks) ? counts[i] : 0u;
    partial[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      unsigned int t = (threadIdx.x >= off) ? partial[threadIdx.x - off] : 0u;
      __syncthreads();
      partial[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n_blocks) counts[i] = (unsigned int)(carry + partial[threadIdx.x] - v);
    __syncthreads();
    if (threadIdx.x == 1023) carry += partial[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(1024) scatter_kernel(const unsigned char *accept,
                                                       const double *qp_cand, long long n,
                                                       long long limit, const unsigned int *offsets,
                                                       int QP, long long out_base, long long out_cap,
                                                       double *qp_out, long long *cand_index_out,
                                                       long long cand_base) {
  __shared__ unsigned int warp_tot[32];
  long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int v = (c < n && c <= limit) ? accept[c] : 0;
  unsigned int ballot = __ballot_sync(0xffffffffu, v);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned int before = __popc(ballot & ((1u << lane) - 1u));
  if (lane == 0) warp_tot[warp] = __popc(ballot);
  __syncthreads();
  unsigned int woff = 0;
  for (int w = 0; w < warp; ++w) woff += warp_tot[w];
  if (v) {
    long long dst = out_base + offsets[blockIdx.x] + woff + before;
    if (dst < out_cap) {
      for (int i = 0; i < QP; ++i) qp_out[dst * QP + i] = qp_cand[c * QP + i];
      if (cand_index_out) cand_index_out[dst] = cand_base + c;
    }
  }
}

}  // namespace hh
