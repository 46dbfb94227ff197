// Launch helpers shared between the translation units of libhh_cuda.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hh_traj.cuh"

namespace hh {

constexpr int MT_N = 624;  // MT19937 state words
constexpr int MT_M = 397;  // recurrence offset
constexpr int SAT_MAX = 64;  // satellite temperatures of one CORRELATION_ARRAY call

// rotor-linear (CH4-CO2) sampler inputs: the rotor's principal moments and the
// stand-in surface's pair constants
struct SamplerExtra {
  double II1[3];
  Ch4Co2Lj lj;
  // PR_MU draws (R0 > 0): R := R0 before the momenta, pR made inward, no rejection
  // step and no pair-state filter (src/hawaii.c:3566-3573)
  double prmu_R0;
};

// sampler (hh_sampler.cu, compiled without floating-point contraction so the
// reference's operation order is kept)
cudaError_t launch_mt_seed(uint32_t seed, uint32_t *state, cudaStream_t st);
cudaError_t launch_mt_generate(uint32_t *state, uint32_t *out, long long n_blocks, cudaStream_t st);
// n_seg segments of MT_SEG_BLOCKS blocks each from the current state (segment start
// states found by jumping ahead; seg_states holds n_seg * 624 words); the state
// advances past the last segment
constexpr long long MT_SEG_BLOCKS = 2048;  // HH_MT_SEG_BLOCKS of hh_mt_jump.h
cudaError_t launch_mt_generate_segments(uint32_t *state, uint32_t *out, int n_seg, uint32_t *seg_states,
                                        const unsigned short *jump_seg, const unsigned short *jump_coarse,
                                        cudaStream_t st);
cudaError_t upload_mt_jump_tables(unsigned short **seg, unsigned short **coarse);
cudaError_t launch_candidates(int sys, double mu, double II, double T, double Rmin, double Rmax,
                              double pesmin, int pair_state, const Co2arTablesGlobal *gtab,
                              const uint32_t *words, long long n_words, long long word_base, int D,
                              long long n_cand, unsigned char *accept, unsigned char *consumed,
                              double *qp, double *energy, unsigned long long *first_irregular,
                              const SamplerExtra &x, cudaStream_t st);
// CORRELATION_ARRAY weights of n trajectories (qp at the base temperature T0)
cudaError_t launch_sat_weights(int sys, double mu, double II, double pesmin, int pair_state,
                               const Co2arTablesGlobal *gtab, const double *qp, long long n, double T0,
                               const double *Ts, const double *ratio, int n_sat, double *w, double *wraw,
                               const SamplerExtra &x, cudaStream_t st);
cudaError_t launch_compact(const unsigned char *accept, const double *qp_cand, long long n,
                           long long limit, int QP, long long out_base, long long out_cap,
                           double *qp_out, long long *cand_index_out, unsigned int *block_counts,
                           unsigned long long *total, cudaStream_t st);

}  // namespace hh
