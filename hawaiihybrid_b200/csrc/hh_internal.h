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
};

// sampler (hh_sampler.cu, compiled without floating-point contraction so the
// reference's operation order is kept)
cudaError_t launch_mt_seed(uint32_t seed, uint32_t *state, cudaStream_t st);
cudaError_t launch_mt_generate(uint32_t *state, uint32_t *out, long long n_blocks, cudaStream_t st);
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
