// Sampler translation unit of libhh_cuda.so (built with -fmad=false).
#include "hh_internal.h"
#include "hh_sampler.cuh"

namespace hh {

cudaError_t launch_mt_seed(uint32_t seed, uint32_t *state, cudaStream_t st) {
  mt_seed_kernel<<<(MT_N + 255) / 256, 256, 0, st>>>(seed, state);
  return cudaGetLastError();
}

cudaError_t launch_mt_generate(uint32_t *state, uint32_t *out, long long n_blocks, cudaStream_t st) {
  if (n_blocks <= 0) return cudaSuccess;
  mt_generate_kernel<<<1, 256, 0, st>>>(state, out, n_blocks);
  return cudaGetLastError();
}

size_t mt_jump_smem() { return MT_JUMP_WIN * sizeof(uint32_t) + 10240 * sizeof(unsigned short); }

cudaError_t launch_mt_generate_segments(uint32_t *state, uint32_t *out, int n_seg, uint32_t *seg_states,
                                        const unsigned short *jump_seg, const unsigned short *jump_coarse,
                                        cudaStream_t st) {
  static_assert(HH_MT_JUMP_SEG_N <= 10240 && HH_MT_JUMP_COARSE_N <= 10240, "jump tables exceed the buffer");
  const size_t smem = mt_jump_smem();
  cudaError_t e = cudaFuncSetAttribute(mt_jump_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // segment 0 starts from the current state
  e = cudaMemcpyAsync(seg_states, state, MT_N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  const int n_coarse = (n_seg + HH_MT_COARSE - 1) / HH_MT_COARSE;
  // coarse chain on one CTA: states 0, C, 2C, ...; then every other segment state
  // by one jump from its interval's start (the fine tables follow the segment table
  // in the same buffer: mt_jump_fine_tables)
  mt_jump_chain_kernel<<<1, MT_JUMP_THREADS, smem, st>>>(seg_states, 0, HH_MT_COARSE, n_coarse - 1, n_seg,
                                                         jump_coarse, HH_MT_JUMP_COARSE_N);
  if (n_seg > 1) {
    e = cudaFuncSetAttribute(mt_jump_fine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    mt_jump_fine_kernel<<<n_coarse * (HH_MT_COARSE - 1), MT_JUMP_THREADS, smem, st>>>(
        seg_states, n_seg, jump_seg + MT_FINE_OFFSET, jump_seg + MT_FINE_OFFSET + (HH_MT_COARSE - 1) * HH_MT_JUMP_FINE_MAX);
  }
  mt_generate_segments_kernel<<<n_seg, 256, 0, st>>>(seg_states, out, n_seg, state);
  return cudaGetLastError();
}

// *seg holds the segment table, then the fine tables (x^(k J) mod phi, k = 1..31, rows
// of HH_MT_JUMP_FINE_MAX) and their lengths
cudaError_t upload_mt_jump_tables(unsigned short **seg, unsigned short **coarse) {
  const size_t n_seg_buf = MT_FINE_OFFSET + (HH_MT_COARSE - 1) * (size_t)HH_MT_JUMP_FINE_MAX + HH_MT_COARSE;
  cudaError_t e = cudaMalloc(seg, n_seg_buf * sizeof(unsigned short));
  if (e == cudaSuccess) e = cudaMalloc(coarse, HH_MT_JUMP_COARSE_N * sizeof(unsigned short));
  if (e == cudaSuccess)
    e = cudaMemcpy(*seg, hh_mt_jump_seg, sizeof hh_mt_jump_seg, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(*seg + MT_FINE_OFFSET, hh_mt_jump_fine, sizeof hh_mt_jump_fine, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(*seg + MT_FINE_OFFSET + (HH_MT_COARSE - 1) * HH_MT_JUMP_FINE_MAX, hh_mt_jump_fine_n,
                   sizeof hh_mt_jump_fine_n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(*coarse, hh_mt_jump_coarse, sizeof hh_mt_jump_coarse, cudaMemcpyHostToDevice);
  return e;
}

cudaError_t launch_candidates(int sys, double mu, double II, double T, double Rmin, double Rmax,
                              double pesmin, int pair_state, const Co2arTablesGlobal *gtab,
                              const uint32_t *words, long long n_words, long long word_base, int D,
                              long long n_cand, unsigned char *accept, unsigned char *consumed,
                              double *qp, double *energy, unsigned long long *first_irregular,
                              const SamplerExtra &x, cudaStream_t st) {
  SamplerArgs a{sys, mu, II, T, Rmin, Rmax, pesmin, pair_state, x};
  size_t smem = (sys == SYS_CO2AR) ? sizeof(Co2arTables<double>) : 0;
  long long blocks = (n_cand + 255) / 256;
  candidate_kernel<<<(unsigned)blocks, 256, smem, st>>>(a, gtab, words, n_words, word_base, D,
                                                         n_cand, accept, consumed, qp, energy,
                                                         first_irregular);
  return cudaGetLastError();
}

cudaError_t launch_sat_weights(int sys, double mu, double II, double pesmin, int pair_state,
                               const Co2arTablesGlobal *gtab, const double *qp, long long n, double T0,
                               const double *Ts, const double *ratio, int n_sat, double *w, double *wraw,
                               const SamplerExtra &x, cudaStream_t st) {
  if (n_sat < 1 || n_sat > SAT_MAX) return cudaErrorInvalidValue;
  SamplerArgs a{sys, mu, II, T0, 0.0, 0.0, pesmin, pair_state, x};
  SatArgs s;
  s.n_sat = n_sat;
  s.T0 = T0;
  for (int k = 0; k < n_sat; ++k) {
    s.Ts[k] = Ts[k];
    s.ratio[k] = ratio[k];
  }
  size_t smem = (sys == SYS_CO2AR) ? sizeof(Co2arTables<double>) : 0;
  long long blocks = (n + 255) / 256;
  sat_weight_kernel<<<(unsigned)blocks, 256, smem, st>>>(a, s, gtab, qp, n, w, wraw);
  return cudaGetLastError();
}

cudaError_t launch_compact(const unsigned char *accept, const double *qp_cand, long long n,
                           long long limit, int QP, long long out_base, long long out_cap,
                           double *qp_out, long long *cand_index_out, unsigned int *block_counts,
                           unsigned long long *total, cudaStream_t st) {
  long long blocks = (n + 1023) / 1024;
  count_kernel<<<(unsigned)blocks, 1024, 0, st>>>(accept, n, limit, block_counts);
  scan_kernel<<<1, 1024, 0, st>>>(block_counts, (int)blocks, total);
  scatter_kernel<<<(unsigned)blocks, 1024, 0, st>>>(accept, qp_cand, n, limit, block_counts, QP,
                                                     out_base, out_cap, qp_out, cand_index_out, 0);
  return cudaGetLastError();
}

}  // namespace hh
