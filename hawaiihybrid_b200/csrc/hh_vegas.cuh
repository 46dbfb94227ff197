// VEGAS integration of the phase-space moment integrands on the GPU, the estimator
// that c_mpi_perform_integration drives (src/hep_hawaii.cpp:332-363 through hep-mc 0.7,
// a third-party library absent from the reference tree; its published algorithm,
// G. P. Lepage, J. Comput. Phys. 27 (1978) 192, is restated here and in the host
// refinement of hh_api.cu).
//
// The integrand is the reference's: a point x of the unit hypercube of dimension
// QP_SIZE maps to a phase point by transform_variables (src/hep_hawaii.cpp:8-120),
// including its use of x[0] for both R = 1/x[0] and Phi = 2 pi x[0], and
//   integrand_M0 = jac |mu(q)|^2 exp(-H / kT)   (src/hep_hawaii.cpp:148-201)
//   integrand_pf = jac exp(-H / kT)              (src/hep_hawaii.cpp:122-146)
// are zero outside [sampler_Rmin, sampler_Rmax] and outside the pair state.
//
// One iteration = one launch: sample i of iteration `it` draws its uniforms from
// Philox4x32-10 at counter (id_lo, id_hi, block, 0) with id = it * npoints + i, maps
// each through the separable grid (NB bins per dimension: bin b = floor(u NB), x =
// e[b] + (u NB - b)(e[b+1] - e[b]), weight prod_d NB (e[b+1] - e[b])), and accumulates
// F = f * weight into per-thread FP64 sums of F and F^2 and the per-bin sums of F^2
// of every dimension (shared-memory histogram per block, then global atomics).  The
// host turns the sums into the iteration's estimate and refines the grid.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hh_m0.cuh"
#include "hh_phase.cuh"

namespace hh {

constexpr int VEGAS_NB = 128;   // bins per dimension
constexpr int VEGAS_MAXD = 10;  // QP_SIZE of the atom-atom and linear-atom systems
constexpr int VEGAS_THREADS = 256;

enum { VEGAS_INTEGRAND_M0 = 0, VEGAS_INTEGRAND_PF = 1 };

struct VegasArgs {
  SamplerArgs s;            // system, masses, R range, pair state (T unused)
  int D;                    // dimensions (QP_SIZE)
  int integrand;            // VEGAS_INTEGRAND_*
  double inv_kT;            // HkT / T
  uint64_t n, id0, seed;    // samples of this iteration, the first one's Philox index, key
  const double *edges;      // [D][NB + 1]
  double *sums;             // [gridDim.x][2]: sum F, sum F^2
  double *hist;             // [D][NB]: sum F^2 per bin (global, atomics)
};

// transform_variables (src/hep_hawaii.cpp:8-120) for ATOM + ATOM and LINEAR + ATOM
__device__ __forceinline__ double vegas_map(const double *x, int D, double *qp) {
  double jac = 1.0;
  qp[4] = 1.0 / x[0];  // R = 1/x0 (IR), jac R^2
  jac *= qp[4] * qp[4];
  qp[5] = tan(HH_PI * (x[5] - 0.5));  // pR
  jac *= HH_PI * (1.0 + qp[5] * qp[5]);
  qp[0] = x[0] * 2.0 * HH_PI;  // Phi from x[0] (the reference's IPHI = 0 index)
  jac *= 2.0 * HH_PI;
  qp[1] = tan(HH_PI * (x[1] - 0.5));  // pPhi
  jac *= HH_PI * (1.0 + qp[1] * qp[1]);
  qp[2] = x[2] * HH_PI;  // Theta
  jac *= HH_PI;
  qp[3] = tan(HH_PI * (x[3] - 0.5));  // pTheta
  jac *= HH_PI * (1.0 + qp[3] * qp[3]);
  if (D == 10) {
    qp[6] = x[6] * 2.0 * HH_PI;  // phi1
    jac *= 2.0 * HH_PI;
    qp[7] = tan(HH_PI * (x[7] - 0.5));
    jac *= HH_PI * (1.0 + qp[7] * qp[7]);
    qp[8] = x[8] * HH_PI;  // theta1
    jac *= HH_PI;
    qp[9] = tan(HH_PI * (x[9] - 0.5));
    jac *= HH_PI * (1.0 + qp[9] * qp[9]);
  }
  return jac;
}

template <int SYS>
__global__ void __launch_bounds__(VEGAS_THREADS) vegas_kernel(VegasArgs a, const Co2arTablesGlobal *gtab,
                                                              const void *dipnet) {
  extern __shared__ __align__(16) unsigned char vg_smem[];
  double *hist_s = reinterpret_cast<double *>(vg_smem);                 // [D][NB]
  double *edges_s = hist_s + VEGAS_MAXD * VEGAS_NB;                     // [D][NB + 1]
  unsigned char *tab_raw = reinterpret_cast<unsigned char *>(edges_s + VEGAS_MAXD * (VEGAS_NB + 1));
  Co2arTables<double> *tb = reinterpret_cast<Co2arTables<double> *>(tab_raw);
  N2arDipFold *fold = reinterpret_cast<N2arDipFold *>(tab_raw);
  const int D = a.D;
  for (int i = threadIdx.x; i < D * VEGAS_NB; i += blockDim.x) hist_s[i] = 0.0;
  for (int i = threadIdx.x; i < D * (VEGAS_NB + 1); i += blockDim.x) edges_s[i] = a.edges[i];
  if (SYS == SYS_CO2AR) load_tables<double>(tb, gtab);
  if (SYS == SYS_N2AR) load_words(fold, dipnet, sizeof(N2arDipFold));
  __syncthreads();
  const uint32_t k0 = (uint32_t)a.seed, k1 = (uint32_t)(a.seed >> 32);
  double sF = 0.0, cF = 0.0, sF2 = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const uint64_t id = a.id0 + i;
    uint32_t w[12];
    philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), 0u, 0u, k0, k1, w);
    philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), 1u, 0u, k0, k1, w + 4);
    philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), 2u, 0u, k0, k1, w + 8);
    double x[VEGAS_MAXD];
    int bin[VEGAS_MAXD];
    double wgt = 1.0;
#pragma unroll
    for (int d = 0; d < VEGAS_MAXD; ++d) {
      if (d < D) {
        const double u = (double(w[d]) + 0.5) * (1.0 / 4294967296.0);
        const double v = u * VEGAS_NB;
        const int b = min(int(v), VEGAS_NB - 1);
        const double lo = edges_s[d * (VEGAS_NB + 1) + b], hi = edges_s[d * (VEGAS_NB + 1) + b + 1];
        x[d] = lo + (v - double(b)) * (hi - lo);
        wgt *= double(VEGAS_NB) * (hi - lo);
        bin[d] = b;
      }
    }
    double qp[VEGAS_MAXD];
    const double jac = vegas_map(x, D, qp);
    double f = 0.0;
    const double R = qp[4];
    if (R >= a.s.Rmin && R <= a.s.Rmax) {
      const double H = kinetic(a.s, qp) + potential(a.s, tb, qp);
      const bool keep = a.s.pair_state == 1 ? !(H < 0.0) : (a.s.pair_state == 2 ? !(H > 0.0) : true);
      if (keep) {
        double dipsq = 1.0;
        if (a.integrand == VEGAS_INTEGRAND_M0) {
          double y[12];
          double d3[3];
          if (SYS == SYS_HEAR) {
            qp_to_state<SYS_HEAR>(qp, y);
            HeArSys<double, double, false> sys;
            sys.dipole(y, d3);
          } else {
            qp_to_state<SYS_CO2AR>(qp, y);
            const double q[6] = {y[0], y[1], y[2], y[6], y[7], y[8]};
            if (SYS == SYS_N2AR) {
              N2ArSys<double, double, false> sys;
              sys.fold = fold;
              sys.dtab = nullptr;
              sys.dipole(q, d3);
            } else {
              Co2ArSys<double, double, false> sys;
              sys.tb = tb;
              sys.dipole(q, d3);
            }
          }
          dipsq = d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2];
        }
        f = jac * dipsq * exp(-H * a.inv_kT);
      }
    }
    const double F = f * wgt;
    // compensated sum of F, plain sum of F^2
    const double yk = F - cF, tk = sF + yk;
    cF = (tk - sF) - yk;
    sF = tk;
    sF2 += F * F;
    if (F != 0.0) {
#pragma unroll
      for (int d = 0; d < VEGAS_MAXD; ++d)
        if (d < D) atomicAdd(&hist_s[d * VEGAS_NB + bin[d]], F * F);
    }
  }
  // block sums in a fixed order
  __shared__ double red[2][VEGAS_THREADS / 32];
  double v = sF - cF, vq = sF2;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, o);
    vq += __shfl_down_sync(0xffffffffu, vq, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = v;
    red[1][threadIdx.x >> 5] = vq;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, q = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      s += red[0][i];
      q += red[1][i];
    }
    a.sums[2 * blockIdx.x] = s;
    a.sums[2 * blockIdx.x + 1] = q;
  }
  for (int i = threadIdx.x; i < D * VEGAS_NB; i += blockDim.x)
    if (hist_s[i] != 0.0) atomicAdd(&a.hist[i], hist_s[i]);
}

template <int SYS> constexpr size_t vegas_smem() {
  return sizeof(double) * (VEGAS_MAXD * VEGAS_NB + VEGAS_MAXD * (VEGAS_NB + 1)) +
         (SYS == SYS_CO2AR ? sizeof(Co2arTables<double>) : SYS == SYS_N2AR ? sizeof(N2arDipFold) : 0);
}

}  // namespace hh
