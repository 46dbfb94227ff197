/*
 * hh_cuda.h -- C ABI of the B200 trajectory library (libhh_cuda.so).
 *
 * Drop-in boundary for HAWAIIHYBRID's trajectory hot path.  The host keeps the
 * reference's C driver, .conf parsing, plugin loading and CF/SF writers; the
 * per-trajectory loop, the zeroth-moment integral and the CF->SF transform call
 * into this library instead.  Plain C types only; every function returns
 * HH_OK (0) or a negative HH_E_* code; output buffers are caller-owned host
 * memory; device memory is owned by the library.  Calls are synchronous and
 * must come from one host thread.
 *
 * Replaced reference interfaces (file:line in the reference tree):
 *   hh_cuda_init             setup_pes/setup_dipole plugin binding (src/driver.c:3097-3181)
 *                            + init_ms (src/hawaii.c:173-270)
 *   hh_cuda_seed             mt_seed32 in init_ms (src/hawaii.c:157-163)
 *   hh_cuda_sample           q_generator/p_generator/reject + pair-state filter
 *                            (src/hawaii.c:1232-1421, 2976-2994)
 *   hh_cuda_correlation      the accumulation loop of calculate_correlation_and_save
 *                            (src/hawaii.c:2970-3012) with correlation_eval
 *                            (src/hawaii.c:2116-2347) per trajectory
 *   hh_cuda_correlation_multi  niterations passes of that loop (src/hawaii.c:2970-3040)
 *   hh_cuda_correlation_array  calculate_correlation_array_and_save's accumulation loop
 *                            (src/hawaii.c:2361-2793; reweighting 2640-2676)
 *   hh_cuda_correlation_ic   correlation_eval over caller-supplied phase points
 *                            (src/hawaii.c:2116-2347, accumulation 3008)
 *   hh_cuda_m0               c_mpi_perform_integration(..., INTEGRAND_M0, ...)
 *                            (src/hep_hawaii.h:16, src/hep_hawaii.cpp:148-201) and
 *                            the M0 scaling of src/driver.c:3425-3431
 *   hh_cuda_idct_cf_to_sf    SFnc idct_cf_to_sf(CFnc) (src/hawaii.h:648,
 *                            src/hawaii.c:5569-5601)
 */
#ifndef HH_CUDA_H_
#define HH_CUDA_H_

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define HH_OK 0
#define HH_E_NOT_INITIALIZED (-1)
#define HH_E_INVALID_ARGUMENT (-2)
#define HH_E_CUDA (-3)
#define HH_E_UNSUPPORTED_SYSTEM (-4)
#define HH_E_OUT_OF_MEMORY (-5)
#define HH_E_NOT_POWER_OF_TWO (-6)
#define HH_E_SAMPLER (-7)
#define HH_E_NO_DEVICE (-8)

/* MonomerType values of the reference (src/hawaii.h:183-190) */
#define HH_MONOMER_ATOM 0
#define HH_MONOMER_LINEAR_MOLECULE 4
#define HH_MONOMER_ROTOR 6

/* PairState of the reference (src/hawaii.h:290-300) */
#define HH_PAIR_STATE_FREE_AND_METASTABLE 1
#define HH_PAIR_STATE_BOUND 2
#define HH_PAIR_STATE_ALL 3

/* device surfaces; a plugin .so names its surface by exporting
 * int hh_cuda_system_id(void) next to pes_lab/dpes_lab/dipole_lab */
#define HH_SYSTEM_HE_AR 1
#define HH_SYSTEM_CO2_AR 2
#define HH_SYSTEM_N2_AR 3   /* PIP-NN surfaces of PES-IDS/ai_pes_n2_ar_pip_nn.cpp, ai_ids_n2_ar_pip_nn.cpp */
#define HH_SYSTEM_CH4_CO2 4 /* ROTOR (CH4, II1) + LINEAR_MOLECULE (CO2, II2): the dipole of
                               PES-IDS/ai_ids_ch4_co2.cpp; the reference tree has no source for its
                               CH4-CO2 PES (PES-IDS/ai_pes_ch4_co2.h), so trajectories run on a
                               site-site Lennard-Jones stand-in whose minimum is the config's pesmin.
                               No M0 (HH_E_UNSUPPORTED_SYSTEM). */

/* precision modes */
#define HH_PRECISION_FP64 0  /* FP64 surfaces and stages: the plain drop-in path */
#define HH_PRECISION_MIXED 1 /* FP32 surfaces and stages, FP64 state */

typedef struct {
    int system_id;          /* HH_SYSTEM_* */
    double mu;              /* pair reduced mass, a.u. (pair_reduced_mass) */
    int monomer1_type;      /* HH_MONOMER_* */
    int monomer2_type;
    double II1[3];          /* inertia of monomer 1, a.u. (II = {...}) */
    double II2[3];
} hh_system_desc;

typedef struct {
    int pair_state;                 /* HH_PAIR_STATE_* (PAIR_STATE) */
    double sampler_Rmin;            /* bohr */
    double sampler_Rmax;            /* bohr */
    double pesmin;                  /* Hartree */
    double sampling_time;           /* a.t.u. */
    size_t MaxTrajectoryLength;
    double Rcut;                    /* bohr */
    double cvode_tolerance;         /* rtol = atol of the FP64 path */
    double partial_partition_function_ratio;
    double mixed_tolerance;         /* rtol = atol of the mixed path; 0 selects 1e-8 */
    long max_steps;                 /* internal steps between two samples; 0 selects 50000 */
    int use_zimmermann_trick;       /* use_zimmermann_trick: C_i(s) = sum_{c<N} d[c].d[c+s] ALU^3 / N
                                       over the dipole series of both branches
                                       (correlation_eval_zimmerman_trick, src/hawaii.c:1888-2114);
                                       only with HH_PAIR_STATE_BOUND (src/hawaii.c:2942-2945) */
} hh_calc_params;

typedef struct {
    uint64_t n_candidates;          /* sampler candidates drawn */
    uint64_t n_accepted;
    uint64_t n_steps;               /* accepted integrator steps (all half-trajectories) */
    uint64_t n_rejected_steps;
    uint64_t n_rhs;                 /* right-hand-side evaluations */
    uint64_t n_samples;             /* dipole samples */
    uint64_t n_dense;               /* steps that needed dense output */
    uint64_t n_failed;              /* trajectories dropped like the reference's `return 1` */
    uint64_t status[8];             /* per half-trajectory: OK, MAXSTEPS, H_UNDERFLOW,
                                       NAN_DIPOLE, OVERFLOW, JUMP */
    double sample_ms;               /* device time of the sampler (CUDA events) */
    double traj_ms;                 /* device time of the trajectory kernel(s) */
    double total_ms;                /* device time of the whole call */
    uint64_t n_kernel_launches;     /* kernels this library launched for the call */
} hh_stats;

/* Select the device and the surface; uploads coefficient tables.  Re-callable. */
int hh_cuda_init(int device, const hh_system_desc *sys);

/* Reseed the sampler stream exactly like mt_seed32(seed) in init_ms. */
int hh_cuda_seed(uint32_t seed);

/* Draw n accepted initial phase points (reference layout, QP_SIZE doubles each)
 * from the stream; seed > 0 reseeds first, seed == 0 continues the stream. */
int hh_cuda_sample(const hh_calc_params *p, double T, uint32_t seed, uint64_t n,
                   double *qp_out, uint64_t *n_candidates);

/* One CORRELATION_SINGLE iteration: sample n_accept phase points (seed as in
 * hh_cuda_sample), integrate both branches of every trajectory and return
 * crln_sum[k] = sum_i ppf * crln_i[k] (length MaxTrajectoryLength) and the
 * trajectory count to add to ntraj. */
int hh_cuda_correlation(const hh_calc_params *p, double T, uint32_t seed, uint64_t n_accept,
                        int precision_mode, double *crln_sum, double *ntraj, hh_stats *stats);

/* n_iterations consecutive iterations of n_per_iteration trajectories each
 * (the stream order of the reference's iteration loop), integrated in one
 * persistent launch so that the long-lived trajectories of one iteration run
 * beside the others: crln_sums[i][k] (n_iterations x MaxTrajectoryLength) and
 * ntraj[i] per iteration. */
int hh_cuda_correlation_multi(const hh_calc_params *p, double T, uint32_t seed,
                              uint64_t n_per_iteration, uint32_t n_iterations, int precision_mode,
                              double *crln_sums, double *ntraj, hh_stats *stats);

/* The reference's CORRELATION_SINGLE run repeated at nT temperatures (one driver
 * run per TEMPERATURE, src/hawaii.c:2970-3012 each): n_per_T phase points are
 * sampled at T[0], then T[1], ... from one stream (seed as in hh_cuda_sample), and
 * all nT * n_per_T trajectories are integrated together, so the long trajectories
 * of the cold sets run beside the short ones of the hot sets.  crln_sums[i][k]
 * (nT x MaxTrajectoryLength) and ntraj[i] per temperature. */
int hh_cuda_correlation_temperatures(const hh_calc_params *p, const double *T, int nT, uint32_t seed,
                                     uint64_t n_per_T, int precision_mode, double *crln_sums,
                                     double *ntraj, hh_stats *stats);

/* Requantization of monomer 1 in PR_MU (no effect on the other paths): the monomer
 * types LINEAR_MOLECULE_REQ_INTEGER / LINEAR_MOLECULE_REQ_HALFINTEGER (src/hawaii.h:183-190)
 * with the Monomer's torque_cache_len and torque_limit (src/hawaii.h:210-235) and
 * CalcParams' even_j_spin_weight / odd_j_spin_weight (src/hawaii.h:336-337).  The
 * linear monomer's |j| is requantized to the nearest integer (find_closest_integer) or
 * half-integer (find_closest_half_integer, src/hawaii.c:360-393) when its trajectory
 * starts and, while the switch is on, at every sample (trajectory_apply_requantization
 * in make_step, src/trajectory.c:93-183); the torque at each sample switches it on
 * after torque_cache_len torques <= torque_limit and off after as many >= it
 * (src/hawaii.c:3604-3662).  Half-integer runs weight each trajectory by the even or
 * odd spin weight of round(j_ini - 1.5) when either is positive.  A NULL argument or
 * mode HH_REQ_NONE switches it off.  Linear-monomer systems (CO2-Ar, N2-Ar). */
#define HH_REQ_NONE 0
#define HH_REQ_INTEGER 1
#define HH_REQ_HALFINTEGER 2
typedef struct {
    int mode;                   /* HH_REQ_* */
    size_t torque_cache_len;    /* 1 .. 16383 */
    double torque_limit;        /* a.u., > 0 */
    double even_j_spin_weight;  /* HH_REQ_HALFINTEGER only; both <= 0: weight 1 */
    double odd_j_spin_weight;
} hh_requantization;
int hh_cuda_set_requantization(const hh_requantization *r);

/* PR_MU spectral function (calculate_spectral_function_using_prmu_representation_and_save,
 * src/hawaii.c:3148-3978), with the requantization of hh_cuda_set_requantization when it is
 * on: n_traj phase points drawn as
 * q_generator, R := R0, p_generator with pR made inward (no rejection step); each trajectory
 * is integrated forward with the dipole sampled at t = (k+1) dt, k = 0..N-1, until R > R0;
 * its Connes-apodized dipole components are Fourier transformed and
 * sf[i] = sum SF_COEFF pR/mu sum_c |F_c(i)|^2 on nu[i] = i / (dt ATU c N) (cm^-1) for the
 * *n_freq = (int)(approx_freq_max / step) + 1 frequencies (sf_len must hold them).  A
 * trajectory whose integration fails, or that is still inside R0 after N samples (unless
 * allow_truncating), is skipped; *ntraj counts the others (divide sf by it, as the reference's
 * final loop does).  N must be a power of two.  Not available for CH4-CO2. */
int hh_cuda_prmu(const hh_calc_params *p, double T, double R0, double approx_freq_max, int allow_truncating,
                 uint32_t seed, uint64_t n_traj, int precision_mode, double *nu, double *sf, size_t sf_len,
                 size_t *n_freq, double *ntraj, hh_stats *stats);

/* CORRELATION_ARRAY: n_accept trajectories sampled at base_T, each added to the
 * C(t) of every satellite temperature sat_T[s] with the reference's reweighting
 * w = exp(-E HkT / base_T / T (base_T - T)) / WTT (0 for free pairs above base_T)
 * times ppf_ratios[s]: crln_sums[s][k] (n_sat x MaxTrajectoryLength),
 * nstar[s] = sum of the weights, *ntraj = n_accept.  n_sat <= 64; the pair state
 * must be FREE_AND_METASTABLE or BOUND. */
int hh_cuda_correlation_array(const hh_calc_params *p, double base_T, const double *sat_T,
                              const double *ppf_ratios, int n_sat, uint32_t seed, uint64_t n_accept,
                              int precision_mode, double *crln_sums, double *nstar, double *ntraj,
                              hh_stats *stats);

/* Same as hh_cuda_correlation, for caller-supplied initial phase points qp0[n][QP_SIZE]. */
int hh_cuda_correlation_ic(const hh_calc_params *p, const double *qp0, uint64_t n,
                           int precision_mode, double *crln_sum, hh_stats *stats);

/* M0 at nT temperatures from n_samples phase-space points (Philox stream
 * `seed`), all temperatures in one launch: m[t] (same units as the reference's
 * "T = ... => M0") and its one-sigma statistical error err[t]. */
int hh_cuda_m0(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
               uint64_t seed, int precision_mode, double *m, double *err);

/* M2 at nT temperatures from n_samples phase-space points (Philox stream `seed`),
 * all temperatures in one launch, in FP64: m[t] in the units of the reference's
 * "T = ... => M2" and its one-sigma statistical error err[t].  Replaces
 * calculate_M2 / mpi_calculate_M2 (src/hawaii.c:1524-1617, 1740-1856) and the VEGAS
 * integrand_M2 (src/hep_hawaii.cpp:228-330): the same phase-space samples as
 * hh_cuda_m0, with the momentum average of |dmu/dt|^2 taken at the sampled kinetic
 * energy.  HH_E_UNSUPPORTED_SYSTEM for CH4-CO2. */
int hh_cuda_m2(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
               uint64_t seed, double *m, double *err);

/* Per-temperature sums of the moment integrand over the Philox samples
 * [sample_offset, sample_offset + n_samples) of stream `seed`: sum_w[t] = sum of w,
 * sum_w2[t] = sum of w^2 (may be NULL), moment 0 (M0, either precision) or 2 (M2,
 * FP64).  This is the per-rank part of the reference's MPI moment integrals
 * (mpi_calculate_M0 / mpi_calculate_M2, src/hawaii.c:1620-1738, 1740-1856: each rank
 * integrates its own points, rank 0 sums the (m, q) pairs): ranks take disjoint
 * counter ranges and the sums add, so M = scale * (sum over ranks of sum_w) / n_total
 * with scale = ZeroCoeff (SecondCoeff) * 4 pi (Rmax - Rmin).  hh_cuda_m0 and
 * hh_cuda_m2 are this call at offset 0 followed by that division. */
int hh_cuda_moment_sums(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
                        uint64_t sample_offset, uint64_t seed, int moment, int precision_mode,
                        double *sum_w, double *sum_w2);

/* VEGAS integration of the reference's phase-space integrands:
 * c_mpi_perform_integration(ms, integrand, params, T, niterations, npoints, &m, &q)
 * (src/hep_hawaii.h:16, src/hep_hawaii.cpp:332-389, driven by src/driver.c:3390-3447 for
 * M0).  integrand HH_INTEGRAND_M0 (integrand_M0, src/hep_hawaii.cpp:148-201) or
 * HH_INTEGRAND_PF (integrand_pf, 122-146) over the unit hypercube through the
 * reference's transform_variables map; niterations iterations of npoints samples
 * each (Philox stream `seed`), the grid (128 bins per dimension) refined after every
 * iteration by Lepage's algorithm (alpha 1.5); m and q are the 1/variance-weighted
 * average of the iterations after the first and its error, in the reference's units
 * before the driver's scaling (M0 = m * ZeroCoeff / pf_analytic).  FP64.  ATOM + ATOM
 * and LINEAR_MOLECULE + ATOM systems; HH_E_UNSUPPORTED_SYSTEM for CH4-CO2. */
#define HH_INTEGRAND_M0 0
#define HH_INTEGRAND_PF 1
int hh_cuda_vegas(const hh_calc_params *p, int integrand, double T, uint64_t niterations, uint64_t npoints,
                  uint64_t seed, double *m, double *q);

/* Allocation-free M0 (no counterpart in the reference).
 *
 * Same arguments, samples and results as hh_cuda_m0, but the call allocates no
 * device memory: its block partials and results live in one fixed array
 * compiled into the library (HH_M0_NOALLOC_SCRATCH_BYTES per device).  It is
 * meant for hosts that must not allocate once their run has started: a job that
 * shares the GPU with an allocator holding most of HBM in its pool (a PyTorch
 * caching allocator, a process under an MPS memory limit), where a cudaMalloc
 * in the middle of a temperature scan can fail, and a host that overlaps this
 * call with work on other streams, which the cudaFree of a growing buffer would
 * stall until the whole device drains.
 *
 * Limits: nT <= HH_M0_NOALLOC_MAX_T, else HH_E_SCRATCH_LIMIT and nothing runs.
 * hh_cuda_init must have been called (it allocates the surface tables once).
 * The array is placed in device memory when the library's module loads, at the
 * latest with the first kernel launch after hh_cuda_init.  The first call after
 * the library is brought up (the first hh_cuda_init, or the first one after
 * hh_cuda_shutdown) looks up the array's device address (cudaGetSymbolAddress),
 * and that lookup must not fall inside a stream capture, so make that first call
 * during set-up.  hh_cuda_shutdown forgets the address, so a context torn down
 * (cudaDeviceReset) after hh_cuda_shutdown and brought up again by hh_cuda_init
 * never reuses a stale one.  There is one array per device: calls whose GPU work
 * overlaps (e.g. from two host threads) race on it. */
#define HH_E_SCRATCH_LIMIT (-9)
#define HH_M0_NOALLOC_MAX_T 256
#define HH_M0_NOALLOC_SCRATCH_BYTES (8 * (1024 * 16 * 2 + 2 * HH_M0_NOALLOC_MAX_T))
int hh_cuda_m0_noalloc(const hh_calc_params *p, const double *T, int nT, uint64_t n_samples,
                       uint64_t seed, int precision_mode, double *m, double *err);

/* CF and SF text files: write_correlation_function_ext / write_spectral_function_ext
 * (src/hawaii.c:4150-4284) with the same bytes (header, then "%.2f %.10e" or
 * "%.10f   %.10e" lines; data divided by ntraj unless normalized), formatted in
 * parallel on the host threads and written with one fwrite, then flushed and fsync'd.
 * fp is an open stream; it is truncated first.  Returns the characters written or a
 * negative HH_E_* code.  No device is needed. */
long hh_write_correlation_function_ext(FILE *fp, const double *t, const double *data, size_t len,
                                       double Temperature, double ntraj, int normalized);
long hh_write_spectral_function_ext(FILE *fp, const double *nu, const double *data, size_t len,
                                    double Temperature, double ntraj, int normalized);

/* CF -> SF: apodizes cf in place (as the reference does), N a power of two. */
int hh_cuda_idct_cf_to_sf(double *cf, size_t N, double dt, double *nu, double *sf);

const char *hh_cuda_strerror(int code);

/* Test and diagnostic entry points (no counterpart in the reference):
 * hh_cuda_mt_stream writes the first n words of the MT19937 stream of `seed`
 * as the sampler consumes them (the stream is left reseeded with `seed`);
 * hh_cuda_debug_inject makes branch `dir` (0 forward, 1 backward) of
 * trajectory `traj` of the next correlation calls end with status `status`
 * (1..5) at sample k, as if its integrator or dipole had failed there; traj < 0
 * switches injection off. */
int hh_cuda_mt_stream(uint32_t seed, uint64_t n, uint32_t *out);
int hh_cuda_debug_inject(int traj, int dir, int k, int status);
/* registers a host buffer of capacity_words uint32 that the next correlation
 * call fills with (steps, samples, start ns, end ns) per half-trajectory item
 * (item 2*traj + dir); NULL unregisters */
int hh_cuda_debug_item_trace(uint32_t *out, uint64_t capacity_words);
/* Diagnostic (no counterpart in the reference; the reference evaluates the N2-Ar
 * dipole in PES-IDS/ai_ids_n2_ar_pip_nn.cpp:83-127): the body-frame dipole
 * (d_x, d_z) of the N2-Ar system at n points (R[i] bohr, T[i] = angle between the
 * intermolecular axis and the N2 axis) as the given precision path evaluates it,
 * into out[2 n]: the FP64 network, or the mixed path's FP32 table. */
int hh_cuda_debug_n2ar_dipole(int precision, const double *R, const double *T, uint64_t n, double *out);
/* Diagnostic (no counterpart in the reference): the CH4-CO2 dipole kernel variant
 * that the tuner picked for the FP64 and the mixed path on the first record-path call
 * of this context: records per lane (1, 2 or 4) of the CUDA-core kernel, -1 for the
 * tensor-core kernel (mixed path only), 0 before that call. */
int hh_cuda_debug_tuning(int *ch4_dip_s_fp64, int *ch4_dip_s_mixed);
/* Tuning knob (no counterpart in the reference): fixes the CH4-CO2 dipole kernel
 * variant of `precision` (values as above; 0 lets the tuner time them again on the
 * next record-path call).  The environment variable HH_CH4_DIP_S (1, 2, 4 or "tc")
 * fixes the first pick instead. */
int hh_cuda_debug_set_ch4_dipole(int precision, int variant);

/* Diagnostic (no counterpart in the reference): where the mixed path's plain C(t)
 * evaluates the dipoles at the sample times.  mode 0: inside the trajectory kernel;
 * 1 (the default, or the environment variable HH_DEFER_SAMPLES): CO2-Ar deferred to
 * the sample kernels (the trajectory kernel writes one dense-output context per step
 * and tests only R > Rcut); 2: CO2-Ar and N2-Ar deferred; -1 leaves the mode as it is.
 * *previous (if not NULL) receives the mode before the call.  Both placements give the
 * same samples and C(t) up to the order of the FP64 sums. */
int hh_cuda_debug_set_defer(int mode, int *previous);
/* Tuning knob (no counterpart in the reference): with deferred samples, whether the
 * contexts written by the bulk trajectory launch are evaluated while the solo launch
 * (the last open trajectories) runs, on a second stream.  on 1 (the default, or the
 * environment variable HH_DEFER_OVERLAP), 0 after the solo launch; -1 leaves it as it
 * is.  *previous (if not NULL) receives the setting before the call.  Both give the
 * same C(t) up to the order of the FP64 sums. */
int hh_cuda_debug_set_defer_overlap(int on, int *previous);

/* Diagnostic (no counterpart in the reference): device time per kernel class.
 * While switched on, every kernel of the classes below is bracketed by CUDA events
 * and waited for (launches of a call then run one after another, so switch it on
 * for a measurement call, not for a timed one).  Each call copies out the
 * milliseconds and launches accumulated since the previous call (n entries at
 * most, HH_KT_COUNT in all), resets them and sets the timer to `enable`. */
#define HH_KT_TRAJ_BULK 0   /* traj_kernel, bulk launch */
#define HH_KT_TRAJ_SOLO 1   /* traj_kernel, solo launch (last open items, one per warp) */
#define HH_KT_CH4_DIPOLE 2  /* CH4-CO2 batched dipole kernel */
#define HH_KT_CH4_SORT 3    /* CH4-CO2 record sort (count, scan, scatter) */
#define HH_KT_CH4_CORR 4    /* CH4-CO2 per-sample tests and C(t) sums */
#define HH_KT_MOMENT 5      /* M0 / M2 kernel */
#define HH_KT_SAMPLES 6     /* deferred samples: dipoles, per-sample tests and C(t) sums */
#define HH_KT_ITEM_START 7  /* precomputed item starts of the deferred-sample path */
#define HH_KT_COUNT 8
int hh_cuda_debug_kernel_ms(int enable, double *ms, uint64_t *launches, int n);
/* Tuning knob (no counterpart in the reference): the trajectory launch's block
 * shape (bulk kernel warps per block, 4 or 8) and hand-off threshold (the launch
 * switches from 32 trajectories per warp to one when at most (solo warp slots) /
 * handoff_div items are open; 1, 2 or 4) for the bound system and `precision`.  The
 * library times the candidates on the first plain-C(t) launch of at least 16,384
 * half-trajectories per system and precision (environment HH_TRAJ_WARPS,
 * HH_TRAJ_HANDOFF_DIV fix them instead).  set_* > 0 fixes a value, set_* < 0
 * forgets the pick (tuned again on the next large call), 0 leaves it; *warps and
 * *handoff_div receive the current pick (0: not tuned yet). */
int hh_cuda_debug_traj_tuning(int precision, int set_warps, int set_handoff_div, int *warps, int *handoff_div);
/* Diagnostic (no counterpart in the reference): shape of the CH4-CO2 dipole's
 * coefficient stream (batches of 4 entries per radial piece, and the (Y1,
 * component, cos/sin) groups they form); HH_E_NOT_INITIALIZED before a CH4-CO2
 * hh_cuda_init. */
int hh_cuda_debug_ch4co2_fold(int *n_batch, int *n_groups);

/* Diagnostic (no counterpart in the reference): measured FMA throughput of the
 * CUDA cores in TFLOP/s (precision HH_PRECISION_FP64 or, for FP32,
 * HH_PRECISION_MIXED), the denominator of the trajectory kernels' roofline. */
int hh_cuda_fma_peak(int precision, double *tflops);

/* Release all device memory of the library. */
void hh_cuda_shutdown(void);

#ifdef __cplusplus
}
#endif

#endif /* HH_CUDA_H_ */
