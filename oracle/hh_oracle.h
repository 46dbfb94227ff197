/*
 * CPU oracle for the HAWAIIHYBRID trajectory hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64, single-stream restatement of
 * the reference algorithm (sampler, Hamilton's equations in the reference's
 * spherical coordinates, PES/IDS plugins, correlation_eval, ensemble sum, IDCT,
 * zeroth-moment Monte Carlo).  It is used by tests/, by the smoke check and by
 * the CPU-baseline leg of bench.py as the checker and the timed CPU baseline.
 * No product code path links or calls it.
 *
 * Pinning: the MT19937 stream, the He-Ar potential/dipole and the CO2-Ar
 * molecular-frame potential/dipole are checked against the reference's own
 * sources compiled under oracle/_ref (mtwist.c, HeAr.h, ai_pes_co2ar.c,
 * ai_ids_co2ar.cpp), the CF->SF transform against the reference's golden pair
 * tests/CF-F-He-Ar-1000.0.txt -> tests/SF-F-He-Ar-1000.0.txt.  The integrator
 * is an FP64 DOP853 at the reference's tolerance: SUNDIALS CVODE 5.2.0 is not
 * available, so per-trajectory states are pinned against converged solutions
 * (tighter tolerance) and not against CVODE itself.
 */
#ifndef HH_ORACLE_H_
#define HH_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { HHO_SYS_HEAR = 0, HHO_SYS_CO2AR = 1, HHO_SYS_N2AR = 2, HHO_SYS_CH4CO2 = 3 };
enum { HHO_PS_FREE_AND_METASTABLE = 1, HHO_PS_BOUND = 2, HHO_PS_ALL = 3 };

/* per-half-trajectory status codes (same numbering as the CUDA library) */
enum {
    HHO_OK = 0,
    HHO_ST_MAXSTEPS = 1,      /* more than max_steps internal steps between two samples */
    HHO_ST_H_UNDERFLOW = 2,   /* step size fell below 10 ulp(t) */
    HHO_ST_NAN_DIPOLE = 3,    /* NaN dipole component (reference: return 1) */
    HHO_ST_OVERFLOW = 4,      /* |mu0 . mu(t)| > 1e100 (reference: return 1) */
    HHO_ST_JUMP = 5,          /* |C_k / C_{k-1}| > 1e10 (reference: return 1) */
};

typedef struct {
    int system;      /* HHO_SYS_* */
    double mu;       /* reduced mass, a.u. */
    double II;       /* moment of inertia of the linear monomer, a.u. (CO2-Ar, N2-Ar; CO2 of CH4-CO2) */
    double II1[3];   /* principal moments of the rotor (CH4 of CH4-CO2), a.u. */
} hho_system;

typedef struct {
    int pair_state;          /* HHO_PS_* */
    double Rmin, Rmax;       /* sampler_Rmin, sampler_Rmax (bohr) */
    double pesmin;           /* Hartree */
    double sampling_time;    /* a.t.u. */
    size_t N;                /* MaxTrajectoryLength */
    double Rcut;             /* bohr */
    double rtol, atol;       /* integrator tolerances (cvode_tolerance) */
    double ppf_ratio;        /* partial_partition_function_ratio */
    long max_steps;          /* internal steps allowed between two samples */
    int zimmermann;          /* use_zimmermann_trick: hho_correlation_sum uses the Zimmermann estimate */
} hho_params;

typedef struct {
    long nsteps, nrej, nrhs, nsamples;
    int status_fwd, status_bwd;
    int failed;              /* 1 when the reference would return 1 (zero contribution) */
} hho_traj_stats;

/* ---- MT19937 (mtwist: mts_seed32 + mt_drand) ---- */
typedef struct { uint32_t mt[624]; int idx; } hho_mt;
void hho_mt_seed(hho_mt *s, uint32_t seed);
uint32_t hho_mt_u32(hho_mt *s);
double hho_mt_drand(hho_mt *s);
void hho_mt_stream(uint32_t seed, size_t n, uint32_t *out);

/* ---- Philox4x32-10 (Salmon et al., SC'11) ---- */
void hho_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- physics ---- */
int hho_qp_size(const hho_system *sys);
double hho_hear_V(double R);
double hho_hear_dV(double R);
double hho_hear_dip(double R);
/* molecular frame CO2-Ar: V in Hartree, derivatives in Hartree/bohr, Hartree/rad */
double hho_co2ar_V_mol(double R, double theta);
void hho_co2ar_dV_mol(double R, double theta, double *dR, double *dtheta);
void hho_co2ar_dip_mol(double R, double theta, double d[3]);
void hho_co2ar_lab_to_mol(const double *qlab, double *qmol);
void hho_co2ar_jacobian(const double *qlab, double *jac25);
/* N2-Ar PIP-NN: energy in cm^-1 (before the en_inf shift) from the distances
 * |N1-N2|, |N1-Ar|, |N2-Ar| with dE/dd; lab-frame V in Hartree; body-frame dipole */
double hho_n2ar_energy_cm(const double d[3], double dEdd[3]);
void hho_n2ar_pes_pip(const double *y, double *p, double *jac);
void hho_n2ar_dip_pip(const double *y, double *p);
double hho_n2ar_V_lab(const double *q);
void hho_n2ar_dip_mol(double R, double Theta, double dm[3]);
double hho_pes(const hho_system *sys, const double *q);
void hho_dpes(const hho_system *sys, const double *q, double *dVdq);
void hho_dipole(const hho_system *sys, const double *q, double d[3]);
void hho_rhs(const hho_system *sys, const double *y, double *dydt);
double hho_kinetic(const hho_system *sys, const double *qp);
double hho_hamiltonian(const hho_system *sys, const double *qp);
/* spherical phase point -> Cartesian (r, p[, u, j]); CH4-CO2: (r, p, quaternion of
 * the CH4 body -> lab rotation, u_CO2, L_CH4, j_CO2), 19 values */
void hho_qp_to_cart(const hho_system *sys, const double *qp, double *cart);
/* CH4-CO2: lab coordinates -> (R, PHI1K, THETA1K, PHI2K, THETA2K) (src/angles_handler.cpp:357-419),
 * the body-frame dipole (PES-IDS/ai_ids_ch4_co2.cpp:672-1067) and the stand-in potential */
void hho_ch4co2_lab_to_kal(const double *qlab, double *qkal);
void hho_ch4co2_dipole_kal(const double *qkal, double d[3]);
double hho_ch4co2_V_lab(const double *q);

/* ---- sampler (hawaii.c:1206-1421, 2976-2994) ---- */
/* draws one candidate; returns 1 when accepted (reject + pair-state filter);
 * *draws receives the number of MT words consumed */
int hho_candidate(hho_mt *s, const hho_system *sys, const hho_params *p, double T,
                  double *qp, double *energy, int *draws);
/* draws candidates until n accepted; qp_out[n*QP]; returns candidates used */
long hho_sample(uint32_t seed, const hho_system *sys, const hho_params *p, double T,
                size_t n, double *qp_out);

/* ---- integrator + correlation_eval (hawaii.c:2116-2347) ---- */
int hho_correlation_eval(const hho_system *sys, const hho_params *p, const double *qp0,
                         double *crln, hho_traj_stats *st);
/* PR_MU spectral function (src/hawaii.c:3148-3978), core: returns the trajectories counted,
 * sf[0..L) the unnormalised sum */
/* requantization of the linear monomer in PR_MU: mode 1 integer, 2 half-integer; torque
 * cache length and limit; even / odd spin weights (half-integer, both <= 0: weight 1) */
typedef struct { int mode, len; double limit, even_w, odd_w; } hho_req;
long hho_prmu_req(const hho_system *sys, const hho_params *p, double T, double R0, int allow_trunc,
                  uint32_t seed, size_t n, const hho_req *rq, double *sf, size_t L, double *qp_out);
long hho_prmu(const hho_system *sys, const hho_params *p, double T, double R0, int allow_trunc, uint32_t seed,
              size_t n, double *sf, size_t L, double *qp_out);
/* correlation_eval_zimmerman_trick (src/hawaii.c:1888-2114) */
int hho_correlation_eval_zimmermann(const hho_system *sys, const hho_params *p, const double *qp0,
                                    double *crln, hho_traj_stats *st);
/* both branches separately (mu0.mu(t_k), no ALU^3 / 2 scaling, no dropping) */
int hho_correlation_parts(const hho_system *sys, const hho_params *p, const double *qp0,
                          double *fw, double *bw, hho_traj_stats *st);
/* integrate one phase point to t_end (dense output at t_end) */
int hho_propagate(const hho_system *sys, const hho_params *p, const double *qp0,
                  double t_end, double *qp_out, long *nsteps);
/* ensemble: sum_i ppf * crln_i over n trajectories given initial conditions;
 * nthreads worker threads; stats (optional) per trajectory */
int hho_correlation_sum(const hho_system *sys, const hho_params *p, const double *qp0,
                        size_t n, int nthreads, double *crln_sum, hho_traj_stats *stats);

/* ---- CORRELATION_ARRAY (hawaii.c:2361-2793) ---- */
/* reweighting of one trajectory of energy E sampled at T0 to Ts[0..n_sat) (hawaii.c:2640-2664) */
void hho_array_weights(int pair_state, double pesmin, double T0, const double *Ts, int n_sat,
                       double E, double *w);
/* out[s][N] = sum_i w[i][s] * crln_i (w carries the partial partition function ratios) */
int hho_correlation_sum_array(const hho_system *sys, const hho_params *p, const double *qp0, size_t n,
                              int nthreads, const double *w, int n_sat, double *out);

/* ---- CF -> SF (hawaii.c:5401-5601); apodizes cf in place like the reference ---- */
int hho_idct_cf_to_sf(double *cf, size_t N, double dt, double *nu, double *sf);

/* ---- zeroth moment, plain MC over Philox samples ---- */
int hho_m0(const hho_system *sys, const hho_params *p, const double *T, int nT,
           uint64_t n_samples, uint64_t seed, uint64_t offset, int nthreads,
           double *wsum, double *wsq);
double hho_m0_scale(const hho_params *p);  /* ZeroCoeff * 4 pi (Rmax - Rmin) */
/* ---- VEGAS of the reference's integrand_M0 (integrand 0) / integrand_pf (1) ---- */
int hho_vegas(const hho_system *sys, const hho_params *p, int integrand, double T, uint64_t niter,
              uint64_t npoints, uint64_t seed, int nthreads, double *m, double *q);
/* ---- second moment on the same samples (momentum average at the sampled K) ---- */
int hho_m2(const hho_system *sys, const hho_params *p, const double *T, int nT,
           uint64_t n_samples, uint64_t seed, uint64_t offset, int nthreads,
           double *wsum, double *wsq);
double hho_m2_scale(const hho_params *p);  /* SecondCoeff * 4 pi (Rmax - Rmin) */
double hho_analytic_pf(const hho_system *sys, double T);

#ifdef __cplusplus
}
#endif
#endif
