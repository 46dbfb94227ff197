/* Stand-in CH4-CO2 potential energy surface.
 *
 * The reference's CH4-CO2 PES (PES-IDS/ai_pes_ch4_co2.h declares pes_ch4co2 and
 * dpes_ch4co2) has no implementation in its source tree, so trajectories of this
 * system run on a synthetic surface of the same shape: a site-site 12-6
 * Lennard-Jones sum between the five sites of a rigid CH4 (C at the centre of
 * mass, H at r_CH (+-1, +-1, +-1)/sqrt(3) with an even number of minus signs, in
 * the molecule's body frame) and the three sites of a rigid CO2 (C at the centre
 * of mass, O at +-r_CO along the molecular axis).  The CO2 centre sits at the
 * intermolecular vector R from the CH4 centre.  Site parameters are common
 * force-field values (OPLS methane, TraPPE carbon dioxide) with Lorentz-Berthelot
 * mixing; every well depth is multiplied by HH_CH4CO2_LJ_SCALE so that the global
 * minimum equals the pesmin of the reference's CH4-CO2 configuration,
 * -1.562522273622102e-03 Hartree (example_configs/CF-F-CH4-CO2.conf:25), which the
 * sampler's rejection step uses as its bound (src/hawaii.c:1382-1421).  The scale
 * was found by minimising the unscaled surface over R and the five angles from
 * 300 random starts (minimum -1.1664304263022e-03 Hartree at R = 6.342 bohr).
 *
 * Plain C: included by the CPU oracle and by the CUDA host code.
 */
#ifndef HH_CH4CO2_STANDIN_H_
#define HH_CH4CO2_STANDIN_H_

#include <math.h>

#define HH_CH4CO2_BOHR_A 0.529177210903        /* angstrom per bohr */
#define HH_CH4CO2_HARTREE_K 315775.02480407     /* kelvin per Hartree */
#define HH_CH4CO2_RCH (1.087 / HH_CH4CO2_BOHR_A) /* bohr */
#define HH_CH4CO2_RCO (1.160 / HH_CH4CO2_BOHR_A) /* bohr */
#define HH_CH4CO2_LJ_SCALE 1.3395760590501438

/* A[a][b] = 4 eps sigma^12 and B[a][b] = 4 eps sigma^6 (Hartree, bohr) for the site
 * pair (CH4 class a: 0 = C, 1 = H; CO2 class b: 0 = C, 1 = O):
 * V = sum over pairs of A / d^12 - B / d^6 */
static inline void hh_ch4co2_lj_pairs(double A[2][2], double B[2][2]) {
    const double sig[2][2] = {{3.50, 2.50}, {2.80, 3.05}};  /* [molecule][class], angstrom */
    const double eps[2][2] = {{33.2, 15.1}, {27.0, 79.0}};  /* kelvin */
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            double s = 0.5 * (sig[0][a] + sig[1][b]) / HH_CH4CO2_BOHR_A;
            double e = sqrt(eps[0][a] * eps[1][b]) / HH_CH4CO2_HARTREE_K * HH_CH4CO2_LJ_SCALE;
            double s6 = s * s * s * s * s * s;
            A[a][b] = 4.0 * e * s6 * s6;
            B[a][b] = 4.0 * e * s6;
        }
}

/* body-frame direction signs of the four H atoms */
static const double hh_ch4co2_hsign[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};

#endif /* HH_CH4CO2_STANDIN_H_ */
