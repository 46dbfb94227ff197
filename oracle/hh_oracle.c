/*
 * CPU oracle for the HAWAIIHYBRID trajectory hot path -- TEST INFRASTRUCTURE ONLY.
 * See hh_oracle.h for what it restates and how it is pinned.  Only tests/, the
 * smoke check and bench.py's CPU-baseline leg load it.  Build flags keep
 * floating-point contraction off so that its arithmetic order is the one written.
 */
#define _GNU_SOURCE
#include "hh_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "../hawaiihybrid_b200/csrc/hh_co2ar_tables.h"
#include "../hawaiihybrid_b200/csrc/hh_n2ar_tables.h"
#include "../hawaiihybrid_b200/csrc/hh_dop853_tableau.h"
#include "../hawaiihybrid_b200/csrc/hh_ch4co2_tables.h"
#include "../hawaiihybrid_b200/csrc/hh_ch4co2_standin.h"

/* ---- constants (src/constants.h:8-53, CODATA 2022) ---- */
#define ALU 5.29177210903e-11
#define Boltzmann 1.380649e-23
#define Hartree 4.3597447222071e-18
#define HTOCM 2.1947463136320e5
#define ATU 2.4188843265857e-17
#define LightSpeed_cm 2.99792458e10
#define ADIPMOMU 8.4783536255e-30
#define EPSILON0 8.8541878128e-12
#define HkT (Hartree / Boltzmann)
#define ZeroCoeff (0.00361479637 / (4.0 * M_PI))
#define SecondCoeff 13856114.29344114  /* src/constants.h:30 */

/* ======================================================================== */
/* MT19937 as configured by mtwist (thirdparty/mtwist.c:372-400, 640-796,   */
/* thirdparty/mtwist.h:624-634): Knuth-69069 seeding of the 624 words, an   */
/* immediate refresh, words consumed in generation order, standard tempering,*/
/* double = word * 2^-32.                                                    */
/* ======================================================================== */
static void mt_refresh(hho_mt *s) {
    uint32_t *m = s->mt;
    for (int i = 0; i < 624; ++i) {
        uint32_t y = (m[i] & 0x80000000u) | (m[(i + 1) % 624] & 0x7fffffffu);
        m[i] = m[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    s->idx = 0;
}

void hho_mt_seed(hho_mt *s, uint32_t seed) {
    if (seed == 0) seed = 4357u;
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i) s->mt[i] = 69069u * s->mt[i - 1];
    mt_refresh(s);
}

uint32_t hho_mt_u32(hho_mt *s) {
    if (s->idx >= 624) mt_refresh(s);
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double hho_mt_drand(hho_mt *s) { return (double)hho_mt_u32(s) * (1.0 / 4294967296.0); }

void hho_mt_stream(uint32_t seed, size_t n, uint32_t *out) {
    hho_mt s;
    hho_mt_seed(&s, seed);
    for (size_t i = 0; i < n; ++i) out[i] = hho_mt_u32(&s);
}

/* ======================================================================== */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)                         */
/* ======================================================================== */
void hho_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* ======================================================================== */
/* He-Ar (PES-IDS/HeAr.h:33-107).  V is an exponential repulsion plus       */
/* damped dispersion -C_2n f_2n(bR)/R^2n, n = 3..8, with the damping          */
/* f_2n(x) = 1 - exp(-x) sum_{k<=2n} x^k/k!; the constants are the          */
/* reference's.  dV/dR is the analytic derivative of the same form.          */
/* ======================================================================== */
static const double HEAR_A = 0.2303058634e2;
static const double HEAR_G1 = 0.163051044e1;   /* exp(-G1 R - G2 R^2) */
static const double HEAR_G2 = 0.4680016e-1;
static const double HEAR_B = 0.16274792500000e1;
static const double HEAR_C[6] = {0.940835513e1, 0.165523018e3, 0.379715796e4,
                                 0.1165179999e6, 0.466258000e7, 0.236861000e9};

double hho_hear_V(double R) {
    double x = HEAR_B * R, ex = exp(-x);
    double term = 1.0, S = 1.0;          /* S = sum_{k<=m} x^k/k! */
    double V = HEAR_A * exp(-HEAR_G1 * R - HEAR_G2 * R * R);
    double R2 = R * R, Rp = R2 * R2;     /* R^4 -> multiplied up to R^2n */
    int m = 0;
    for (int n = 3; n <= 8; ++n) {
        while (m < 2 * n) { ++m; term *= x / m; S += term; }
        Rp *= R2;
        V -= HEAR_C[n - 3] * (1.0 - ex * S) / Rp;
    }
    return V;
}

double hho_hear_dV(double R) {
    double x = HEAR_B * R, ex = exp(-x);
    double term = 1.0, S = 1.0;
    double dV = HEAR_A * exp(-HEAR_G1 * R - HEAR_G2 * R * R) * (-HEAR_G1 - 2.0 * HEAR_G2 * R);
    double R2 = R * R, Rp = R2 * R2;
    int m = 0;
    for (int n = 3; n <= 8; ++n) {
        while (m < 2 * n) { ++m; term *= x / m; S += term; }
        Rp *= R2;
        double f = 1.0 - ex * S;
        double fp = HEAR_B * ex * term;  /* d f/dR = b e^-x x^2n/(2n)! */
        dV -= HEAR_C[n - 3] * (fp / Rp - 2.0 * n * f / (Rp * R));
    }
    return dV;
}

double hho_hear_dip(double R) {
    return exp(0.47293181 - 0.40100613 * R - 0.10292726 * R * R) - 148.55391 * pow(R, -7);
}

/* ======================================================================== */
/* CO2-Ar molecular-frame surfaces from the generated tables                 */
/* (PES-IDS/ai_pes_co2ar.c:27-459, PES-IDS/ai_ids_co2ar.cpp:21-491).         */
/* ======================================================================== */
static int co2ar_interval(double R) {
    int i = 0;
    while (i < HH_CO2AR_NINT - 1 && !(R < hh_co2ar_rbound[i])) ++i;
    return i;
}

/* radial function c(R) and c'(R) of one table row */
static void co2ar_radial(const double *row, double R, double rlo, double *c, double *dc) {
    double t = R - rlo;
    double v = ((row[3] * t + row[2]) * t + row[1]) * t + row[0];
    double d = (3.0 * row[3] * t + 2.0 * row[2]) * t + row[1];
    double iR = 1.0 / R;
    double iR4 = iR * iR * iR * iR;
    double iR5 = iR4 * iR, iR6 = iR5 * iR, iR7 = iR6 * iR;
    v += row[4] * iR4 + row[5] * iR5 + row[6] * iR6 + row[7] * iR7;
    d -= (4.0 * row[4] * iR4 + 5.0 * row[5] * iR5 + 6.0 * row[6] * iR6 + 7.0 * row[7] * iR7) * iR;
    if (row[8] != 0.0) {
        double e = row[8] * exp(row[9] * R);
        v += e;
        d += row[9] * e;
    }
    *c = v;
    if (dc) *dc = d;
}

/* P_l(x), l = 0..10 (gsl_sf_legendre_Pl_array), and P_l'(x) */
static void legendre_P(double x, double P[11], double dP[11]) {
    P[0] = 1.0; P[1] = x;
    for (int l = 1; l < 10; ++l) P[l + 1] = ((2 * l + 1) * x * P[l] - l * P[l - 1]) / (l + 1);
    if (dP) {
        dP[0] = 0.0; dP[1] = 1.0;
        for (int l = 1; l < 10; ++l) dP[l + 1] = dP[l - 1] + (2 * l + 1) * P[l];
    }
}

double hho_co2ar_V_mol(double R, double theta) {
    double P[11];
    legendre_P(cos(theta), P, NULL);
    int i = co2ar_interval(R);
    double V = 0.0;
    for (int li = 0; li < HH_CO2AR_NL; ++li) {
        double c;
        co2ar_radial(hh_co2ar_pes[i][li], R, hh_co2ar_rlo[i], &c, NULL);
        V += P[2 * li] * c;
    }
    return V / HTOCM;
}

void hho_co2ar_dV_mol(double R, double theta, double *dR, double *dtheta) {
    double P[11], dP[11];
    double x = cos(theta), s = sin(theta);
    legendre_P(x, P, dP);
    int i = co2ar_interval(R);
    double vR = 0.0, vx = 0.0;
    for (int li = 0; li < HH_CO2AR_NL; ++li) {
        double c, dc;
        co2ar_radial(hh_co2ar_pes[i][li], R, hh_co2ar_rlo[i], &c, &dc);
        vR += P[2 * li] * dc;
        vx += dP[2 * li] * c;
    }
    *dR = vR / HTOCM;
    *dtheta = -s * vx / HTOCM;
}

/* body-frame dipole (d_x, 0, d_z): d_x = sum_l P_l^1 a_l(R) with the
 * Condon-Shortley phase (GSL csphase = -1), d_z = sum_l P_l b_l(R) */
void hho_co2ar_dip_mol(double R, double theta, double d[3]) {
    double x = cos(theta);
    double P[11];
    legendre_P(x, P, NULL);
    /* associated P_l^1 by the upward recurrence from P_1^1 = -sqrt(1-x^2) */
    double P1[11];
    P1[0] = 0.0;
    P1[1] = -sqrt((1.0 - x) * (1.0 + x));
    P1[2] = 3.0 * x * P1[1];
    for (int l = 2; l < 10; ++l) P1[l + 1] = ((2 * l + 1) * x * P1[l] - (l + 1) * P1[l - 1]) / l;
    int i = co2ar_interval(R);
    double dx = 0.0, dz = 0.0;
    for (int li = 0; li < HH_CO2AR_NL; ++li) {
        double a, b;
        co2ar_radial(hh_co2ar_dipx[i][li], R, hh_co2ar_rlo[i], &a, NULL);
        co2ar_radial(hh_co2ar_dipz[i][li], R, hh_co2ar_rlo[i], &b, NULL);
        dx += P1[2 * li] * a;
        dz += P[2 * li] * b;
    }
    d[0] = dx; d[1] = 0.0; d[2] = dz;
}

/* rotations with the reference's sign conventions (src/angles_handler.cpp:45-104) */
static void Sz(double a, double m[3][3]) {
    double s = sin(a), c = cos(a);
    double r[3][3] = {{c, s, 0}, {-s, c, 0}, {0, 0, 1}};
    memcpy(m, r, sizeof r);
}
static void Sz_dot(double a, double m[3][3]) {
    double s = sin(a), c = cos(a);
    double r[3][3] = {{-s, c, 0}, {-c, -s, 0}, {0, 0, 0}};
    memcpy(m, r, sizeof r);
}
static void Sx(double a, double m[3][3]) {
    double s = sin(a), c = cos(a);
    double r[3][3] = {{1, 0, 0}, {0, c, s}, {0, -s, c}};
    memcpy(m, r, sizeof r);
}
static void Sx_dot(double a, double m[3][3]) {
    double s = sin(a), c = cos(a);
    double r[3][3] = {{0, 0, 0}, {0, -s, c}, {0, -c, -s}};
    memcpy(m, r, sizeof r);
}
static void mv(double m[3][3], const double v[3], double o[3]) {
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = m[i][0] * v[0] + m[i][1] * v[1] + m[i][2] * v[2];
    memcpy(o, t, sizeof t);
}
static void mtv(double m[3][3], const double v[3], double o[3]) {
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = m[0][i] * v[0] + m[1][i] * v[1] + m[2][i] * v[2];
    memcpy(o, t, sizeof t);
}

/* linear_molecule_atom_lab_to_mol (src/angles_handler.cpp:106-138):
 * qlab (PHI THETA R PHI1 THETA1) -> qmol (R PHIEM THETAEM PSIEM THETAM) */
void hho_co2ar_lab_to_mol(const double *qlab, double *qmol) {
    qmol[0] = qlab[2];
    qmol[1] = qlab[0] + M_PI / 2.0;
    qmol[2] = qlab[1];
    double Mz[3][3], Mx[3][3];
    Sz(qmol[1], Mz);
    Sx(qmol[2], Mx);
    double u[3] = {cos(qlab[3]) * sin(qlab[4]), sin(qlab[3]) * sin(qlab[4]), cos(qlab[4])};
    double dd[3];
    mv(Mz, u, dd);
    mv(Mx, dd, dd);
    qmol[4] = acos(dd[2]);
    double st = sqrt(1 - dd[2] * dd[2]);
    qmol[3] = atan2(dd[1] / st, dd[0] / st);
}

/* linear_molecule_atom_Jacobi_mol_by_lab (src/angles_handler.cpp:140-193):
 * jac[i*5 + j] = d qmol_j / d qlab_i */
void hho_co2ar_jacobian(const double *q, double *jac) {
    double qmol[5];
    hho_co2ar_lab_to_mol(q, qmol);
    memset(jac, 0, 25 * sizeof(double));
    jac[2 * 5 + 0] = 1.0;
    jac[0 * 5 + 1] = 1.0;
    jac[1 * 5 + 2] = 1.0;
    double Mz[3][3], Mx[3][3], Mzd[3][3], Mxd[3][3];
    Sz(qmol[1], Mz); Sx(qmol[2], Mx);
    Sz_dot(qmol[1], Mzd); Sx_dot(qmol[2], Mxd);
    double sphi = sin(q[3]), cphi = cos(q[3]), sth = sin(q[4]), cth = cos(q[4]);
    double u[3] = {cphi * sth, sphi * sth, cth};
    double u_phi[3] = {-sphi * sth, cphi * sth, 0.0};
    double u_th[3] = {cphi * cth, sphi * cth, -sth};
    double sin_thetam = sin(qmol[4]);
    double spsi = sin(qmol[3]), cpsi = cos(qmol[3]);
    double d[3];
    /* row r <- derivative of dd along lab coordinate r:
     * d(thetam) = -d(dd_z)/sin(thetam), d(psiem) = (d(dd_y) cos psi - d(dd_x) sin psi)/sin(thetam) */
    mv(Mz, u_phi, d); mv(Mx, d, d);
    jac[3 * 5 + 4] = -d[2] / sin_thetam;
    jac[3 * 5 + 3] = (d[1] * cpsi - d[0] * spsi) / sin_thetam;
    mv(Mz, u_th, d); mv(Mx, d, d);
    jac[4 * 5 + 4] = -d[2] / sin_thetam;
    jac[4 * 5 + 3] = (d[1] * cpsi - d[0] * spsi) / sin_thetam;
    mv(Mzd, u, d); mv(Mx, d, d);
    jac[0 * 5 + 4] = -d[2] / sin_thetam;
    jac[0 * 5 + 3] = (d[1] * cpsi - d[0] * spsi) / sin_thetam;
    mv(Mz, u, d); mv(Mxd, d, d);
    jac[1 * 5 + 4] = -d[2] / sin_thetam;
    jac[1 * 5 + 3] = (d[1] * cpsi - d[0] * spsi) / sin_thetam;
}

/* dpes_lab (PES-IDS/ai_pes_co2ar_lib.cpp:11-30): dV/dq_lab = J (dV/dR, 0, 0, 0, dV/dthetam) */
static void co2ar_dpes_lab(const double *q, double *dVdq) {
    double qmol[5], jac[25];
    hho_co2ar_lab_to_mol(q, qmol);
    double dR, dth;
    hho_co2ar_dV_mol(qmol[0], qmol[4], &dR, &dth);
    hho_co2ar_jacobian(q, jac);
    for (int i = 0; i < 5; ++i) dVdq[i] = jac[i * 5 + 0] * dR + jac[i * 5 + 4] * dth;
}

/* dipole_lab (PES-IDS/ai_ids_co2ar_lib.cpp:12-37) */
static void co2ar_dipole_lab(const double *q, double out[3]) {
    double qmol[5];
    hho_co2ar_lab_to_mol(q, qmol);
    double dm[3];
    hho_co2ar_dip_mol(qmol[0], qmol[4], dm);
    double Mphi[3][3], Mth[3][3], Mpsi[3][3];
    Sz(qmol[1], Mphi); Sx(qmol[2], Mth); Sz(qmol[3], Mpsi);
    double t[3];
    mtv(Mpsi, dm, t);
    mtv(Mth, t, t);
    mtv(Mphi, t, out);
}

/* ======================================================================== */
/* CH4-CO2 (ROTOR + LINEAR).  Lab coordinates q (PHI THETA R PHI1 THETA1 PSI1 */
/* PHI2 THETA2), src/angles_handler.cpp:357-365.                             */
/* ======================================================================== */
/* Sy_filler_non_standard (src/angles_handler.cpp:91-97) and its derivative */
static void Sy_ns(double a, double m[3][3]) {
    double s = sin(a), c = cos(a);
    double r[3][3] = {{c, 0, s}, {0, 1, 0}, {-s, 0, c}};
    memcpy(m, r, sizeof r);
}
static void mm(double a[3][3], double b[3][3], double o[3][3]) {
    double t[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) t[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
    memcpy(o, t, sizeof t);
}

/* unit vectors of the intermolecular axis and of the CO2 axis in the lab frame:
 * Sz(PHI)^T Sy_ns(THETA)^T z = (-sin THETA cos PHI, -sin THETA sin PHI, cos THETA)
 * (src/angles_handler.cpp:396, 408) */
static void ch4co2_axis(double Phi, double Th, double u[3]) {
    u[0] = -sin(Th) * cos(Phi);
    u[1] = -sin(Th) * sin(Phi);
    u[2] = cos(Th);
}

/* S1 = Spsi1 Sx(theta1) Sz(phi1): lab -> CH4 body frame (src/angles_handler.cpp:384-394) */
static void ch4co2_S1(double phi, double th, double psi, double S1[3][3]) {
    double A[3][3], B[3][3], C[3][3];
    Sz(psi, A); Sx(th, B); Sz(phi, C);
    mm(A, B, S1);
    mm(S1, C, S1);
}

/* CH4_linear_molecule_lab_to_kal (src/angles_handler.cpp:357-419):
 * qkal = (R, PHI1K, THETA1K, PHI2K, THETA2K), the directions of the intermolecular
 * axis and of the CO2 axis in the CH4 body frame */
void hho_ch4co2_lab_to_kal(const double *qlab, double *qkal) {
    qkal[0] = qlab[2];
    double SPhi[3][3], STheta[3][3], S1[3][3], Sphi2[3][3], Stheta2[3][3];
    Sz(qlab[0], SPhi); Sy_ns(qlab[1], STheta);
    ch4co2_S1(qlab[3], qlab[4], qlab[5], S1);
    Sz(qlab[6], Sphi2); Sy_ns(qlab[7], Stheta2);
    double z[3] = {0, 0, 1}, dd[3];
    mtv(STheta, z, dd); mtv(SPhi, dd, dd); mv(S1, dd, dd);
    double c1 = dd[2], s1 = sqrt(1 - c1 * c1);
    qkal[2] = acos(c1);
    qkal[1] = atan2(dd[1] / s1, dd[0] / s1);
    mtv(Stheta2, z, dd); mtv(Sphi2, dd, dd); mv(S1, dd, dd);
    double c2 = dd[2], s2 = sqrt(1.0 - dd[2] * dd[2]);
    qkal[4] = acos(c2);
    qkal[3] = atan2(dd[1] / s2, dd[0] / s2);
}

/* GSL_SF_LEGENDRE_NONE with the Condon-Shortley phase, index l(l+1)/2 + m */
static void legendre_lm(int lmax, double x, double *P) {
    double s = sqrt((1.0 - x) * (1.0 + x));
    double pmm = 1.0;
    for (int m = 0; m <= lmax; ++m) {
        if (m > 0) pmm *= -(2.0 * m - 1.0) * s;
        P[m * (m + 1) / 2 + m] = pmm;
        if (m + 1 <= lmax) {
            double p1 = x * (2.0 * m + 1.0) * pmm, p0 = pmm;
            P[(m + 1) * (m + 2) / 2 + m] = p1;
            for (int l = m + 2; l <= lmax; ++l) {
                double pl = ((2.0 * l - 1.0) * x * p1 - (double)(l + m - 1) * p0) / (double)(l - m);
                P[l * (l + 1) / 2 + m] = pl;
                p0 = p1;
                p1 = pl;
            }
        }
    }
}

/* radial function b at R (piece tables of hh_ch4co2_tables.h) */
static double ch4co2_rad(int b, double R) {
    int s = 0;
    while (s < HH_CH4CO2_NSEG - 1 && R >= hh_ch4co2_seg_hi[s]) ++s;
    const double *c = hh_ch4co2_rad[b][s];
    double x = R - hh_ch4co2_centre[s];
    double v = c[0] + x * (c[1] + x * (c[2] + x * c[3]));
    return (s == HH_CH4CO2_NSEG - 1) ? v * pow(R, -6) : v;
}

/* dipole_vector (PES-IDS/ai_ids_ch4_co2.cpp:672-1067): sum over the 320 basis
 * functions of rad_b(R) times the real part of their angular functions, here in
 * the expanded form of hh_ch4co2_tables.h; Legendre functions of cos(theta) and
 * cos(k phi), sin(k phi) from the angles, as the reference computes them */
void hho_ch4co2_dipole_kal(const double *qkal, double d[3]) {
    double R = qkal[0];
    double P1[(HH_CH4CO2_L1MAX + 1) * (HH_CH4CO2_L1MAX + 2) / 2];
    double P2[(HH_CH4CO2_L2MAX + 1) * (HH_CH4CO2_L2MAX + 2) / 2];
    legendre_lm(HH_CH4CO2_L1MAX, cos(qkal[2]), P1);
    legendre_lm(HH_CH4CO2_L2MAX, cos(qkal[4]), P2);
    double t1[2][HH_CH4CO2_L1MAX + 1], t2[2][HH_CH4CO2_L2MAX + 1];
    for (int k = 0; k <= HH_CH4CO2_L1MAX; ++k) { t1[0][k] = cos(k * qkal[1]); t1[1][k] = sin(k * qkal[1]); }
    for (int k = 0; k <= HH_CH4CO2_L2MAX; ++k) { t2[0][k] = cos(k * qkal[3]); t2[1][k] = sin(k * qkal[3]); }
    double rad[HH_CH4CO2_NB];
    for (int b = 0; b < HH_CH4CO2_NB; ++b) rad[b] = ch4co2_rad(b, R);
    /* harmonic values by code 2 * (l(l+1)/2 + m) + cs */
    double Y1[(HH_CH4CO2_L1MAX + 1) * (HH_CH4CO2_L1MAX + 2)], Y2[(HH_CH4CO2_L2MAX + 1) * (HH_CH4CO2_L2MAX + 2)];
    for (int l = 0; l <= HH_CH4CO2_L1MAX; ++l)
        for (int m = 0; m <= l; ++m)
            for (int cs = 0; cs < 2; ++cs) {
                int i = l * (l + 1) / 2 + m;
                Y1[2 * i + cs] = P1[i] * (m ? t1[cs][m] : 1.0);
            }
    for (int l = 0; l <= HH_CH4CO2_L2MAX; ++l)
        for (int m = 0; m <= l; ++m)
            for (int cs = 0; cs < 2; ++cs) {
                int i = l * (l + 1) / 2 + m;
                Y2[2 * i + cs] = P2[i] * (m ? t2[cs][m] : 1.0);
            }
    double acc[HH_CH4CO2_NB][3];
    memset(acc, 0, sizeof acc);
    for (int t = 0; t < HH_CH4CO2_NTERM; ++t) {
        const short *ix = hh_ch4co2_tidx[t];
        acc[ix[0]][ix[1]] += hh_ch4co2_tcoef[t] * Y1[ix[2]] * Y2[ix[3]];
    }
    d[0] = d[1] = d[2] = 0.0;
    for (int b = 0; b < HH_CH4CO2_NB; ++b)
        for (int c = 0; c < 3; ++c) d[c] += acc[b][c] * rad[b];
}

/* dipole_lab (PES-IDS/ai_ids_ch4_co2_lib.cpp:8-33): S1^T times the body-frame dipole */
static void ch4co2_dipole_lab(const double *q, double out[3]) {
    double qkal[5], dk[3], S1[3][3];
    hho_ch4co2_lab_to_kal(q, qkal);
    hho_ch4co2_dipole_kal(qkal, dk);
    ch4co2_S1(q[3], q[4], q[5], S1);
    mtv(S1, dk, out);
}

/* the stand-in surface (hh_ch4co2_standin.h) from the lab-frame site positions;
 * with grad != NULL also dV/dq (8 lab coordinates) */
static double ch4co2_V(const double *q, double *grad) {
    double A[2][2], B[2][2];
    hh_ch4co2_lj_pairs(A, B);
    double rh[3], u2[3], S1[3][3];
    ch4co2_axis(q[0], q[1], rh);
    ch4co2_axis(q[6], q[7], u2);
    ch4co2_S1(q[3], q[4], q[5], S1);
    const double R = q[2], a = HH_CH4CO2_RCH / sqrt(3.0);
    double x1[5][3], hb[5][3], x2[3][3];
    for (int s = 0; s < 5; ++s) {
        for (int i = 0; i < 3; ++i) hb[s][i] = s ? a * hh_ch4co2_hsign[s - 1][i] : 0.0;
        mtv(S1, hb[s], x1[s]);
    }
    for (int i = 0; i < 3; ++i) {
        x2[0][i] = R * rh[i];
        x2[1][i] = R * rh[i] + HH_CH4CO2_RCO * u2[i];
        x2[2][i] = R * rh[i] - HH_CH4CO2_RCO * u2[i];
    }
    double V = 0.0, g1[5][3], g2[3][3];
    memset(g1, 0, sizeof g1);
    memset(g2, 0, sizeof g2);
    for (int s = 0; s < 5; ++s)
        for (int t = 0; t < 3; ++t) {
            double dx[3] = {x2[t][0] - x1[s][0], x2[t][1] - x1[s][1], x2[t][2] - x1[s][2]};
            double i2 = 1.0 / (dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
            double i6 = i2 * i2 * i2;
            double Ap = A[s ? 1 : 0][t ? 1 : 0], Bp = B[s ? 1 : 0][t ? 1 : 0];
            V += i6 * (Ap * i6 - Bp);
            double f = -(12.0 * Ap * i6 - 6.0 * Bp) * i6 * i2;  /* (dV/dd) / d */
            for (int i = 0; i < 3; ++i) {
                g2[t][i] += f * dx[i];
                g1[s][i] -= f * dx[i];
            }
        }
    if (grad) {
        double Gr[3], Gu[3];
        for (int i = 0; i < 3; ++i) {
            Gr[i] = g2[0][i] + g2[1][i] + g2[2][i];
            Gu[i] = HH_CH4CO2_RCO * (g2[1][i] - g2[2][i]);
        }
        double sT = sin(q[1]), cT = cos(q[1]), sP = sin(q[0]), cP = cos(q[0]);
        double r_Phi[3] = {sT * sP, -sT * cP, 0.0}, r_Th[3] = {-cT * cP, -cT * sP, -sT};
        double s2 = sin(q[7]), c2 = cos(q[7]), sp2 = sin(q[6]), cp2 = cos(q[6]);
        double u_phi[3] = {s2 * sp2, -s2 * cp2, 0.0}, u_th[3] = {-c2 * cp2, -c2 * sp2, -s2};
        grad[0] = grad[1] = grad[2] = grad[6] = grad[7] = 0.0;
        for (int i = 0; i < 3; ++i) {
            grad[0] += Gr[i] * R * r_Phi[i];
            grad[1] += Gr[i] * R * r_Th[i];
            grad[2] += Gr[i] * rh[i];
            grad[6] += Gu[i] * u_phi[i];
            grad[7] += Gu[i] * u_th[i];
        }
        /* dS1/d(angle) = Spsi Sx Sz_dot(phi), Spsi Sx_dot Sz, Sz_dot(psi) Sx Sz */
        double Zp[3][3], Xt[3][3], Zs[3][3], Zpd[3][3], Xtd[3][3], Zsd[3][3], D[3][3][3];
        Sz(q[3], Zp); Sx(q[4], Xt); Sz(q[5], Zs);
        Sz_dot(q[3], Zpd); Sx_dot(q[4], Xtd); Sz_dot(q[5], Zsd);
        mm(Zs, Xt, D[0]); mm(D[0], Zpd, D[0]);
        mm(Zs, Xtd, D[1]); mm(D[1], Zp, D[1]);
        mm(Zsd, Xt, D[2]); mm(D[2], Zp, D[2]);
        for (int k = 0; k < 3; ++k) {
            double acc = 0.0;
            for (int s = 1; s < 5; ++s) {
                double dx[3];
                mtv(D[k], hb[s], dx);
                acc += g1[s][0] * dx[0] + g1[s][1] * dx[1] + g1[s][2] * dx[2];
            }
            grad[3 + k] = acc;
        }
    }
    return V;
}

double hho_ch4co2_V_lab(const double *q) { return ch4co2_V(q, NULL); }

/* ======================================================================== */
/* N2-Ar PIP-NN surfaces.  PES: PES-IDS/ai_pes_n2_ar_pip_nn.cpp:8-146 with   */
/* PES-IDS/mlp.hpp:178-256 (forward, backward) and the lab chain rule of     */
/* examples/correlation_n2_ar.cpp:18-50.  Dipole: PES-IDS/ai_ids_n2_ar_pip_nn */
/* .cpp:11-128 with PES-IDS/QModel.hpp:144-257.  PIP bases and weights are   */
/* the tables of hh_n2ar_tables.h.                                           */
/* ======================================================================== */
#define L_N2 2.07856749                     /* src/constants.h:80 */
#define N2AR_EN_INF 0.0384490895371528      /* ai_pes_n2_ar_pip_nn.cpp:130 */

/* quintic switch 10r^3 - 15r^4 + 6r^5 on [xi, xf] (ai_pes_n2_ar_pip_nn.cpp:14-41) */
static double n2ar_sw(double x, double xi, double xf) {
    if (x < xi) return 0.0;
    if (x < xf) {
        double r = (x - xi) / (xf - xi), r3 = r * r * r, r4 = r3 * r, r5 = r4 * r;
        return 10.0 * r3 - 15.0 * r4 + 6.0 * r5;
    }
    return 1.0;
}
static double n2ar_dsw(double x, double xi, double xf) {
    if (x < xi || !(x < xf)) return 0.0;
    double t = (x - xi) / (xf - xi), t2 = t * t, t3 = t2 * t, t4 = t3 * t;
    return (30.0 * t2 - 60.0 * t3 + 30.0 * t4) / (xf - xi);
}
static double silu(double x) { return x / (1.0 + exp(-x)); }
static double dsilu(double x) {
    double e = exp(-x), d = 1.0 + e;
    return 1.0 / d + x * e / d / d;
}

/* PIPs p[17] of y[3] and (jac != NULL) jac[k * 17 + i] = d p_i / d y_k, from
 * the monomial table (c_basis_2_1_4_purify.cc; the Jacobian is differentiated
 * here, c_jac_2_1_4_purify.cc is the reference's own) */
void hho_n2ar_pes_pip(const double *y, double *p, double *jac) {
    memset(p, 0, HH_N2AR_PES_NPIP * sizeof(double));
    if (jac) memset(jac, 0, 3 * HH_N2AR_PES_NPIP * sizeof(double));
    for (int m = 0; m < HH_N2AR_PES_NMONO; ++m) {
        const signed char *v = hh_n2ar_pes_var[m];
        int deg = 0;
        while (deg < 4 && v[deg] >= 0) ++deg;
        double prod = 1.0;
        for (int j = 0; j < deg; ++j) prod *= y[v[j]];
        p[hh_n2ar_pes_poly[m]] += prod;
        if (!jac) continue;
        for (int j = 0; j < deg; ++j) {  /* d(monomial)/dy[v[j]] */
            double dp = 1.0;
            for (int i = 0; i < deg; ++i)
                if (i != j) dp *= y[v[i]];
            jac[v[j] * HH_N2AR_PES_NPIP + hh_n2ar_pes_poly[m]] += dp;
        }
    }
}

/* PIPs p[308] of y[10] of the dipole model (the three bases in model order) */
void hho_n2ar_dip_pip(const double *y, double *p) {
    memset(p, 0, HH_N2AR_DIP_NPIP * sizeof(double));
    for (int m = 0; m < HH_N2AR_DIP_NMONO; ++m) {
        double prod = 1.0;
        for (int j = 0; j < 3 && hh_n2ar_dip_var[m][j] >= 0; ++j) prod *= y[hh_n2ar_dip_var[m][j]];
        p[hh_n2ar_dip_poly[m]] += prod;
    }
}

/* PES energy (cm^-1, before the en_inf shift) from the distances
 * d[0] = |N1-N2|, d[1] = |N1-Ar|, d[2] = |N2-Ar|; dEdd (optional) receives dE/dd */
double hho_n2ar_energy_cm(const double d[3], double dEdd[3]) {
    double y[3], dy[3];
    y[0] = exp(-d[0] / 2.0);
    dy[0] = -0.5 * y[0];
    for (int k = 1; k < 3; ++k) {
        double s = n2ar_sw(d[k], 6.0, 20.0), ds = n2ar_dsw(d[k], 6.0, 20.0);
        double e = exp(-d[k] / 2.0), d6 = pow(d[k], 6), d7 = d6 * d[k];
        y[k] = (1.0 - s) * e + s * 1e4 / d6;
        dy[k] = -ds * e - (1.0 - s) * e / 2.0 + ds * 1e4 / d6 - s * 6e4 / d7;
    }
    double p[HH_N2AR_PES_NPIP], J[3][HH_N2AR_PES_NPIP];
    hho_n2ar_pes_pip(y, p, &J[0][0]);
    double ptr[HH_N2AR_PES_NPIP];
    for (int i = 0; i < HH_N2AR_PES_NPIP; ++i) ptr[i] = (p[i] - hh_n2ar_pes_xmean[i]) / hh_n2ar_pes_xscale[i];
    double out = hh_n2ar_pes_b1[0], g[HH_N2AR_PES_HIDDEN];
    for (int j = 0; j < HH_N2AR_PES_HIDDEN; ++j) {
        double h = hh_n2ar_pes_b0[j];
        for (int i = 0; i < HH_N2AR_PES_NPIP; ++i) h += ptr[i] * hh_n2ar_pes_w0[i][j];
        out += silu(h) * hh_n2ar_pes_w1[j];
        g[j] = dsilu(h) * hh_n2ar_pes_w1[j];
    }
    const double ymean = hh_n2ar_pes_y[0], yscale = hh_n2ar_pes_y[1];
    if (dEdd) {
        double dEdp[HH_N2AR_PES_NPIP];
        for (int i = 0; i < HH_N2AR_PES_NPIP; ++i) {
            double a = 0.0;
            for (int j = 0; j < HH_N2AR_PES_HIDDEN; ++j) a += hh_n2ar_pes_w0[i][j] * g[j];
            dEdp[i] = a / hh_n2ar_pes_xscale[i];
        }
        for (int k = 0; k < 3; ++k) {
            double a = 0.0;
            for (int i = 0; i < HH_N2AR_PES_NPIP; ++i) a += J[k][i] * dEdp[i];
            dEdd[k] = a * dy[k] * yscale;
        }
    }
    return yscale * out + ymean;
}

/* lab_to_xyz (ai_pes_n2_ar_pip_nn.cpp:103-121): N1, N2, Ar */
static void n2ar_lab_xyz(const double *q, double x[9]) {
    double Phi = q[0], Theta = q[1], R = q[2], ph = q[3], th = q[4];
    double h = L_N2 / 2.0;
    double u[3] = {cos(ph) * sin(th), sin(ph) * sin(th), cos(th)};
    for (int i = 0; i < 3; ++i) { x[i] = h * u[i]; x[3 + i] = -h * u[i]; }
    x[6] = R * cos(Phi) * sin(Theta);
    x[7] = R * sin(Phi) * sin(Theta);
    x[8] = R * cos(Theta);
}

static double n2ar_xyz_energy(const double x[9], double dx[9]) {
    static const int pi_[3] = {0, 0, 1}, pj_[3] = {1, 2, 2};
    double d[3], e[3][3];
    for (int k = 0; k < 3; ++k) {
        double s = 0.0;
        for (int c = 0; c < 3; ++c) {
            e[k][c] = x[3 * pi_[k] + c] - x[3 * pj_[k] + c];
            s += e[k][c] * e[k][c];
        }
        d[k] = sqrt(s);
    }
    double g[3];
    double E = hho_n2ar_energy_cm(d, dx ? g : NULL);
    if (dx) {
        memset(dx, 0, 9 * sizeof(double));
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) {
                dx[3 * pi_[k] + c] += g[k] * e[k][c] / d[k];
                dx[3 * pj_[k] + c] -= g[k] * e[k][c] / d[k];
            }
    }
    return E;
}

double hho_n2ar_V_lab(const double *q) {
    double x[9];
    n2ar_lab_xyz(q, x);
    return (n2ar_xyz_energy(x, NULL) - N2AR_EN_INF) / HTOCM;
}

/* dpes (examples/correlation_n2_ar.cpp:18-50) */
static void n2ar_dpes_lab(const double *q, double *dV) {
    double x[9], c[9];
    n2ar_lab_xyz(q, x);
    n2ar_xyz_energy(x, c);
    double Phi = q[0], Theta = q[1], R = q[2];
    double sP = sin(Phi), cP = cos(Phi), sT = sin(Theta), cT = cos(Theta);
    dV[0] = R * (-sP * sT * c[6] + cP * sT * c[7]) / HTOCM;
    dV[1] = R * (cP * cT * c[6] + sP * cT * c[7] - sT * c[8]) / HTOCM;
    dV[2] = (cP * sT * c[6] + sP * sT * c[7] + cT * c[8]) / HTOCM;
    double sp = sin(q[3]), cp = cos(q[3]), st = sin(q[4]), ct = cos(q[4]);
    dV[3] = L_N2 / 2.0 * (-sp * st * c[0] + cp * st * c[1] + sp * st * c[3] - cp * st * c[4]) / HTOCM;
    dV[4] = L_N2 / 2.0 * (cp * ct * c[0] + sp * ct * c[1] - st * c[2] - cp * ct * c[3] - sp * ct * c[4] +
                          st * c[5]) / HTOCM;
}

/* one charge model (0 short, 1 long range): charges q[5] of N1, N2, N1', N2', Ar
 * from the 10 site distances (pairs i < j in site order), y = exp(-d / a0);
 * dist == NULL gives the model's charges at infinite separation (all PIPs
 * zero, QModel::forward_inf) */
static void n2ar_charges(int model, const double *dist, double a0, double q[5]) {
    double p[HH_N2AR_DIP_NPIP] = {0};
    if (dist) {
        double y[10];
        for (int k = 0; k < 10; ++k) y[k] = exp(-dist[k] / a0);
        hho_n2ar_dip_pip(y, p);
    }
    double ptr[HH_N2AR_DIP_NPIP];
    for (int i = 0; i < HH_N2AR_DIP_NPIP; ++i)
        ptr[i] = (p[i] - hh_n2ar_dip_xmean[model][i]) / hh_n2ar_dip_xscale[model][i];
    for (int s = 0; s < 3; ++s) {
        const int nin = hh_n2ar_dip_arch[s][0], nhid = hh_n2ar_dip_arch[s][1], nout = hh_n2ar_dip_arch[s][2];
        const double *w0 = &hh_n2ar_dip_w0[model][hh_n2ar_dip_w0off[s]];
        const double *b0 = &hh_n2ar_dip_b0[model][hh_n2ar_dip_b0off[s]];
        const double *w1 = &hh_n2ar_dip_w1[model][hh_n2ar_dip_w1off[s]];
        const double *b1 = &hh_n2ar_dip_b1[model][hh_n2ar_dip_qoff[s]];
        const double *x = ptr + hh_n2ar_dip_pipoff[s];
        double h[16];
        for (int j = 0; j < nhid; ++j) {
            double a = b0[j];
            for (int i = 0; i < nin; ++i) a += x[i] * w0[i * nhid + j];
            h[j] = silu(a);
        }
        for (int o = 0; o < nout; ++o) {
            double a = b1[o];
            for (int j = 0; j < nhid; ++j) a += h[j] * w1[j * nout + o];
            q[hh_n2ar_dip_qoff[s] + o] = a;
        }
    }
}

/* dipole_bf (ai_ids_n2_ar_pip_nn.cpp:83-127): body-frame dipole at (R, Theta) */
void hho_n2ar_dip_mol(double R, double Theta, double dm[3]) {
    double h = L_N2 / 2.0, s = sin(Theta), c = cos(Theta);
    double x[5][3] = {{h * s, 0.0, h * c}, {-h * s, 0.0, -h * c}, {h * c, 0.0, -h * s},
                      {-h * c, 0.0, h * s}, {0.0, 0.0, R}};
    double dist[10];
    int k = 0;
    for (int i = 0; i < 5; ++i)
        for (int j = i + 1; j < 5; ++j) {
            double a = x[i][0] - x[j][0], b = x[i][1] - x[j][1], e = x[i][2] - x[j][2];
            dist[k++] = sqrt(a * a + b * b + e * e);
        }
    double out[2][3];
    const double a0[2] = {2.0, 6.0};
    for (int m = 0; m < 2; ++m) {
        double q[5], qi[5];
        n2ar_charges(m, dist, a0[m], q);
        n2ar_charges(m, NULL, a0[m], qi);
        for (int cc = 0; cc < 3; ++cc) {
            out[m][cc] = 0.0;
            for (int i = 0; i < 5; ++i) out[m][cc] += (q[i] - qi[i]) * x[i][cc];
        }
    }
    /* R of the N-site centre to Ar (the centre is the origin here) */
    double cx = 0.25 * (x[0][0] + x[1][0] + x[2][0] + x[3][0]);
    double cy = 0.25 * (x[0][1] + x[1][1] + x[2][1] + x[3][1]);
    double cz = 0.25 * (x[0][2] + x[1][2] + x[2][2] + x[3][2]);
    double Rc = sqrt((cx - x[4][0]) * (cx - x[4][0]) + (cy - x[4][1]) * (cy - x[4][1]) +
                     (cz - x[4][2]) * (cz - x[4][2]));
    double sw = n2ar_sw(Rc, 9.5, 12.5);
    for (int cc = 0; cc < 3; ++cc) dm[cc] = (1.0 - sw) * out[0][cc] + sw * out[1][cc];
}

/* dipole_lab (examples/correlation_n2_ar.cpp:52-76) */
static void n2ar_dipole_lab(const double *q, double out[3]) {
    double qmol[5];
    hho_co2ar_lab_to_mol(q, qmol);
    double dm[3];
    hho_n2ar_dip_mol(qmol[0], qmol[4], dm);
    double Mphi[3][3], Mth[3][3], Mpsi[3][3];
    Sz(qmol[1], Mphi); Sx(qmol[2], Mth); Sz(qmol[3], Mpsi);
    double t[3];
    mtv(Mpsi, dm, t);
    mtv(Mth, t, t);
    mtv(Mphi, t, out);
}

/* systems with a linear monomer (phase point of 10, inertia II) */
static int is_linear(const hho_system *sys) {
    return sys->system == HHO_SYS_CO2AR || sys->system == HHO_SYS_N2AR;
}

int hho_qp_size(const hho_system *sys) {
    return sys->system == HHO_SYS_HEAR ? 6 : (sys->system == HHO_SYS_CH4CO2 ? 16 : 10);
}

double hho_pes(const hho_system *sys, const double *q) {
    if (sys->system == HHO_SYS_HEAR) return hho_hear_V(q[2]);
    if (sys->system == HHO_SYS_N2AR) return hho_n2ar_V_lab(q);
    if (sys->system == HHO_SYS_CH4CO2) return ch4co2_V(q, NULL);
    double qmol[5];
    hho_co2ar_lab_to_mol(q, qmol);
    return hho_co2ar_V_mol(qmol[0], qmol[4]);
}

void hho_dpes(const hho_system *sys, const double *q, double *dVdq) {
    if (sys->system == HHO_SYS_HEAR) {
        dVdq[0] = 0.0; dVdq[1] = 0.0; dVdq[2] = hho_hear_dV(q[2]);
        return;
    }
    if (sys->system == HHO_SYS_N2AR) {
        n2ar_dpes_lab(q, dVdq);
        return;
    }
    if (sys->system == HHO_SYS_CH4CO2) {
        ch4co2_V(q, dVdq);
        return;
    }
    co2ar_dpes_lab(q, dVdq);
}

void hho_dipole(const hho_system *sys, const double *q, double d[3]) {
    if (sys->system == HHO_SYS_HEAR) {
        double Phi = q[0], Theta = q[1], dl = hho_hear_dip(q[2]);
        d[0] = dl * sin(Theta) * cos(Phi);
        d[1] = dl * sin(Theta) * sin(Phi);
        d[2] = dl * cos(Theta);
        return;
    }
    if (sys->system == HHO_SYS_N2AR) {
        n2ar_dipole_lab(q, d);
        return;
    }
    if (sys->system == HHO_SYS_CH4CO2) {
        ch4co2_dipole_lab(q, d);
        return;
    }
    co2ar_dipole_lab(q, d);
}

/* ======================================================================== */
/* Hamilton's equations (src/hawaii.c:474-616), kinetic energy (1041-1137)   */
/* phase point: PHI PPHI THETA PTHETA R PR [phi1 pphi1 theta1 ptheta1]        */
/* ======================================================================== */
static void extract_q(const hho_system *sys, const double *qp, double *q) {
    int n = hho_qp_size(sys);
    for (int k = 0; k < n; k += 2) q[k / 2] = qp[k];
}

/* rhsMonomer for ROTOR (src/hawaii.c:501-532) at y[0..5] = (phi pphi theta ptheta psi ppsi) */
static void rotor_rhs(const double *II, const double *y, const double *dV, double *yd) {
    double pPhi = y[1], theta = y[2], pTheta = y[3], psi = y[4], pPsi = y[5];
    double sin_theta = sin(theta), cos_theta = cos(theta);
    double sin_psi = sin(psi), cos_psi = cos(psi);
    double t1 = (pPhi - pPsi * cos_theta) * sin_psi + pTheta * sin_theta * cos_psi;
    double t2 = (pPhi - pPsi * cos_theta) * cos_psi - pTheta * sin_theta * sin_psi;
    yd[0] = t1 * sin_psi / (II[0] * sin_theta * sin_theta) + t2 * cos_psi / (II[1] * sin_theta * sin_theta);
    yd[1] = -dV[0];
    yd[2] = t1 * cos_psi / (II[0] * sin_theta) - t2 * sin_psi / (II[1] * sin_theta);
    double t3 = pPhi * cos_theta - pPsi;
    double t4 = pPsi * cos_theta - pPhi;
    yd[3] = -t3 * (t4 * (II[0] - II[1]) * cos_psi * cos_psi +
                   pTheta * (II[0] - II[1]) * sin_theta * sin_psi * cos_psi + t4 * II[1]) /
                (II[0] * II[1] * sin_theta * sin_theta * sin_theta) - dV[1];
    yd[4] = -t1 * cos_theta * sin_psi / (II[0] * sin_theta * sin_theta) -
            t2 * cos_theta * cos_psi / (II[1] * sin_theta * sin_theta) + pPsi / II[2];
    yd[5] = -t1 * t2 / (II[0] * sin_theta * sin_theta) + t1 * t2 / (II[1] * sin_theta * sin_theta) - dV[2];
}

/* rhsMonomer for LINEAR_MOLECULE (src/hawaii.c:481-494) at y[0..3] */
static void linear_rhs(double I, const double *y, const double *dV, double *yd) {
    double pphi = y[1], th = y[2], pth = y[3];
    double s = sin(th), c = cos(th);
    yd[0] = pphi / I / s / s;
    yd[1] = -dV[0];
    yd[2] = pth / I;
    yd[3] = pphi * pphi * c / I / s / s / s - dV[1];
}

void hho_rhs(const hho_system *sys, const double *y, double *yd) {
    double q[8], dV[8];
    extract_q(sys, y, q);
    hho_dpes(sys, q, dV);
    double mu = sys->mu;
    double pPhi = y[1], Theta = y[2], pTheta = y[3], R = y[4], pR = y[5];
    double R2 = R * R, R3 = R2 * R;
    double sT = sin(Theta), cT = cos(Theta);
    double sT2 = sT * sT, sT3 = sT2 * sT;
    yd[4] = pR / mu;
    yd[5] = pTheta * pTheta / (mu * R3) + pPhi * pPhi / (mu * R3 * sT2) - dV[2];
    yd[0] = pPhi / (mu * R2 * sT2);
    yd[1] = -dV[0];
    yd[2] = pTheta / (mu * R2);
    yd[3] = pPhi * pPhi * cT / (mu * R2 * sT3) - dV[1];
    if (is_linear(sys)) linear_rhs(sys->II, y + 6, dV + 3, yd + 6);
    if (sys->system == HHO_SYS_CH4CO2) {
        rotor_rhs(sys->II1, y + 6, dV + 3, yd + 6);
        linear_rhs(sys->II, y + 12, dV + 6, yd + 12);
    }
}

/* kinetic energy of a ROTOR (src/hawaii.c:1090-1110) at qp[0..5] */
static double rotor_kinetic(const double *II, const double *qp) {
    double pphi = qp[1], theta = qp[2], ptheta = qp[3], psi = qp[4], ppsi = qp[5];
    double sin_theta = sin(theta), cos_theta = cos(theta), sin_psi = sin(psi), cos_psi = cos(psi);
    double a = (pphi - ppsi * cos_theta) * sin_psi + ptheta * sin_theta * cos_psi;
    double b = (pphi - ppsi * cos_theta) * cos_psi - ptheta * sin_theta * sin_psi;
    return a * a / (2.0 * II[0] * sin_theta * sin_theta) + b * b / (2.0 * II[1] * sin_theta * sin_theta) +
           ppsi * ppsi / (2.0 * II[2]);
}

/* kinetic energy of a LINEAR_MOLECULE (src/hawaii.c:1076-1084) at qp[0..3] */
static double linear_kinetic(double I, const double *qp) {
    double pphi = qp[1], th = qp[2], pth = qp[3];
    double s = sin(th);
    return pth * pth / (2.0 * I) + pphi * pphi / (2.0 * I * s * s);
}

double hho_kinetic(const hho_system *sys, const double *qp) {
    double mu = sys->mu;
    double pPhi = qp[1], Theta = qp[2], pTheta = qp[3], R = qp[4], pR = qp[5];
    double sT = sin(Theta);
    double K = pR * pR / (2.0 * mu) + pTheta * pTheta / (2.0 * mu * R * R) +
               pPhi * pPhi / (2.0 * mu * R * R * sT * sT);
    if (is_linear(sys)) K += linear_kinetic(sys->II, qp + 6);
    if (sys->system == HHO_SYS_CH4CO2) K += rotor_kinetic(sys->II1, qp + 6) + linear_kinetic(sys->II, qp + 12);
    return K;
}

double hho_hamiltonian(const hho_system *sys, const double *qp) {
    double q[8];
    extract_q(sys, qp, q);
    double V = hho_pes(sys, q);
    return hho_kinetic(sys, qp) + V;
}

static void quat_mul(const double a[4], const double b[4], double o[4]) {
    double t[4] = {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                   a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
                   a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
                   a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
    memcpy(o, t, sizeof t);
}

/* CH4-CO2 in the reference's lab frame: r = R (-sin T cos P, -sin T sin P, cos T),
 * p the Cartesian momentum of (R, THETA, PHI); the CH4 orientation as the unit
 * quaternion of S1^T = Sz(phi1)^T Sx(theta1)^T Sz(psi1)^T (body -> lab), its lab
 * angular momentum S1^T L_body with L_body = (t1 / sin theta, t2 / sin theta, ppsi)
 * of the rotor's kinetic energy (src/hawaii.c:1090-1110); the CO2 axis u and
 * j = u x p_u */
static void ch4co2_qp_to_cart(const hho_system *sys, const double *qp, double *cart) {
    (void)sys;
    double Phi = qp[0], pPhi = qp[1], Th = qp[2], pTh = qp[3], R = qp[4], pR = qp[5];
    double sT = sin(Th), cT = cos(Th), sP = sin(Phi), cP = cos(Phi);
    double rh[3] = {-sT * cP, -sT * sP, cT};
    double eT[3] = {-cT * cP, -cT * sP, -sT};
    double eP[3] = {sP, -cP, 0.0};
    for (int i = 0; i < 3; ++i) {
        cart[i] = R * rh[i];
        cart[3 + i] = pR * rh[i] + pTh / R * eT[i] + pPhi / (R * sT) * eP[i];
    }
    double phi = qp[6], pphi = qp[7], th = qp[8], pth = qp[9], psi = qp[10], ppsi = qp[11];
    double qa[4] = {cos(0.5 * phi), 0, 0, sin(0.5 * phi)};
    double qb[4] = {cos(0.5 * th), sin(0.5 * th), 0, 0};
    double qc[4] = {cos(0.5 * psi), 0, 0, sin(0.5 * psi)};
    double qq[4];
    quat_mul(qa, qb, qq);
    quat_mul(qq, qc, cart + 6);
    double st = sin(th), ct = cos(th), sp = sin(psi), cp = cos(psi);
    double Lb[3] = {((pphi - ppsi * ct) * sp + pth * st * cp) / st,
                    ((pphi - ppsi * ct) * cp - pth * st * sp) / st, ppsi};
    double S1[3][3];
    ch4co2_S1(phi, th, psi, S1);
    mtv(S1, Lb, cart + 13);
    double ph2 = qp[12], pph2 = qp[13], th2 = qp[14], pth2 = qp[15];
    double s2 = sin(th2), c2 = cos(th2), sp2 = sin(ph2), cp2 = cos(ph2);
    double u[3] = {-s2 * cp2, -s2 * sp2, c2};
    double u_th[3] = {-c2 * cp2, -c2 * sp2, -s2};
    double u_ph[3] = {s2 * sp2, -s2 * cp2, 0.0};
    double pu[3];
    for (int i = 0; i < 3; ++i) pu[i] = pth2 * u_th[i] + pph2 / (s2 * s2) * u_ph[i];
    for (int i = 0; i < 3; ++i) cart[10 + i] = u[i];
    cart[16] = u[1] * pu[2] - u[2] * pu[1];
    cart[17] = u[2] * pu[0] - u[0] * pu[2];
    cart[18] = u[0] * pu[1] - u[1] * pu[0];
}

void hho_qp_to_cart(const hho_system *sys, const double *qp, double *cart) {
    if (sys->system == HHO_SYS_CH4CO2) {
        ch4co2_qp_to_cart(sys, qp, cart);
        return;
    }
    double Phi = qp[0], pPhi = qp[1], Th = qp[2], pTh = qp[3], R = qp[4], pR = qp[5];
    double sT = sin(Th), cT = cos(Th), sP = sin(Phi), cP = cos(Phi);
    double Rh[3] = {sT * cP, sT * sP, cT};
    double Th_h[3] = {cT * cP, cT * sP, -sT};
    double Ph_h[3] = {-sP, cP, 0.0};
    for (int i = 0; i < 3; ++i) {
        cart[i] = R * Rh[i];
        cart[3 + i] = pR * Rh[i] + pTh / R * Th_h[i] + pPhi / (R * sT) * Ph_h[i];
    }
    if (is_linear(sys)) {
        double ph = qp[6], pph = qp[7], th = qp[8], pth = qp[9];
        double s = sin(th), c = cos(th), sp = sin(ph), cp = cos(ph);
        double u[3] = {s * cp, s * sp, c};
        double th_h[3] = {c * cp, c * sp, -s};
        double ph_h[3] = {-sp, cp, 0.0};
        for (int i = 0; i < 3; ++i) {
            cart[6 + i] = u[i];
            cart[9 + i] = pth * ph_h[i] - pph / s * th_h[i];  /* j = u x p_u (j_monomer, hawaii.c:398-431) */
        }
    }
}

/* ======================================================================== */
/* Sampler (src/hawaii.c:1206-1421) and pair-state filter (2976-2994)        */
/* ======================================================================== */
static double generate_normal(hho_mt *s, int *draws) {
    for (;;) {
        double U = hho_mt_drand(s);
        double V = hho_mt_drand(s);
        *draws += 2;
        double logU = log(U);
        if (isnan(logU) || isinf(logU)) continue;
        return 1.0 * sqrt(-2 * logU) * cos(2.0 * M_PI * V);
    }
}

/* q_generator + p_generator (hawaii.c:1232-1380); R0 > 0 replaces the drawn R before the
 * momenta, as the PR_MU loop does (hawaii.c:3566-3567) */
static void gen_qp(hho_mt *s, const hho_system *sys, const hho_params *p, double T, double *qp, int *draws,
                   double R0) {
    double RMIN = p->Rmin, RMAX = p->Rmax;
    /* q_generator */
    double R3 = hho_mt_drand(s) * (RMAX * RMAX * RMAX - RMIN * RMIN * RMIN) + RMIN * RMIN * RMIN;
    qp[4] = pow(R3, 1.0 / 3.0);
    qp[0] = hho_mt_drand(s) * 2.0 * M_PI;
    qp[2] = acos(2.0 * hho_mt_drand(s) - 1.0);
    *draws += 3;
    if (is_linear(sys)) {
        qp[6] = hho_mt_drand(s) * 2.0 * M_PI;
        qp[8] = acos(2.0 * hho_mt_drand(s) - 1.0);
        *draws += 2;
    }
    if (sys->system == HHO_SYS_CH4CO2) {  /* ROTOR, then LINEAR_MOLECULE (hawaii.c:1260-1290) */
        qp[6] = hho_mt_drand(s) * 2.0 * M_PI;
        qp[8] = acos(2.0 * hho_mt_drand(s) - 1.0);
        qp[10] = hho_mt_drand(s) * 2.0 * M_PI;
        qp[12] = hho_mt_drand(s) * 2.0 * M_PI;
        qp[14] = acos(2.0 * hho_mt_drand(s) - 1.0);
        *draws += 5;
    }
    if (R0 > 0) qp[4] = R0;
    /* p_generator */
    double sqrt_MUKT = sqrt(sys->mu / HkT * T);
    double sinTheta = sin(qp[2]);
    double x[3];
    for (int i = 0; i < 3; ++i) x[i] = generate_normal(s, draws);
    qp[1] = sqrt_MUKT * qp[4] * sinTheta * x[0];
    qp[3] = sqrt_MUKT * qp[4] * x[1];
    qp[5] = sqrt_MUKT * x[2];
    if (is_linear(sys)) {
        double sqrt_IIKT = sqrt(sys->II / HkT * T);
        double sin_theta = sin(qp[8]);
        double x0 = generate_normal(s, draws);
        double x1 = generate_normal(s, draws);
        qp[7] = sqrt_IIKT * sin_theta * x1;
        qp[9] = sqrt_IIKT * x0;
    }
    if (sys->system == HHO_SYS_CH4CO2) {
        /* p_generator_rotor (hawaii.c:1305-1327) */
        double sIx = sqrt(sys->II1[0] / HkT * T), sIy = sqrt(sys->II1[1] / HkT * T), sIz = sqrt(sys->II1[2] / HkT * T);
        double st = sin(qp[8]), ct = cos(qp[8]), sp = sin(qp[10]), cp = cos(qp[10]);
        double x0 = generate_normal(s, draws);
        double x1 = generate_normal(s, draws);
        double x2 = generate_normal(s, draws);
        qp[7] = sIx * st * sp * x0 + sIy * st * cp * x1 + sIz * ct * x2;
        qp[9] = sIx * cp * x0 - sIy * sp * x1;
        qp[11] = sIz * x2;
        /* p_generator_linear_molecule (hawaii.c:1292-1303) */
        double sqrt_IIKT = sqrt(sys->II / HkT * T);
        double sin_theta = sin(qp[14]);
        double y0 = generate_normal(s, draws);
        double y1 = generate_normal(s, draws);
        qp[13] = sqrt_IIKT * sin_theta * y1;
        qp[15] = sqrt_IIKT * y0;
    }
}

int hho_candidate(hho_mt *s, const hho_system *sys, const hho_params *p, double T,
                  double *qp, double *energy, int *draws) {
    *draws = 0;
    gen_qp(s, sys, p, T, qp, draws, 0.0);
    /* Hamiltonian, then reject() */
    double E = hho_hamiltonian(sys, qp);
    double u = hho_mt_drand(s);
    *draws += 1;
    double Mval = exp(-p->pesmin * HkT / T);
    double M = 1.5 * Mval;
    double kin = hho_kinetic(sys, qp);
    double q[8];
    extract_q(sys, qp, q);
    double pot = hho_pes(sys, q);
    double proposal = exp(-kin * HkT / T);
    double desired = exp(-(kin + pot) * HkT / T);
    double weight = desired / proposal / M;
    *energy = E;
    if (weight < u) return 0;
    if (p->pair_state == HHO_PS_FREE_AND_METASTABLE && E < 0.0) return 0;
    if (p->pair_state == HHO_PS_BOUND && E > 0.0) return 0;
    return 1;
}

long hho_sample(uint32_t seed, const hho_system *sys, const hho_params *p, double T,
                size_t n, double *qp_out) {
    hho_mt s;
    hho_mt_seed(&s, seed);
    int QP = hho_qp_size(sys);
    long cand = 0;
    size_t got = 0;
    double qp[16], E;
    int draws;
    while (got < n) {
        ++cand;
        if (hho_candidate(&s, sys, p, T, qp, &E, &draws)) {
            memcpy(qp_out + got * QP, qp, QP * sizeof(double));
            ++got;
        }
    }
    return cand;
}

/* ======================================================================== */
/* DOP853 with dense output (Hairer-Norsett-Wanner); step control and        */
/* initial step as in the standard published algorithm.                      */
/* ======================================================================== */
#define NMAX 16

typedef struct {
    const hho_system *sys;
    int n;
    double rtol, atol;
    long nrhs;
} integ;

static void f_eval(integ *I, const double *y, double *f) {
    hho_rhs(I->sys, y, f);
    I->nrhs++;
}

static double rms(const double *v, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += v[i] * v[i];
    return sqrt(s / n);
}

static double initial_step(integ *I, const double *y0, const double *f0, double span) {
    int n = I->n;
    double sc[NMAX], tmp[NMAX], y1[NMAX], f1[NMAX];
    for (int i = 0; i < n; ++i) sc[i] = I->atol + fabs(y0[i]) * I->rtol;
    for (int i = 0; i < n; ++i) tmp[i] = y0[i] / sc[i];
    double d0 = rms(tmp, n);
    for (int i = 0; i < n; ++i) tmp[i] = f0[i] / sc[i];
    double d1 = rms(tmp, n);
    double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
    if (h0 > span) h0 = span;
    for (int i = 0; i < n; ++i) y1[i] = y0[i] + h0 * f0[i];
    f_eval(I, y1, f1);
    for (int i = 0; i < n; ++i) tmp[i] = (f1[i] - f0[i]) / sc[i];
    double d2 = rms(tmp, n) / h0;
    double h1;
    if (d1 <= 1e-15 && d2 <= 1e-15) h1 = fmax(1e-6, h0 * 1e-3);
    else h1 = pow(0.01 / fmax(d1, d2), 1.0 / 8.0);
    return fmin(fmin(100 * h0, h1), span);
}

/* one adaptive step from (t, y, f): on success y_new/f_new/K filled, *h is the
 * step taken and *h_next the proposal.  returns 0 or HHO_ST_H_UNDERFLOW */
static int dop853_step(integ *I, double t, const double *y, const double *f, double *h_io,
                       double *h_taken, double K[16][NMAX], double *y_new, long *nrej) {
    int n = I->n;
    double h = *h_io;
    int rejected = 0;
    for (;;) {
        double min_step = 10.0 * fabs(nextafter(t, INFINITY) - t);
        if (h < min_step) return HHO_ST_H_UNDERFLOW;
        double ys[NMAX];
        memcpy(K[0], f, n * sizeof(double));
        for (int s = 1; s < 12; ++s) {
            for (int i = 0; i < n; ++i) {
                double acc = 0.0;
                for (int j = 0; j < s; ++j) acc += hh_dop853_a[s][j] * K[j][i];
                ys[i] = y[i] + h * acc;
            }
            f_eval(I, ys, K[s]);
        }
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int j = 0; j < 12; ++j) acc += hh_dop853_a[12][j] * K[j][i];
            y_new[i] = y[i] + h * acc;
        }
        f_eval(I, y_new, K[12]);
        double e5 = 0.0, e3 = 0.0;
        for (int i = 0; i < n; ++i) {
            double sc = I->atol + fmax(fabs(y[i]), fabs(y_new[i])) * I->rtol;
            double a5 = 0.0, a3 = 0.0;
            for (int j = 0; j < 13; ++j) {
                a5 += hh_dop853_e5[j] * K[j][i];
                a3 += hh_dop853_e3[j] * K[j][i];
            }
            a5 /= sc; a3 /= sc;
            e5 += a5 * a5; e3 += a3 * a3;
        }
        double err;
        if (e5 == 0.0 && e3 == 0.0) err = 0.0;
        else err = fabs(h) * e5 / sqrt((e5 + 0.01 * e3) * n);
        if (err < 1.0) {
            double fac = (err == 0.0) ? 10.0 : fmin(10.0, 0.9 * pow(err, -1.0 / 8.0));
            if (rejected) fac = fmin(1.0, fac);
            *h_taken = h;
            *h_io = h * fac;
            return 0;
        }
        h *= fmax(0.2, 0.9 * pow(err, -1.0 / 8.0));
        rejected = 1;
        (*nrej)++;
    }
}

/* dense output coefficients F[7][n] for the step (y_old, h) -> y_new */
static void dop853_dense(integ *I, const double *y_old, const double *y_new, double h,
                         double K[16][NMAX], double F[7][NMAX]) {
    int n = I->n;
    double ys[NMAX];
    for (int s = 13; s < 16; ++s) {
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int j = 0; j < s; ++j) acc += hh_dop853_a[s][j] * K[j][i];
            ys[i] = y_old[i] + h * acc;
        }
        f_eval(I, ys, K[s]);
    }
    for (int i = 0; i < n; ++i) {
        double dy = y_new[i] - y_old[i];
        F[0][i] = dy;
        F[1][i] = h * K[0][i] - dy;
        F[2][i] = 2 * dy - h * (K[12][i] + K[0][i]);
        for (int r = 0; r < 4; ++r) {
            double acc = 0.0;
            for (int j = 0; j < 16; ++j) acc += hh_dop853_d[r][j] * K[j][i];
            F[3 + r][i] = h * acc;
        }
    }
}

static void dense_eval(int n, const double *y_old, double F[7][NMAX], double x, double *y) {
    for (int i = 0; i < n; ++i) {
        double v = 0.0;
        for (int r = 6; r >= 0; --r) {
            v += F[r][i];
            v *= ((6 - r) % 2 == 0) ? x : (1.0 - x);
        }
        y[i] = y_old[i] + v;
    }
}

/* one direction of correlation_eval: samples k = 1..N-1 of mu0 . mu(t_k) */
static int half_traj_ex(const hho_system *sys, const hho_params *p, const double *y0,
                        const double mu0[3], double *corr, double *vec, int vstep, hho_traj_stats *st,
                        int *hard, int nochecks, int *exited);
static int half_traj(const hho_system *sys, const hho_params *p, const double *y0,
                     const double mu0[3], double *corr, hho_traj_stats *st, int *hard) {
    return half_traj_ex(sys, p, y0, mu0, corr, NULL, 0, st, hard, 0, NULL);
}

/* one direction of correlation_eval: samples k = 1..N-1 of mu0 . mu(t_k); with vec != NULL
 * also the dipole vector of sample k at vec + 3 * k * vstep (vstep = +-1).  nochecks (the
 * PR_MU loop, hawaii.c:3661-3688): a NaN dipole leaves its sample at zero and no other test
 * runs; *exited (optional) tells whether the branch ended by R > Rcut */
static int half_traj_ex(const hho_system *sys, const hho_params *p, const double *y0,
                        const double mu0[3], double *corr, double *vec, int vstep, hho_traj_stats *st,
                        int *hard, int nochecks, int *exited) {
    if (exited) *exited = 0;
    integ I = {sys, hho_qp_size(sys), p->rtol, p->atol, 0};
    int n = I.n;
    double y[NMAX], f[NMAX], y_new[NMAX], K[16][NMAX], F[7][NMAX], ys[NMAX];
    memcpy(y, y0, n * sizeof(double));
    f_eval(&I, y, f);
    double dt = p->sampling_time;
    double span = dt * (double)(p->N - 1);
    double h = initial_step(&I, y, f, span);
    double t = 0.0;
    size_t k = 1;
    long since = 0;
    double prev = 0.0, curr = 0.0;
    int status = HHO_OK;
    *hard = 0;
    while (k < p->N) {
        double ht;
        int rc = dop853_step(&I, t, y, f, &h, &ht, K, y_new, &st->nrej);
        if (rc) { status = rc; break; }
        st->nsteps++;
        double t_new = t + ht;
        int dense = 0;
        while (k < p->N && (double)k * dt <= t_new) {
            if (!dense) { dop853_dense(&I, y, y_new, ht, K, F); dense = 1; }
            double x = ((double)k * dt - t) / ht;
            dense_eval(n, y, F, x, ys);
            double q[8], d[3];
            extract_q(sys, ys, q);
            hho_dipole(sys, q, d);
            st->nsamples++;
            if (nochecks) {
                if (!(isnan(d[0]) || isnan(d[1]) || isnan(d[2]))) {
                    if (vec) for (int c = 0; c < 3; ++c) vec[3 * (long)k * vstep + c] = d[c];
                    if (ys[4] > p->Rcut) { ++k; if (exited) *exited = 1; goto done; }
                }
                ++k;
                since = 0;
                continue;
            }
            if (isnan(d[0]) || isnan(d[1]) || isnan(d[2])) { status = HHO_ST_NAN_DIPOLE; *hard = 1; goto done; }
            prev = curr;
            curr = mu0[0] * d[0] + mu0[1] * d[1] + mu0[2] * d[2];
            if (fabs(curr) > 1e100) { status = HHO_ST_OVERFLOW; *hard = 1; goto done; }
            if (k > 1) {
                double ratio = fabs(curr / prev);
                if (ratio > 1e10) { status = HHO_ST_JUMP; *hard = 1; goto done; }
            }
            corr[k] = curr;
            if (vec) for (int c = 0; c < 3; ++c) vec[3 * (long)k * vstep + c] = d[c];
            ++k;
            since = 0;
            if (ys[4] > p->Rcut) goto done;
        }
        t = t_new;
        memcpy(y, y_new, n * sizeof(double));
        memcpy(f, K[12], n * sizeof(double));
        if (++since > p->max_steps) { status = HHO_ST_MAXSTEPS; break; }
    }
done:
    st->nrhs += I.nrhs;
    return status;
}

int hho_correlation_eval(const hho_system *sys, const hho_params *p, const double *qp0,
                         double *crln, hho_traj_stats *st) {
    int n = hho_qp_size(sys);
    size_t N = p->N;
    double *fw = calloc(N, sizeof(double)), *bw = calloc(N, sizeof(double));
    memset(crln, 0, N * sizeof(double));
    memset(st, 0, sizeof *st);
    double q[8], mu0[3];
    extract_q(sys, qp0, q);
    hho_dipole(sys, q, mu0);
    fw[0] = bw[0] = mu0[0] * mu0[0] + mu0[1] * mu0[1] + mu0[2] * mu0[2];
    int hard = 0;
    st->status_fwd = half_traj(sys, p, qp0, mu0, fw, st, &hard);
    if (!hard) {
        double y[NMAX];
        memcpy(y, qp0, n * sizeof(double));
        for (int i = 1; i < n; i += 2) y[i] = -y[i];   /* invert_momenta (hawaii.c:1171-1188) */
        st->status_bwd = half_traj(sys, p, y, mu0, bw, st, &hard);
    }
    if (hard) {
        st->failed = 1;      /* reference returns 1: crln stays zero */
    } else {
        for (size_t i = 0; i < N; ++i) crln[i] = 0.5 * (fw[i] + bw[i]) * ALU * ALU * ALU;
    }
    free(fw); free(bw);
    return st->failed;
}

int hho_correlation_parts(const hho_system *sys, const hho_params *p, const double *qp0,
                          double *fw, double *bw, hho_traj_stats *st) {
    int n = hho_qp_size(sys);
    size_t N = p->N;
    memset(fw, 0, N * sizeof(double));
    memset(bw, 0, N * sizeof(double));
    memset(st, 0, sizeof *st);
    double q[8], mu0[3];
    extract_q(sys, qp0, q);
    hho_dipole(sys, q, mu0);
    fw[0] = bw[0] = mu0[0] * mu0[0] + mu0[1] * mu0[1] + mu0[2] * mu0[2];
    int hard = 0;
    st->status_fwd = half_traj(sys, p, qp0, mu0, fw, st, &hard);
    double y[NMAX];
    memcpy(y, qp0, n * sizeof(double));
    for (int i = 1; i < n; i += 2) y[i] = -y[i];
    int hard2 = 0;
    st->status_bwd = half_traj(sys, p, y, mu0, bw, st, &hard2);
    st->failed = hard || hard2;
    return st->failed;
}

/* correlation_eval_zimmerman_trick (src/hawaii.c:1888-2114): dipole vectors d[2N-1] with
 * d[N-1] = mu0, d[N-1+k] = mu(t_k), d[N-1-k] = mu(-t_k) (zero past an exit), then
 * crln[s] = sum_{c < N} d[c] . d[c+s] * ALU^3 / N.  A failure of either branch returns 1
 * with crln zero, like the reference's return 1 */
int hho_correlation_eval_zimmermann(const hho_system *sys, const hho_params *p, const double *qp0,
                                    double *crln, hho_traj_stats *st) {
    int n = hho_qp_size(sys);
    size_t N = p->N;
    double *d = calloc(3 * (2 * N - 1), sizeof(double));
    double *tmp = calloc(N, sizeof(double));
    memset(crln, 0, N * sizeof(double));
    memset(st, 0, sizeof *st);
    double q[8], mu0[3];
    extract_q(sys, qp0, q);
    hho_dipole(sys, q, mu0);
    double *centre = d + 3 * (N - 1);
    for (int c = 0; c < 3; ++c) centre[c] = mu0[c];
    int hard = 0;
    st->status_fwd = half_traj_ex(sys, p, qp0, mu0, tmp, centre, 1, st, &hard, 0, NULL);
    if (!hard) {
        double y[NMAX];
        memcpy(y, qp0, n * sizeof(double));
        for (int i = 1; i < n; i += 2) y[i] = -y[i];
        st->status_bwd = half_traj_ex(sys, p, y, mu0, tmp, centre, -1, st, &hard, 0, NULL);
    }
    if (hard) {
        st->failed = 1;
    } else {
        for (size_t s = 0; s < N; ++s) {
            double acc = 0.0;
            for (size_t c = 0; c < N; ++c)
                acc += (d[3 * c] * d[3 * (c + s)] + d[3 * c + 1] * d[3 * (c + s) + 1] +
                        d[3 * c + 2] * d[3 * (c + s) + 2]) * ALU * ALU * ALU;
            crln[s] = acc / (double)N;
        }
    }
    free(d);
    free(tmp);
    return st->failed;
}

static void fft_backward(double *re, double *im, size_t L);

/* PR_MU (calculate_spectral_function_using_prmu_representation_and_save, hawaii.c:3148-3978)
 * without requantization, collision times, spin weights and histograms.  n trajectories are
 * drawn from the stream of `seed` (q_generator, R := R0, p_generator, pR made inward; no
 * rejection step); each is integrated forward with samples at t = (k+1) dt, k = 0..N-1, until
 * R > R0; its dipole components are apodized (Connes), Fourier transformed and
 * sf[i] += SF_COEFF pR/mu sum_c |F_c(i)|^2 for i < L.  A trajectory whose integration fails, or
 * that is still inside R0 after N samples (unless allow_trunc), is skipped and not counted.
 * qp_out (optional) receives the drawn phase points.  Returns the trajectories counted. */
/* ---- requantization of the linear monomer in PR_MU ------------------------------- */
/* find_closest_integer / find_closest_half_integer (src/hawaii.c:360-393) */
static double req_closest_ref(int mode, double j) {
    if (mode == 1) return round(j);
    if (j < 0.25) return 0.0;
    if (j < 1.0) return (fabs(j - 0.5) < fabs(j - 1.5)) ? 0.5 : 1.5;
    double r = 0.0;
    while (j - r >= 1.0) r += 1.0;
    double lower = r + 0.5, higher = r + 1.5;
    return (fabs(j - lower) < fabs(j - higher)) ? lower : higher;
}

/* j_monomer of the linear monomer at qp[6..9] = (phi, p_phi, theta, p_theta)
 * (src/hawaii.c:398-431) */
static double j_len(const double *qp) {
    double phi = qp[6], pphi = qp[7], th = qp[8], pth = qp[9];
    double j0 = -pth * sin(phi) - pphi * cos(phi) / tan(th);
    double j1 = pth * cos(phi) - pphi * sin(phi) / tan(th);
    return sqrt(j0 * j0 + j1 * j1 + pphi * pphi);
}

/* trajectory_apply_requantization (src/trajectory.c:93-136) */
static void req_apply(int mode, double *qp) {
    double jl = j_len(qp);
    double s = (jl > 1e-15) ? req_closest_ref(mode, jl) / jl : 0.0;
    qp[7] *= s;
    qp[9] *= s;
}

/* torque_monomer (src/hawaii.c:433-472): |tau| from dV/dphi, dV/dtheta of monomer 1 */
static double torque_len(const hho_system *sys, const double *qp) {
    double q[8], dV[8];
    extract_q(sys, qp, q);
    hho_dpes(sys, q, dV);
    double phi = qp[6], th = qp[8], dphi = dV[3], dth = dV[4];
    double tx = sin(phi) * dth + cos(phi) / tan(th) * dphi;
    double ty = -cos(phi) * dth + sin(phi) / tan(th) * dphi;
    double tz = -dphi;
    return sqrt(tx * tx + ty * ty + tz * tz);
}

/* one DOP853 step from (t, y, f) whose attempts are cut to end at t_land when they
 * would pass it; *landed tells whether the accepted step ends there.  A cut step that
 * is accepted keeps the longer of the current and the proposed next step. */
static int dop853_step_land(integ *I, double t, const double *y, const double *f, double *h_io,
                            double *h_taken, double K[16][NMAX], double *y_new, long *nrej, double t_land,
                            int *landed) {
    double h = *h_io;
    for (;;) {
        double h_att = h;
        int clamp = 0;
        if (h_att >= t_land - t) { h_att = t_land - t; clamp = 1; }
        double hh = h_att, ht = 0.0;
        long nr0 = *nrej;
        int rc = dop853_step(I, t, y, f, &hh, &ht, K, y_new, nrej);
        if (rc) return rc;
        if (*nrej == nr0) {   /* accepted at the first attempt of size h_att */
            *h_taken = h_att;
            *h_io = clamp ? fmax(h, hh) : hh;
            *landed = clamp;
            return 0;
        }
        /* dop853_step shrank and retried internally; its accepted step is shorter
         * than t_land - t, so the step did not land */
        *h_taken = ht;
        *h_io = hh;
        *landed = 0;
        return 0;
    }
}

/* PR_MU branch with requantization (src/hawaii.c:3604-3700): steps land on every sample
 * time; at sample k the switch of sample k - 1 requantizes j (and restarts the stages),
 * the torque at the sample then updates the switch (on after `len` torques <= limit,
 * off after `len` >= limit; the cache starts with zeros); the dipole is stored unless
 * NaN, and the branch ends after R > Rcut */
static int half_traj_req(const hho_system *sys, const hho_params *p, const double *y0, const hho_req *rq,
                         double *vec, hho_traj_stats *st, int *exited) {
    *exited = 0;
    integ I = {sys, hho_qp_size(sys), p->rtol, p->atol, 0};
    int n = I.n;
    double y[NMAX], f[NMAX], y_new[NMAX], K[16][NMAX];
    memcpy(y, y0, n * sizeof(double));
    f_eval(&I, y, f);
    double dt = p->sampling_time;
    double h = initial_step(&I, y, f, dt * (double)(p->N - 1));
    double t = 0.0;
    size_t k = 1;
    long since = 0;
    int on = 1, le = rq->len, ge = 0;
    int status = HHO_OK;
    while (k < p->N) {
        double ht;
        int landed = 0;
        int rc = dop853_step_land(&I, t, y, f, &h, &ht, K, y_new, &st->nrej, (double)k * dt, &landed);
        if (rc) { status = rc; break; }
        st->nsteps++;
        if (landed) {
            memcpy(f, K[12], n * sizeof(double));
            double tq = torque_len(sys, y_new);
            if (on) {
                req_apply(rq->mode, y_new);
                f_eval(&I, y_new, f);
            }
            le = (tq <= rq->limit) ? (le + 1 > rq->len ? rq->len : le + 1) : 0;
            ge = (tq >= rq->limit) ? (ge + 1 > rq->len ? rq->len : ge + 1) : 0;
            if (le >= rq->len) on = 1;
            else if (ge >= rq->len) on = 0;
            double q[8], d[3];
            extract_q(sys, y_new, q);
            hho_dipole(sys, q, d);
            st->nsamples++;
            t = (double)k * dt;
            memcpy(y, y_new, n * sizeof(double));
            since = 0;
            if (!(isnan(d[0]) || isnan(d[1]) || isnan(d[2]))) {
                for (int c = 0; c < 3; ++c) vec[3 * (long)k + c] = d[c];
                if (y[4] > p->Rcut) { ++k; *exited = 1; break; }
            }
            ++k;
        } else {
            t += ht;
            memcpy(y, y_new, n * sizeof(double));
            memcpy(f, K[12], n * sizeof(double));
            if (++since > p->max_steps) { status = HHO_ST_MAXSTEPS; break; }
        }
    }
    st->nrhs += I.nrhs;
    return status;
}

long hho_prmu_req(const hho_system *sys, const hho_params *p, double T, double R0, int allow_trunc,
                  uint32_t seed, size_t n, const hho_req *rq, double *sf, size_t L, double *qp_out) {
    hho_mt s;
    hho_mt_seed(&s, seed);
    const size_t N = p->N;
    const int QP = hho_qp_size(sys);
    const double SF_COEFF = Hartree * pow(ALU, 6) * ATU * R0 * R0 * p->sampling_time * p->sampling_time;
    hho_params pp = *p;
    pp.N = N + 1;
    pp.Rcut = R0;
    double *re = malloc(N * sizeof(double)), *im = malloc(N * sizeof(double));
    double *vec = calloc(3 * (N + 1), sizeof(double));
    memset(sf, 0, L * sizeof(double));
    long counted = 0;
    for (size_t t = 0; t < n; ++t) {
        double qp[16];
        int draws = 0;
        gen_qp(&s, sys, p, T, qp, &draws, R0);
        if (qp[5] > 0.0) qp[5] = -qp[5];
        if (qp_out) memcpy(qp_out + t * QP, qp, QP * sizeof(double));
        const double pr_mu = -qp[5] / sys->mu;
        req_apply(rq->mode, qp);   /* the switch is on when the trajectory starts */
        double w = 1.0;
        if (rq->mode == 2 && (rq->even_w > 0.0 || rq->odd_w > 0.0)) {
            int j_int = (int)round(j_len(qp) - 1.5);
            w = (j_int % 2 == 0) ? rq->even_w : rq->odd_w;
        }
        hho_traj_stats st;
        memset(&st, 0, sizeof st);
        memset(vec, 0, 3 * (N + 1) * sizeof(double));
        int exited = 0;
        int status = half_traj_req(sys, &pp, qp, rq, vec, &st, &exited);
        if (status != HHO_OK) continue;
        if (!exited && !allow_trunc) continue;
        for (int c = 0; c < 3; ++c) {
            for (size_t j = 0; j < N; ++j) {
                double r = (double)j / (double)N;
                re[j] = vec[3 * (j + 1) + c] * (1.0 - r * r) * (1.0 - r * r);
                im[j] = 0.0;
            }
            fft_backward(re, im, N);
            for (size_t i = 0; i < L; ++i) sf[i] += SF_COEFF * pr_mu * (re[i] * re[i] + im[i] * im[i]) * w;
        }
        ++counted;
    }
    free(re); free(im); free(vec);
    return counted;
}

long hho_prmu(const hho_system *sys, const hho_params *p, double T, double R0, int allow_trunc, uint32_t seed,
              size_t n, double *sf, size_t L, double *qp_out) {
    hho_mt s;
    hho_mt_seed(&s, seed);
    const size_t N = p->N;
    const int QP = hho_qp_size(sys);
    const double SF_COEFF = Hartree * pow(ALU, 6) * ATU * R0 * R0 * p->sampling_time * p->sampling_time;
    hho_params pp = *p;
    pp.N = N + 1;       /* samples k = 1..N at t = k dt */
    pp.Rcut = R0;
    double *re = malloc(N * sizeof(double)), *im = malloc(N * sizeof(double));
    double *vec = calloc(3 * (N + 1), sizeof(double));
    double *tmp = calloc(N + 1, sizeof(double));
    memset(sf, 0, L * sizeof(double));
    long counted = 0;
    for (size_t t = 0; t < n; ++t) {
        double qp[16];
        int draws = 0;
        gen_qp(&s, sys, p, T, qp, &draws, R0);
        if (qp[5] > 0.0) qp[5] = -qp[5];
        if (qp_out) memcpy(qp_out + t * QP, qp, QP * sizeof(double));
        const double pr_mu = -qp[5] / sys->mu;
        hho_traj_stats st;
        memset(&st, 0, sizeof st);
        memset(vec, 0, 3 * (N + 1) * sizeof(double));
        int hard = 0, exited = 0;
        const double mu0[3] = {0, 0, 0};
        int status = half_traj_ex(sys, &pp, qp, mu0, tmp, vec, 1, &st, &hard, 1, &exited);
        if (status != HHO_OK) continue;
        if (!exited && !allow_trunc) continue;
        for (int c = 0; c < 3; ++c) {
            for (size_t j = 0; j < N; ++j) {
                double r = (double)j / (double)N;   /* connes_apodization, hawaii.c:5401-5410 */
                re[j] = vec[3 * (j + 1) + c] * (1.0 - r * r) * (1.0 - r * r);
                im[j] = 0.0;
            }
            fft_backward(re, im, N);
            for (size_t i = 0; i < L; ++i) sf[i] += SF_COEFF * pr_mu * (re[i] * re[i] + im[i] * im[i]);
        }
        ++counted;
    }
    free(re); free(im); free(vec); free(tmp);
    return counted;
}

int hho_propagate(const hho_system *sys, const hho_params *p, const double *qp0,
                  double t_end, double *qp_out, long *nsteps) {
    integ I = {sys, hho_qp_size(sys), p->rtol, p->atol, 0};
    int n = I.n;
    double y[NMAX], f[NMAX], y_new[NMAX], K[16][NMAX], F[7][NMAX];
    memcpy(y, qp0, n * sizeof(double));
    f_eval(&I, y, f);
    double dt = p->sampling_time;
    double h = initial_step(&I, y, f, dt * (double)(p->N - 1));
    double t = 0.0;
    long ns = 0, nrej = 0;
    for (;;) {
        double ht;
        int rc = dop853_step(&I, t, y, f, &h, &ht, K, y_new, &nrej);
        if (rc) return rc;
        ++ns;
        if (t + ht >= t_end) {
            dop853_dense(&I, y, y_new, ht, K, F);
            dense_eval(n, y, F, (t_end - t) / ht, qp_out);
            break;
        }
        t += ht;
        memcpy(y, y_new, n * sizeof(double));
        memcpy(f, K[12], n * sizeof(double));
    }
    if (nsteps) *nsteps = ns;
    return 0;
}

typedef struct {
    const hho_system *sys;
    const hho_params *p;
    const double *qp0;
    size_t begin, end;
    double *sum;
    hho_traj_stats *stats;
    const double *w;   /* CORRELATION_ARRAY: [n][n_sat] weights, or NULL */
    int n_sat;
    int zimmermann;
} corr_job;

static void *corr_worker(void *arg) {
    corr_job *J = arg;
    int n = hho_qp_size(J->sys);
    size_t N = J->p->N;
    double *crln = malloc(N * sizeof(double));
    for (size_t i = J->begin; i < J->end; ++i) {
        hho_traj_stats st;
        if (J->zimmermann) hho_correlation_eval_zimmermann(J->sys, J->p, J->qp0 + i * n, crln, &st);
        else hho_correlation_eval(J->sys, J->p, J->qp0 + i * n, crln, &st);
        if (J->w) {
            for (int s = 0; s < J->n_sat; ++s)
                for (size_t k = 0; k < N; ++k) J->sum[s * N + k] += J->w[i * J->n_sat + s] * crln[k];
        } else {
            for (size_t k = 0; k < N; ++k) J->sum[k] += J->p->ppf_ratio * crln[k];
        }
        if (J->stats) J->stats[i] = st;
    }
    free(crln);
    return NULL;
}

int hho_correlation_sum(const hho_system *sys, const hho_params *p, const double *qp0,
                        size_t n, int nthreads, double *crln_sum, hho_traj_stats *stats) {
    if (nthreads < 1) nthreads = 1;
    size_t N = p->N;
    pthread_t th[256];
    corr_job jobs[256];
    if (nthreads > 256) nthreads = 256;
    for (int w = 0; w < nthreads; ++w) {
        jobs[w] = (corr_job){sys, p, qp0, n * w / nthreads, n * (w + 1) / nthreads,
                             calloc(N, sizeof(double)), stats, NULL, 0, p->zimmermann};
        pthread_create(&th[w], NULL, corr_worker, &jobs[w]);
    }
    memset(crln_sum, 0, N * sizeof(double));
    for (int w = 0; w < nthreads; ++w) {
        pthread_join(th[w], NULL);
        for (size_t k = 0; k < N; ++k) crln_sum[k] += jobs[w].sum[k];
        free(jobs[w].sum);
    }
    return 0;
}

/* ======================================================================== */
/* CF -> SF (src/hawaii.c:5401-5410, 5478-5553, 5569-5601)                   */
/* ======================================================================== */
static void fft_backward(double *re, double *im, size_t L) {
    /* iterative radix-2, unnormalised exp(+i...) */
    for (size_t i = 1, j = 0; i < L; ++i) {
        size_t bit = L >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = re[i]; re[i] = re[j]; re[j] = t;
            t = im[i]; im[i] = im[j]; im[j] = t;
        }
    }
    for (size_t len = 2; len <= L; len <<= 1) {
        size_t half = len / 2;
        for (size_t k = 0; k < half; ++k) {
            double ang = 2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (size_t i = k; i < L; i += len) {
                size_t j = i + half;
                double xr = re[j] * wr - im[j] * wi;
                double xi = re[j] * wi + im[j] * wr;
                re[j] = re[i] - xr; im[j] = im[i] - xi;
                re[i] += xr; im[i] += xi;
            }
        }
    }
}

int hho_idct_cf_to_sf(double *cf, size_t N, double dt, double *nu, double *sf) {
    if (N == 0 || (N & (N - 1))) return -1;
    double Xscale = 1.0 / LightSpeed_cm / ATU / 2.0 / M_PI;
    double Yscale = ATU * ADIPMOMU * ADIPMOMU / (4.0 * M_PI * EPSILON0);
    double tmax_a = dt * (double)N;
    for (size_t i = 0; i < N; ++i) {
        double tc = dt * (double)i;
        double f = (1.0 - (tc / tmax_a) * (tc / tmax_a)) * (1.0 - (tc / tmax_a) * (tc / tmax_a));
        cf[i] *= f;
    }
    size_t L = 2 * N;
    double *re = calloc(L, sizeof(double)), *im = calloc(L, sizeof(double));
    for (size_t k = 0; k < N; ++k) {
        double a = M_PI * (double)k / (2.0 * N);
        re[k] = cf[k] * cos(a) / (2.0 * N);
        im[k] = cf[k] * sin(a) / (2.0 * N);
    }
    for (size_t k = N + 1; k < L; ++k) {
        size_t i = L - k;
        double a = M_PI * (double)k / (2.0 * N);
        re[k] = -cf[i] * cos(a) / (2.0 * N);
        im[k] = -cf[i] * sin(a) / (2.0 * N);
    }
    fft_backward(re, im, L);
    double tmax = (double)N * dt;
    for (size_t i = 0; i < N; ++i) {
        nu[i] = (double)i * M_PI / tmax * Xscale;
        sf[i] = re[i] * tmax / M_PI * Yscale;
    }
    free(re); free(im);
    return 0;
}

/* ======================================================================== */
/* Zeroth moment by plain Monte Carlo (the M0 integrand of                  */
/* src/hep_hawaii.cpp:148-201 sampled with R uniform on [Rmin, Rmax],       */
/* isotropic angles and Gaussian momenta):                                   */
/*   M0(T) = ZeroCoeff * 4 pi (Rmax - Rmin) < R^2 |mu|^2 exp(-V/kT) 1[filter] >*/
/* Only the kinetic energy K = kT * kappa of the momenta enters; kappa is    */
/* half a chi^2 with 3 (atom-atom) or 5 (linear-atom) degrees of freedom,    */
/* drawn by Box-Muller sums.                                                 */
/* ======================================================================== */
static inline double u24(uint32_t w) { return ((double)(w >> 8) + 0.5) * (1.0 / 16777216.0); }

typedef struct {
    const hho_system *sys;
    const hho_params *p;
    const double *T;
    int nT;
    uint64_t begin, end, seed;
    double *wsum, *wsq;
    int moment;  /* 0: M0, 2: M2 */
} m0_job;

/* Second moment (calculate_M2, src/hawaii.c:1524-1617; integrand_M2,               */
/* src/hep_hawaii.cpp:228-330) in the reference's own coordinates: D = dmu/dq by     */
/* central differences with h = 1e-3 in q = (Phi, Theta, R[, phi, theta]) as there,  */
/* and the momentum average at kinetic energy K, E[|D^T qdot|^2 | K] =              */
/* (2K/nu) sum_i |dmu/dq_i|^2 (M^-1)_ii with the diagonal inverse metric of H:       */
/* 1/(mu R^2 sin^2 Theta), 1/(mu R^2), 1/mu, 1/(I sin^2 theta), 1/I.                */
static double m2_geometry_q(const hho_system *sys, const double *q0, int nq) {
    const double h = 1.0e-3;
    double q[5], dp[3], dm[3], g = 0.0;
    for (int i = 0; i < nq; ++i) q[i] = q0[i];
    const double R = q0[2], sT = sin(q0[1]);
    double minv[5] = {1.0 / (sys->mu * R * R * sT * sT), 1.0 / (sys->mu * R * R), 1.0 / sys->mu, 0.0, 0.0};
    if (nq == 5) {
        const double st = sin(q0[4]);
        minv[3] = 1.0 / (sys->II * st * st);
        minv[4] = 1.0 / sys->II;
    }
    for (int i = 0; i < nq; ++i) {
        q[i] = q0[i] + h;
        hho_dipole(sys, q, dp);
        q[i] = q0[i] - h;
        hho_dipole(sys, q, dm);
        q[i] = q0[i];
        double s2 = 0.0;
        for (int c = 0; c < 3; ++c) s2 += (dp[c] - dm[c]) * (dp[c] - dm[c]);
        g += s2 / (4.0 * h * h) * minv[i];
    }
    return g;
}

static void *m0_worker(void *arg) {
    m0_job *J = arg;
    int nT = J->nT;
    double invkT[64];
    for (int t = 0; t < nT; ++t) invkT[t] = HkT / J->T[t];
    uint32_t key[2] = {(uint32_t)J->seed, (uint32_t)(J->seed >> 32)};
    double Rmin = J->p->Rmin, dR = J->p->Rmax - J->p->Rmin;
    for (uint64_t i = J->begin; i < J->end; ++i) {
        uint32_t w[12];
        for (uint32_t c = 0; c < 3; ++c) {
            uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), c, 0u};
            hho_philox4x32_10(ctr, key, w + 4 * c);
        }
        double R = Rmin + dR * u24(w[0]);
        double Phi = 2.0 * M_PI * u24(w[1]);
        double cT = 2.0 * u24(w[2]) - 1.0;
        double q[5] = {Phi, acos(cT), R, 0.0, 0.0};
        double kappa;
        double zc = cos(2.0 * M_PI * u24(w[8]));
        if (is_linear(J->sys)) {
            q[3] = 2.0 * M_PI * u24(w[3]);
            q[4] = acos(2.0 * u24(w[4]) - 1.0);
            kappa = -log(u24(w[5])) - log(u24(w[6])) - log(u24(w[7])) * zc * zc;
        } else {
            kappa = -log(u24(w[5])) - log(u24(w[7])) * zc * zc;
        }
        double V = hho_pes(J->sys, q);
        double d[3];
        hho_dipole(J->sys, q, d);
        double base = R * R * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (J->moment == 2) {
            const int nq = is_linear(J->sys) ? 5 : 3;
            base = R * R * m2_geometry_q(J->sys, q, nq) * 2.0 / (is_linear(J->sys) ? 5.0 : 3.0);
        }
        for (int t = 0; t < nT; ++t) {
            double H = kappa / invkT[t] + V;
            int keep = 1;
            if (J->p->pair_state == HHO_PS_FREE_AND_METASTABLE) keep = (H >= 0.0);
            else if (J->p->pair_state == HHO_PS_BOUND) keep = (H <= 0.0);
            double wv = keep ? base * exp(-V * invkT[t]) : 0.0;
            if (J->moment == 2) wv *= kappa / invkT[t];  /* (2K/nu) G, K = kappa kT */
            J->wsum[t] += wv;
            J->wsq[t] += wv * wv;
        }
    }
    return NULL;
}

static int moment_mc(const hho_system *sys, const hho_params *p, const double *T, int nT,
                     uint64_t n_samples, uint64_t seed, uint64_t offset, int nthreads,
                     double *wsum, double *wsq, int moment) {
    if (sys->system == HHO_SYS_CH4CO2) return -1;  /* no CH4-CO2 moment integrand */
    if (nT > 64 || nT < 1) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    m0_job jobs[256];
    for (int w = 0; w < nthreads; ++w) {
        jobs[w] = (m0_job){sys, p, T, nT, offset + n_samples * w / nthreads,
                           offset + n_samples * (w + 1) / nthreads, seed,
                           calloc(nT, sizeof(double)), calloc(nT, sizeof(double)), moment};
        pthread_create(&th[w], NULL, m0_worker, &jobs[w]);
    }
    for (int t = 0; t < nT; ++t) wsum[t] = wsq[t] = 0.0;
    for (int w = 0; w < nthreads; ++w) {
        pthread_join(th[w], NULL);
        for (int t = 0; t < nT; ++t) { wsum[t] += jobs[w].wsum[t]; wsq[t] += jobs[w].wsq[t]; }
        free(jobs[w].wsum); free(jobs[w].wsq);
    }
    return 0;
}

int hho_m0(const hho_system *sys, const hho_params *p, const double *T, int nT,
           uint64_t n_samples, uint64_t seed, uint64_t offset, int nthreads,
           double *wsum, double *wsq) {
    return moment_mc(sys, p, T, nT, n_samples, seed, offset, nthreads, wsum, wsq, 0);
}

int hho_m2(const hho_system *sys, const hho_params *p, const double *T, int nT,
           uint64_t n_samples, uint64_t seed, uint64_t offset, int nthreads,
           double *wsum, double *wsq) {
    return moment_mc(sys, p, T, nT, n_samples, seed, offset, nthreads, wsum, wsq, 2);
}

double hho_m0_scale(const hho_params *p) { return ZeroCoeff * 4.0 * M_PI * (p->Rmax - p->Rmin); }
double hho_m2_scale(const hho_params *p) { return SecondCoeff * 4.0 * M_PI * (p->Rmax - p->Rmin); }

/* ======================================================================== */
/* VEGAS (c_mpi_perform_integration, src/hep_hawaii.cpp:332-389, through    */
/* hep-mc 0.7, absent here): Lepage's algorithm (J. Comput. Phys. 27 (1978) */
/* 192) restated.  The integrand and its unit-hypercube map follow          */
/* integrand_M0 / integrand_pf and transform_variables                     */
/* (src/hep_hawaii.cpp:8-201), including x[0] for both R and Phi.  Sample i */
/* of iteration it draws Philox4x32-10 words at counter (id_lo, id_hi, b, 0),*/
/* id = it * npoints + i, b = 0..2; u = (w + 1/2) 2^-32.                    */
/* ======================================================================== */
#define VG_NB 128
#define VG_MAXD 10

static double vg_integrand(const hho_system *sys, const hho_params *p, int integrand, double invkT,
                           const double *x, int D) {
    double qp[16], jac = 1.0;
    qp[4] = 1.0 / x[0]; jac *= qp[4] * qp[4];
    qp[5] = tan(M_PI * (x[5] - 0.5)); jac *= M_PI * (1.0 + qp[5] * qp[5]);
    qp[0] = x[0] * 2.0 * M_PI; jac *= 2.0 * M_PI;
    qp[1] = tan(M_PI * (x[1] - 0.5)); jac *= M_PI * (1.0 + qp[1] * qp[1]);
    qp[2] = x[2] * M_PI; jac *= M_PI;
    qp[3] = tan(M_PI * (x[3] - 0.5)); jac *= M_PI * (1.0 + qp[3] * qp[3]);
    if (D == 10) {
        qp[6] = x[6] * 2.0 * M_PI; jac *= 2.0 * M_PI;
        qp[7] = tan(M_PI * (x[7] - 0.5)); jac *= M_PI * (1.0 + qp[7] * qp[7]);
        qp[8] = x[8] * M_PI; jac *= M_PI;
        qp[9] = tan(M_PI * (x[9] - 0.5)); jac *= M_PI * (1.0 + qp[9] * qp[9]);
    }
    double R = qp[4];
    if (R < p->Rmin || R > p->Rmax) return 0.0;
    double H = hho_hamiltonian(sys, qp);
    if (p->pair_state == HHO_PS_FREE_AND_METASTABLE && H < 0.0) return 0.0;
    if (p->pair_state == HHO_PS_BOUND && H > 0.0) return 0.0;
    double dipsq = 1.0;
    if (integrand == 0) {
        double q[8], d[3];
        extract_q(sys, qp, q);
        hho_dipole(sys, q, d);
        dipsq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    }
    return jac * dipsq * exp(-H * invkT);
}

typedef struct {
    const hho_system *sys;
    const hho_params *p;
    int integrand, D;
    double invkT;
    uint64_t id0, begin, end, seed;
    const double *edges;
    double s, s2;
    double *hist;
} vg_job;

static void *vg_worker(void *arg) {
    vg_job *J = arg;
    uint32_t key[2] = {(uint32_t)J->seed, (uint32_t)(J->seed >> 32)};
    for (uint64_t i = J->begin; i < J->end; ++i) {
        uint64_t id = J->id0 + i;
        uint32_t w[12];
        for (uint32_t c = 0; c < 3; ++c) {
            uint32_t ctr[4] = {(uint32_t)id, (uint32_t)(id >> 32), c, 0u};
            hho_philox4x32_10(ctr, key, w + 4 * c);
        }
        double x[VG_MAXD], wgt = 1.0;
        int bin[VG_MAXD];
        for (int d = 0; d < J->D; ++d) {
            double u = ((double)w[d] + 0.5) / 4294967296.0;
            double v = u * VG_NB;
            int b = (int)v;
            if (b > VG_NB - 1) b = VG_NB - 1;
            const double *e = J->edges + d * (VG_NB + 1);
            x[d] = e[b] + (v - b) * (e[b + 1] - e[b]);
            wgt *= VG_NB * (e[b + 1] - e[b]);
            bin[d] = b;
        }
        double F = vg_integrand(J->sys, J->p, J->integrand, J->invkT, x, J->D) * wgt;
        J->s += F;
        J->s2 += F * F;
        if (F != 0.0)
            for (int d = 0; d < J->D; ++d) J->hist[d * VG_NB + bin[d]] += F * F;
    }
    return NULL;
}

/* one refinement step per dimension: 3-point smoothing (2-point at the ends), the
 * compression m_i = ((1 - r_i) / ln(1 / r_i))^alpha of the normalised r_i, and new
 * edges at equal steps of the cumulative m */
static void vg_refine(double *edges, const double *hist, int D, double alpha) {
    for (int d = 0; d < D; ++d) {
        const double *h = hist + d * VG_NB;
        double *e = edges + d * (VG_NB + 1);
        double sm[VG_NB], m[VG_NB], cum[VG_NB + 1], ne[VG_NB + 1], tot = 0.0, M = 0.0;
        sm[0] = 0.5 * (h[0] + h[1]);
        for (int i = 1; i < VG_NB - 1; ++i) sm[i] = (h[i - 1] + h[i] + h[i + 1]) / 3.0;
        sm[VG_NB - 1] = 0.5 * (h[VG_NB - 2] + h[VG_NB - 1]);
        for (int i = 0; i < VG_NB; ++i) tot += sm[i];
        if (!(tot > 0.0)) continue;
        for (int i = 0; i < VG_NB; ++i) {
            double r = sm[i] / tot;
            m[i] = (r > 0.0 && r < 1.0) ? pow((1.0 - r) / log(1.0 / r), alpha) : (r >= 1.0 ? 1.0 : 0.0);
            M += m[i];
        }
        if (!(M > 0.0)) continue;
        cum[0] = 0.0;
        for (int i = 0; i < VG_NB; ++i) cum[i + 1] = cum[i] + m[i];
        ne[0] = e[0];
        ne[VG_NB] = e[VG_NB];
        int j = 0;
        for (int k = 1; k < VG_NB; ++k) {
            double target = M * k / VG_NB;
            while (j < VG_NB - 1 && cum[j + 1] < target) ++j;
            double fr = m[j] > 0.0 ? (target - cum[j]) / m[j] : 0.0;
            if (fr < 0.0) fr = 0.0;
            if (fr > 1.0) fr = 1.0;
            ne[k] = e[j] + fr * (e[j + 1] - e[j]);
        }
        memcpy(e, ne, sizeof ne);
    }
}

int hho_vegas(const hho_system *sys, const hho_params *p, int integrand, double T, uint64_t niter,
              uint64_t npoints, uint64_t seed, int nthreads, double *m, double *q) {
    if (sys->system == HHO_SYS_CH4CO2 || niter == 0 || npoints < 2) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    const int D = hho_qp_size(sys);
    double edges[VG_MAXD * (VG_NB + 1)];
    for (int d = 0; d < D; ++d)
        for (int k = 0; k <= VG_NB; ++k) edges[d * (VG_NB + 1) + k] = (double)k / VG_NB;
    double wsum = 0.0, wv = 0.0, v0 = 0.0, e0 = 0.0;
    for (uint64_t it = 0; it < niter; ++it) {
        pthread_t th[256];
        vg_job jobs[256];
        for (int t = 0; t < nthreads; ++t) {
            jobs[t] = (vg_job){sys, p, integrand, D, HkT / T, it * npoints, npoints * t / nthreads,
                               npoints * (t + 1) / nthreads, seed, edges, 0.0, 0.0,
                               calloc(D * VG_NB, sizeof(double))};
            pthread_create(&th[t], NULL, vg_worker, &jobs[t]);
        }
        double S = 0.0, S2 = 0.0, hist[VG_MAXD * VG_NB];
        memset(hist, 0, sizeof hist);
        for (int t = 0; t < nthreads; ++t) {
            pthread_join(th[t], NULL);
            S += jobs[t].s;
            S2 += jobs[t].s2;
            for (int i = 0; i < D * VG_NB; ++i) hist[i] += jobs[t].hist[i];
            free(jobs[t].hist);
        }
        double n = (double)npoints, mean = S / n;
        double var = (S2 / n - mean * mean);
        if (var < 0.0) var = 0.0;
        var /= (n - 1.0);
        if (it == 0) { v0 = mean; e0 = sqrt(var); }
        else if (var > 0.0) { wsum += 1.0 / var; wv += mean / var; }
        if (it + 1 < niter) vg_refine(edges, hist, D, 1.5);
    }
    if (niter == 1 || !(wsum > 0.0)) { *m = v0; *q = e0; }
    else { *m = wv / wsum; *q = sqrt(1.0 / wsum); }
    return 0;
}

/* analytic_full_partition_function_by_V (src/hawaii.c:5071-5090) */
double hho_analytic_pf(const hho_system *sys, double T) {
    if (sys->system == HHO_SYS_HEAR) return pow(2.0 * M_PI * sys->mu * T / HkT, 1.5);
    return 4.0 * M_PI * pow(2.0 * M_PI * T / HkT, 2.5) * pow(sys->mu, 1.5) * sys->II;
}

/* ======================================================================== */
/* CORRELATION_ARRAY (src/hawaii.c:2361-2793): trajectories sampled at the   */
/* base temperature T0 are reweighted to satellite temperatures Ts           */
/* (accumulation at hawaii.c:2640-2676)                                      */
/* ======================================================================== */
void hho_array_weights(int pair_state, double pesmin, double T0, const double *Ts, int n_sat,
                       double E, double *w) {
    for (int s = 0; s < n_sat; ++s) {
        double T = Ts[s], WTT = 1.0;
        if (pair_state == HHO_PS_BOUND && T < T0) WTT = exp(-pesmin * HkT / T0 / T * (T0 - T));
        double weight = exp(-E * HkT / T0 / T * (T0 - T)) / WTT;
        if (pair_state == HHO_PS_FREE_AND_METASTABLE && T > T0) weight = 0.0;
        w[s] = weight;
    }
}

int hho_correlation_sum_array(const hho_system *sys, const hho_params *p, const double *qp0, size_t n,
                              int nthreads, const double *w, int n_sat, double *out) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    size_t N = p->N;
    pthread_t th[256];
    corr_job jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = (corr_job){sys, p, qp0, n * t / nthreads, n * (t + 1) / nthreads,
                             calloc(N * n_sat, sizeof(double)), NULL, w, n_sat};
        pthread_create(&th[t], NULL, corr_worker, &jobs[t]);
    }
    memset(out, 0, N * n_sat * sizeof(double));
    for (int t = 0; t < nthreads; ++t) {
        pthread_join(th[t], NULL);
        for (size_t k = 0; k < N * n_sat; ++k) out[k] += jobs[t].sum[k];
        free(jobs[t].sum);
    }
    return 0;
}
