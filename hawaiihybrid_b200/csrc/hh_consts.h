// Physical constants of the reference (src/constants.h:8-53, CODATA 2022) and
// status codes shared by the CUDA library and its host-side mirror.
#pragma once

#define HH_ALU 5.29177210903e-11
#define HH_BOLTZMANN 1.380649e-23
#define HH_HARTREE 4.3597447222071e-18
#define HH_HTOCM 2.1947463136320e5
#define HH_ATU 2.4188843265857e-17
#define HH_LIGHTSPEED_CM 2.99792458e10
#define HH_ADIPMOMU 8.4783536255e-30
#define HH_EPSILON0 8.8541878128e-12
#define HH_HKT (HH_HARTREE / HH_BOLTZMANN)
#define HH_PI 3.14159265358979323846
#define HH_LOG2E 1.44269504088896340736  /* log2(e) */
#define HH_ZEROCOEFF (0.00361479637 / (4.0 * HH_PI))
#define HH_SECONDCOEFF 13856114.29344114  // src/constants.h:30

// per-half-trajectory status codes (the reference's failure modes,
// src/hawaii.c:2172-2243)
#define HH_ST_OK 0
#define HH_ST_MAXSTEPS 1     // more than max_steps internal steps between two samples
#define HH_ST_H_UNDERFLOW 2  // step size below 10 ulp(t)
#define HH_ST_NAN_DIPOLE 3   // NaN dipole: the reference returns 1, trajectory contributes 0
#define HH_ST_OVERFLOW 4     // |mu0.mu(t)| > 1e100: same
#define HH_ST_JUMP 5         // |C_k/C_{k-1}| > 1e10: same
#define HH_ST_COUNT 6
