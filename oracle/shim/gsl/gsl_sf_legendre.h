/* Minimal stand-in for the two GSL Legendre routines the reference CO2-Ar
 * plugins call, so that their sources compile into oracle/_ref without GSL.
 * Test infrastructure only. */
#ifndef HH_GSL_SHIM_LEGENDRE_H_
#define HH_GSL_SHIM_LEGENDRE_H_
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef enum {
    GSL_SF_LEGENDRE_SCHMIDT,
    GSL_SF_LEGENDRE_SPHARM,
    GSL_SF_LEGENDRE_FULL,
    GSL_SF_LEGENDRE_NONE
} gsl_sf_legendre_t;
int gsl_sf_legendre_Pl_array(const int lmax, const double x, double *result_array);
size_t gsl_sf_legendre_array_n(const size_t lmax);
int gsl_sf_legendre_array_e(const gsl_sf_legendre_t norm, const size_t lmax, const double x,
                            const double csphase, double result_array[]);
#ifdef __cplusplus
}
#endif
#endif
