/* Unnormalised Legendre functions with GSL's calling conventions
 * (result index l(l+1)/2 + m, Condon-Shortley phase supplied as csphase).
 * Test infrastructure only: lets the reference CO2-Ar plugin sources compile
 * into oracle/_ref. */
#include <math.h>
#include "shim/gsl/gsl_sf_legendre.h"

int gsl_sf_legendre_Pl_array(const int lmax, const double x, double *r) {
    r[0] = 1.0;
    if (lmax >= 1) r[1] = x;
    for (int l = 1; l < lmax; ++l) r[l + 1] = ((2 * l + 1) * x * r[l] - l * r[l - 1]) / (l + 1);
    return 0;
}

size_t gsl_sf_legendre_array_n(const size_t lmax) { return (lmax + 1) * (lmax + 2) / 2; }

int gsl_sf_legendre_array_e(const gsl_sf_legendre_t norm, const size_t lmax, const double x,
                            const double csphase, double r[]) {
    (void)norm; /* only GSL_SF_LEGENDRE_NONE is used by the reference */
    double s = sqrt((1.0 - x) * (1.0 + x));
    double pmm = 1.0;
    for (size_t m = 0; m <= lmax; ++m) {
        if (m > 0) pmm *= csphase * (2.0 * m - 1.0) * s;
        r[m * (m + 1) / 2 + m] = pmm;
        if (m + 1 <= lmax) {
            double p1 = x * (2.0 * m + 1.0) * pmm;
            r[(m + 1) * (m + 2) / 2 + m] = p1;
            double p0 = pmm;
            for (size_t l = m + 2; l <= lmax; ++l) {
                double pl = ((2.0 * l - 1.0) * x * p1 - (double)(l + m - 1) * p0) / (double)(l - m);
                r[l * (l + 1) / 2 + m] = pl;
                p0 = p1;
                p1 = pl;
            }
        }
    }
    return 0;
}
