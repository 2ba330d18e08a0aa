/* Stand-in for GSL's <gsl/gsl_sf_bessel.h>: the one declaration the
 * reference's Matern kernels use (GSL's published signature).  The
 * definition is in oracle/ref_shim/ref_shim.c. */
#ifndef ORACLE_REF_GSL_SF_BESSEL_H
#define ORACLE_REF_GSL_SF_BESSEL_H
double gsl_sf_bessel_Knu(const double nu, const double x);
#endif
