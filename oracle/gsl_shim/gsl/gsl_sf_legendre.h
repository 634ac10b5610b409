/* Project-written stand-in declarations (TEST INFRASTRUCTURE ONLY): the
   Legendre arrays the reference's SCF potential calls, with the GSL 2
   array layout (P_l^m at l (l + 1) / 2 + m), defined in
   oracle/gsl_shim/gsl_shim.c by the upward recurrences in l. */
#ifndef ORACLE_SHIM_GSL_SF_LEGENDRE_H
#define ORACLE_SHIM_GSL_SF_LEGENDRE_H
#include <stddef.h>
#ifndef GSL_MAJOR_VERSION
#define GSL_MAJOR_VERSION 2
#endif
typedef enum { GSL_SF_LEGENDRE_SCHMIDT, GSL_SF_LEGENDRE_SPHARM, GSL_SF_LEGENDRE_FULL,
               GSL_SF_LEGENDRE_NONE } gsl_sf_legendre_t;
int gsl_sf_legendre_Pl_array(int lmax, double x, double *result_array);
int gsl_sf_legendre_Pl_deriv_array(int lmax, double x, double *result_array,
                                   double *result_deriv_array);
int gsl_sf_legendre_array_e(gsl_sf_legendre_t norm, size_t lmax, double x, double csphase,
                            double result_array[]);
int gsl_sf_legendre_deriv_array_e(gsl_sf_legendre_t norm, size_t lmax, double x, double csphase,
                                  double result_array[], double result_deriv_array[]);
#endif
