/* oracle/gsl_shim/gsl/gsl_sf_expint.h -- TEST INFRASTRUCTURE ONLY.
   Stand-in declaration for building the reference's C sources without GSL
   (definition in gsl_shim.c, computed by oracle/incgamma.c). */
#ifndef ORACLE_GSL_SF_EXPINT_H
#define ORACLE_GSL_SF_EXPINT_H
double gsl_sf_expint_E1(double x);
#endif
