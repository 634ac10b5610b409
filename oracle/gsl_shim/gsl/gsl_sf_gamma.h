/* Project-written stand-in declarations (TEST INFRASTRUCTURE ONLY): lets the
   reference's own C sources compile into oracle/_ref without GSL.  The
   definitions live in oracle/gsl_shim/gsl_shim.c (tgamma and oracle/incgamma.c). */
#ifndef ORACLE_SHIM_GSL_SF_GAMMA_H
#define ORACLE_SHIM_GSL_SF_GAMMA_H
double gsl_sf_gamma(double x);
double gsl_sf_gamma_inc_P(double a, double x);
double gsl_sf_gamma_inc(double a, double x);
double gsl_sf_gamma_inc_Q(double a, double x);
#endif
