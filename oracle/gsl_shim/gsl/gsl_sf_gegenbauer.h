/* Project-written stand-in declaration (TEST INFRASTRUCTURE ONLY): the
   Gegenbauer polynomial array the reference's SCF potential calls, defined
   in oracle/gsl_shim/gsl_shim.c by the three-term recurrence. */
#ifndef ORACLE_SHIM_GSL_SF_GEGENBAUER_H
#define ORACLE_SHIM_GSL_SF_GEGENBAUER_H
int gsl_sf_gegenpoly_array(int nmax, double lambda, double x, double *result_array);
#endif
