/* oracle/gsl_shim/gsl_shim.c -- TEST INFRASTRUCTURE ONLY.
   Definitions behind the stand-in GSL headers, linked only into oracle/_ref
   (the reference's own C sources built by oracle/Makefile).  The gamma
   functions and E1 are computed by oracle/incgamma.c (published series and
   continued fractions) and C99 tgamma; the spline entry points exist only to satisfy the
   linker and abort if reached. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_sf_expint.h"
#include "gsl/gsl_sf_gamma.h"
#include "gsl/gsl_spline.h"

double oracle_gamma_inc_P(double a, double x);
double oracle_gamma_inc_Q(double a, double x);
double oracle_expint_E1(double x);

double gsl_sf_gamma(double x) { return tgamma(x); }
double gsl_sf_gamma_inc_P(double a, double x) { return oracle_gamma_inc_P(a, x); }
double gsl_sf_gamma_inc(double a, double x) { return tgamma(a) * oracle_gamma_inc_Q(a, x); }
double gsl_sf_gamma_inc_Q(double a, double x) { return oracle_gamma_inc_Q(a, x); }
double gsl_sf_expint_E1(double x) { return oracle_expint_E1(x); }

static void shim_unreachable(const char *what)
{
  fprintf(stderr, "oracle/_ref: GSL stand-in %s called; not supported in this build\n", what);
  abort();
}
const gsl_interp_type *gsl_interp_cspline = NULL;
gsl_interp_accel *gsl_interp_accel_alloc(void) { shim_unreachable("gsl_interp_accel_alloc"); return NULL; }
void gsl_interp_accel_free(gsl_interp_accel *a) { (void)a; }
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t n) { (void)T; (void)n; shim_unreachable("gsl_spline_alloc"); return NULL; }
void gsl_spline_free(gsl_spline *s) { (void)s; }
int gsl_spline_init(gsl_spline *s, const double xa[], const double ya[], size_t n) { (void)s; (void)xa; (void)ya; (void)n; shim_unreachable("gsl_spline_init"); return 0; }
double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a) { (void)s; (void)x; (void)a; shim_unreachable("gsl_spline_eval"); return 0.; }
double gsl_spline_eval_deriv(const gsl_spline *s, double x, gsl_interp_accel *a) { (void)s; (void)x; (void)a; shim_unreachable("gsl_spline_eval_deriv"); return 0.; }
