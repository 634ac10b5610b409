/* oracle/gsl_shim/gsl_shim.c -- TEST INFRASTRUCTURE ONLY.
   Definitions behind the stand-in GSL headers, linked only into oracle/_ref
   (the reference's own C sources built by oracle/Makefile).  The gamma
   functions and E1 are computed by oracle/incgamma.c (published series and
   continued fractions) and C99 tgamma; the Gegenbauer and Legendre arrays
   by their three-term recurrences (DLMF 18.9.1, 14.10.3, 14.10.5), checked
   against scipy in the tests; the spline entry points exist only to satisfy
   the linker and abort if reached. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_sf_expint.h"
#include "gsl/gsl_sf_gamma.h"
#include "gsl/gsl_sf_gegenbauer.h"
#include "gsl/gsl_sf_legendre.h"
#include "gsl/gsl_spline.h"

double oracle_gamma_inc_P(double a, double x);
double oracle_gamma_inc_Q(double a, double x);
double oracle_expint_E1(double x);

double gsl_sf_gamma(double x) { return tgamma(x); }
double gsl_sf_gamma_inc_P(double a, double x) { return oracle_gamma_inc_P(a, x); }
double gsl_sf_gamma_inc(double a, double x) { return tgamma(a) * oracle_gamma_inc_Q(a, x); }
double gsl_sf_gamma_inc_Q(double a, double x) { return oracle_gamma_inc_Q(a, x); }
double gsl_sf_expint_E1(double x) { return oracle_expint_E1(x); }

/* C_n^lam(x), n = 0..nmax: (n+1) C_{n+1} = 2 (n + lam) x C_n - (n + 2 lam - 1) C_{n-1} */
int gsl_sf_gegenpoly_array(int nmax, double lambda, double x, double *C)
{
  C[0] = 1.;
  if (nmax >= 1) C[1] = 2. * lambda * x;
  for (int n = 1; n < nmax; n++)
    C[n + 1] = (2. * (n + lambda) * x * C[n] - (n + 2. * lambda - 1.) * C[n - 1]) / (n + 1.);
  return 0;
}

/* P_l^m(x) (unnormalised; Condon-Shortley phase when csphase = -1) for
   0 <= m <= l <= lmax at l (l + 1) / 2 + m, and dP/dx from (x^2 - 1)
   dP_l^m/dx = l x P_l^m - (l + m) P_{l-1}^m (the m = 0 end points x = +-1 from
   P_l'(+-1) = (+-1)^(l+1) l (l + 1) / 2) */
static void shim_legendre(int lmax, double x, double csphase, double *P, double *dP)
{
  double s = sqrt((1. - x) * (1. + x)), pmm = 1.;
  for (int m = 0; m <= lmax; m++) {
    if (m > 0) pmm *= csphase * (2. * m - 1.) * s;
    double pm2 = 0., pm1 = pmm;
    for (int l = m; l <= lmax; l++) {
      double p;
      if (l == m)
        p = pmm;
      else if (l == m + 1)
        p = x * (2. * m + 1.) * pmm;
      else
        p = ((2. * l - 1.) * x * pm1 - (l + m - 1.) * pm2) / (l - m);
      double prev = l == m ? 0. : pm1;
      int i = l * (l + 1) / 2 + m;
      P[i] = p;
      if (dP) {
        if (fabs(x) == 1. && m == 0)
          dP[i] = (x > 0. || l % 2 == 1 ? 1. : -1.) * 0.5 * l * (l + 1.);
        else
          dP[i] = (l * x * p - (l + m) * prev) / (x * x - 1.);
      }
      if (l > m) {
        pm2 = pm1;
        pm1 = p;
      }
    }
  }
}

int gsl_sf_legendre_array_e(gsl_sf_legendre_t norm, size_t lmax, double x, double csphase,
                            double result_array[])
{
  (void)norm;
  shim_legendre((int)lmax, x, csphase, result_array, NULL);
  return 0;
}

int gsl_sf_legendre_deriv_array_e(gsl_sf_legendre_t norm, size_t lmax, double x, double csphase,
                                  double result_array[], double result_deriv_array[])
{
  (void)norm;
  shim_legendre((int)lmax, x, csphase, result_array, result_deriv_array);
  return 0;
}

/* P_l(x), l = 0..lmax (m = 0 of the above, packed by l) */
int gsl_sf_legendre_Pl_deriv_array(int lmax, double x, double *P, double *dP)
{
  double pm2 = 0., pm1 = 1.;
  for (int l = 0; l <= lmax; l++) {
    double p = l == 0 ? 1. : (l == 1 ? x : ((2. * l - 1.) * x * pm1 - (l - 1.) * pm2) / l);
    double prev = l == 0 ? 0. : pm1;
    P[l] = p;
    if (dP) {
      if (fabs(x) == 1.)
        dP[l] = (x > 0. || l % 2 == 1 ? 1. : -1.) * 0.5 * l * (l + 1.);
      else
        dP[l] = (l * x * p - l * prev) / (x * x - 1.);
    }
    if (l > 0) pm2 = pm1;
    pm1 = p;
  }
  return 0;
}

int gsl_sf_legendre_Pl_array(int lmax, double x, double *P)
{
  return gsl_sf_legendre_Pl_deriv_array(lmax, x, P, NULL);
}

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
