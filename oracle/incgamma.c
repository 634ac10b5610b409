/*
 * oracle/incgamma.c -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * Regularised lower incomplete gamma function P(a,x) for a > 0, x >= 0, used
 * by the CPU oracle for the mass of PowerSphericalPotentialwCutoff.  The
 * reference calls GSL's gsl_sf_gamma_inc_P / gsl_sf_gamma_inc here
 * (galpy/potential/potential_c_ext/PowerSphericalPotentialwCutoff.c:10,23);
 * GSL is not part of the reference tree, so this file restates the published
 * method instead of GSL's code:
 *   - x < a+1 : power series  P = x^a e^-x / Gamma(a+1) * sum_n x^n / (a+1)_n
 *               (Abramowitz & Stegun 6.5.29)
 *   - x >= a+1: Legendre continued fraction for Q = 1-P
 *               (Abramowitz & Stegun 6.5.31), evaluated with the modified
 *               Lentz algorithm (Numerical Recipes, 2nd ed., sec. 5.2/6.2).
 * The same functions back the GSL stand-in used to build the reference's own
 * C sources (oracle/gsl_shim), so both CPU paths share one P(a,x).
 * Accuracy is checked against scipy.special.gammainc in tests/test_oracle.py.
 */
#include <math.h>
#include <float.h>

#define IG_EPS 1.0e-16
#define IG_TINY 1.0e-300
#define IG_MAXIT 100000

/* log of the common prefactor x^a e^-x / Gamma(a) */
static double ig_logpref(double a, double x) { return a * log(x) - x - lgamma(a); }

static double ig_series_P(double a, double x)
{
  double ap = a, term = 1.0 / a, sum = term;
  for (int n = 0; n < IG_MAXIT; n++) {
    ap += 1.0;
    term *= x / ap;
    sum += term;
    if (fabs(term) < fabs(sum) * IG_EPS) break;
  }
  return sum * exp(ig_logpref(a, x));
}

static double ig_cf_Q(double a, double x)
{
  double b = x + 1.0 - a, c = 1.0 / IG_TINY, d = 1.0 / b, h = d;
  for (int i = 1; i < IG_MAXIT; i++) {
    double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (fabs(d) < IG_TINY) d = IG_TINY;
    c = b + an / c;
    if (fabs(c) < IG_TINY) c = IG_TINY;
    d = 1.0 / d;
    double del = d * c;
    h *= del;
    if (fabs(del - 1.0) < IG_EPS) break;
  }
  return exp(ig_logpref(a, x)) * h;
}

double oracle_gamma_inc_P(double a, double x)
{
  if (!(a > 0.0) || x < 0.0) return NAN;
  if (x == 0.0) return 0.0;
  if (x < a + 1.0) return ig_series_P(a, x);
  return 1.0 - ig_cf_Q(a, x);
}

double oracle_gamma_inc_Q(double a, double x)
{
  if (!(a > 0.0) || x < 0.0) return NAN;
  if (x == 0.0) return 1.0;
  if (x < a + 1.0) return 1.0 - ig_series_P(a, x);
  return ig_cf_Q(a, x);
}

/* Exponential integral E1(x), x > 0, for ExpTruncNFWPotential (the reference
   calls GSL's gsl_sf_expint_E1, ExpTruncNFWPotential.c): the power series
   E1 = -gamma_E - ln x - sum_k (-x)^k / (k k!) for x <= 1 (Abramowitz &
   Stegun 5.1.11) and the continued fraction E1 = e^-x / (x + 1 - 1 / (x + 3
   - 4 / (x + 5 - ...))) for x > 1 (A&S 5.1.22), evaluated with the modified
   Lentz algorithm.  Checked against scipy.special.exp1 in tests. */
double oracle_expint_E1(double x)
{
  if (!(x > 0.0)) return x == 0.0 ? INFINITY : NAN;
  if (x <= 1.0) {
    const double euler_gamma = 0.57721566490153286061;
    double term = 1.0, sum = 0.0;
    for (int k = 1; k < IG_MAXIT; k++) {
      term *= -x / k;
      const double d = term / k;
      sum += d;
      if (fabs(d) < IG_EPS * fabs(sum)) break;
    }
    return -euler_gamma - log(x) - sum;
  }
  double b = x + 1.0, c = 1.0 / IG_TINY, d = 1.0 / b, h = d;
  for (int i = 1; i < IG_MAXIT; i++) {
    const double an = -(double)i * i;
    b += 2.0;
    d = 1.0 / (an * d + b);
    c = b + an / c;
    const double del = c * d;
    h *= del;
    if (fabs(del - 1.0) < IG_EPS) break;
  }
  return h * exp(-x);
}
