// galpy_b200/csrc/compile_potential.h
//
// Host-side "potential compiler": turns galpy's flat (pot_type, pot_args)
// stream (as built by galpy/orbit/integrateFullOrbit.py:43-614 and
// integratePlanarOrbit.py:33-663, decoded in C by
// integrateFullOrbit.c:69-1040 / integratePlanarOrbit.c:55-742) into the
// device records of potentials.cuh, with every per-component constant
// precomputed once per call instead of once per force evaluation.
#pragma once
#include <math.h>
#include <stddef.h>
#include <string.h>

#include <vector>

#include "potentials.cuh"

namespace gpc {

// number of galpy arguments of a supported type (3D PowerSphericalwCutoff
// carries two extra cache slots, integrateFullOrbit.py:178-180); an
// ellipsoidal component's count depends on its own arguments
// (integrateFullOrbit.c case 21: 30 + npsi + 2 glorder), read from p
// (-1 without them)
inline int galpy_nargs(int type, int planar, const double* p = nullptr)
{
  if (type == T_SCF) {  // (a, isNonAxi, N, L, M, Nt, coefficients, 11 cache slots)
    if (!p) return -1;
    const int nonaxi = (int)p[1], N = (int)p[2], L = (int)p[3], M = (int)p[4];
    if ((int)p[5] != 0 || N < 1 || L < 1 || M < 1) return -1;  // time-dependent coefficients
    if (nonaxi && M != L) return -1;
    return 6 + (1 + nonaxi) * N * L * M + 11;
  }
  if (is_ellipsoidal(type)) {
    if (!p) return -1;
    const int npsi = (int)p[16];
    if (npsi < 0 || npsi > 16) return -1;
    const int order = (int)p[29 + npsi];
    return order < 1 ? -1 : 30 + npsi + 2 * order;
  }
  switch (type) {
    case T_LOGHALO: return 4;
    case T_MN: return 3;
    case T_HERNQUIST: return 2;
    case T_NFW: return 2;
    case T_PSWC: return planar ? 3 : 5;
    case T_POWER: case T_JAFFE: case T_ISOCHRONE: case T_PLUMMER: case T_PSEUDOISO:
    case T_BURKERT: case T_DEHNENCORE: return 2;
    case T_DEHNEN: case T_HOMSPHERE: case T_EINASTO: case T_EXPTRUNCNFW: return 3;
    case T_NULL: return 0;
    case T_FLATPOWER: return planar ? 3 : 4;
    case T_KKS: return 3;
    case T_HENONHEILES: return planar ? 1 : -1;  // (amp); a planarPotential only
    case T_KUZMINDISK: return 2;
    case T_DEHNENBAR: return 6;
    case T_NEEDLEBAR: return 13;  // (amp, a, b, c^2, pa, omegab, 7 cache slots)
    case T_SPIRALARMS:  // (nCs, amp, N, sin alpha, tan alpha, r_ref, phi_ref, Rs, H, omega, Cs)
      return p && (int)p[0] >= 1 && (int)p[0] <= kSpiralMaxTerms ? 10 + (int)p[0] : -1;
    case T_TRANSPIRAL: case T_STEADYSPIRAL: return planar ? 8 : -1;  // planarPotentials only
    case T_ELLDISK: return planar ? 6 : -1;
    case T_LOPSIDED: return planar ? 4 : -1;
    case T_COSMPHI: return planar ? 9 : -1;
    default: return -1;
  }
}

// gamma*(a, u) = P(a, u) / u^a = e^-u sum_n u^n / Gamma(a+n+1) in extended
// precision (all terms positive: no cancellation).
inline long double gamma_star_ld(long double a, long double u)
{
  long double term = 1.0L / tgammal(a + 1.0L), sum = term;
  for (int n = 1; n < 2000; n++) {
    term *= u / (a + n);
    sum += term;
    if (term < 1e-22L * sum) break;
  }
  return sum * expl(-u);
}

// Smallest integer U with Q(a, U) ~ U^(a-1) e^-U / Gamma(a) below 1e-18, so
// that P(a, u) = 1 in double precision for u >= U.
inline double gamma_star_cutoff(double a)
{
  long double U = 20.0L;
  while (expl(-U) * powl(U, (long double)a - 1.0L) / tgammal((long double)a) > 1e-18L) U += 1.0L;
  return (double)U;
}

// Chebyshev interpolation of gamma*(a, u) on kChebN equal intervals of
// [0, U], kChebC nodes each (values at the Chebyshev points, coefficients
// by the discrete cosine sums), converted to the power basis of the
// interval's local variable x in [-1, 1] (T_j expanded by its three-term
// recurrence), all in long double.
inline void build_gamma_star_table(double a, double U, double (*cheb)[kChebC])
{
  const long double w = (long double)U / kChebN;
  const long double pi = 3.141592653589793238462643383279502884L;
  // power-basis coefficients of T_0 .. T_{kChebC-1}
  long double T[kChebC][kChebC] = {};
  T[0][0] = 1.0L;
  if (kChebC > 1) T[1][1] = 1.0L;
  for (int j = 2; j < kChebC; j++)
    for (int m = 0; m < kChebC; m++)
      T[j][m] = (m > 0 ? 2.0L * T[j - 1][m - 1] : 0.0L) - T[j - 2][m];
  long double f[kChebC], cj[kChebC];
  for (int k = 0; k < kChebN; k++) {
    for (int i = 0; i < kChebC; i++) {
      const long double x = cosl(pi * (i + 0.5L) / kChebC);
      f[i] = gamma_star_ld((long double)a, w * (k + 0.5L * (x + 1.0L)));
    }
    for (int j = 0; j < kChebC; j++) {
      long double s = 0.0L;
      for (int i = 0; i < kChebC; i++) s += f[i] * cosl(pi * j * (i + 0.5L) / kChebC);
      s *= 2.0L / kChebC;
      if (j == 0) s *= 0.5L;
      cj[j] = s;
    }
    for (int m = 0; m < kChebC; m++) {
      long double s = 0.0L;
      for (int j = 0; j < kChebC; j++) s += cj[j] * T[j][m];
      cheb[k][m] = (double)s;
    }
  }
}

// Degree-11 Chebyshev interpolants of f(m) on the eighths [1 + j/8,
// 1 + (j+1)/8] of a binade, converted to the power basis of the local
// variable t = 16 m - (17 + 2 j) in [-1, 1] (the binade tables of
// potentials.cuh), in long double.
template <class F>
inline void build_binade_table(F f, double (*out)[kChebC])
{
  const long double pi = 3.141592653589793238462643383279502884L;
  long double T[kChebC][kChebC] = {};
  T[0][0] = 1.0L;
  T[1][1] = 1.0L;
  for (int j = 2; j < kChebC; j++)
    for (int m = 0; m < kChebC; m++)
      T[j][m] = (m > 0 ? 2.0L * T[j - 1][m - 1] : 0.0L) - T[j - 2][m];
  for (int k = 0; k < kBinSub; k++) {
    long double fv[kChebC], cj[kChebC];
    for (int i = 0; i < kChebC; i++) {
      const long double t = cosl(pi * (i + 0.5L) / kChebC);
      fv[i] = f((17.0L + 2.0L * k + t) / 16.0L);
    }
    for (int j = 0; j < kChebC; j++) {
      long double s = 0.0L;
      for (int i = 0; i < kChebC; i++) s += fv[i] * cosl(pi * j * (i + 0.5L) / kChebC);
      s *= 2.0L / kChebC;
      if (j == 0) s *= 0.5L;
      cj[j] = s;
    }
    for (int m = 0; m < kChebC; m++) {
      long double s = 0.0L;
      for (int j = 0; j < kChebC; j++) s += cj[j] * T[j][m];
      out[k][m] = (double)s;
    }
  }
}

// 2^(p e) for the binade exponent e + 1024 = 64 hi + lo (PSwC power tables);
// values beyond the double range (binades far outside any orbit) are
// clamped to finite numbers.
inline void build_power_exponent_tables(long double p, double* e2hi, double* e2lo)
{
  auto fin = [](long double v) {
    const long double big = 1.0e300L, tiny = 1.0e-300L;
    return (double)(v > big ? big : (v < tiny ? tiny : v));
  };
  for (int hi = 0; hi < 32; hi++) e2hi[hi] = fin(exp2l(p * 64.0L * (hi - 16)));
  for (int lo = 0; lo < 64; lo++) e2lo[lo] = fin(exp2l(p * lo));
}

// Point every record at the first earlier record of the same type whose
// tables are identical (GpComp::tab), so that parameter groups share one
// copy of each table.
inline void share_tables(GpComp* c, int n)
{
  const size_t off = offsetof(GpComp, cheb);
  const size_t len = sizeof(GpComp) - off;
  for (int i = 0; i < n; i++) {
    c[i].tab = 0;
    if (c[i].type != T_PSWC && c[i].type != T_NFW) continue;
    for (int j = 0; j < i; j++) {
      if (c[j].type == c[i].type && c[j].tab == 0 &&
          memcmp(reinterpret_cast<const char*>(&c[j]) + off,
                 reinterpret_cast<const char*>(&c[i]) + off, len) == 0) {
        c[i].tab = j - i;
        break;
      }
    }
  }
}

// Payload doubles of an SCF component (coefficients with m <= l of the
// summed orders, then the Gegenbauer recurrence table), from galpy's args.
inline int scf_payload_len(const double* p)
{
  const int nonaxi = (int)p[1], N = (int)p[2], L = (int)p[3];
  const int Me = nonaxi ? L : 1;
  int pairs = 0;
  for (int m = 0; m < Me; m++) pairs += L - m;
  return pairs * N * (1 + nonaxi) + kScfTable * L * (N - 1);
}

// Records one component takes: 1, plus continuation records for an SCF
// expansion's payload.
inline int comp_records(int type, const double* p)
{
  if (type != T_SCF) return 1;
  const int len = scf_payload_len(p);
  return 1 + (len + kPayloadDoubles - 1) / kPayloadDoubles;
}

// Arguments of a wrapper after its wrapped entries.
inline int wrapper_nargs(int type)
{
  return type == T_WRAP_SMOOTH ? 4 : type == T_WRAP_COROT ? 5 : 3;
}

// Records of n entries of galpy's (type, args) streams, advancing both; a
// wrapper (one level deep) is its record plus its wrapped entries' records.
// -3 (unsupported type, nested wrapper) or -1 (bad args).
inline int count_entries(int planar, int n, const int*& tp, const double*& p, int depth)
{
  int rec = 0;
  for (int k = 0; k < n; k++) {
    const int type = *tp++;
    if (is_wrapper(type)) {
      if (depth > 0) return -3;
      const int nw = (int)*p++;
      if (nw < 1 || nw > kMaxComp) return -1;
      const int inner = count_entries(planar, nw, tp, p, depth + 1);
      if (inner < 0) return inner;
      rec += 1 + inner;
      p += wrapper_nargs(type);
      continue;
    }
    const int na = galpy_nargs(type, planar, p);
    if (na < 0) return -3;
    rec += comp_records(type, p);
    p += na;
  }
  return rec;
}

// Records of one group (the stride of a parameter group in the device
// array, the launch's ncomp); -3 (unsupported type) or -1 (bad args).
inline int group_records(int planar, int npot, const int* pot_type, const double* pot_args)
{
  if (npot < 1 || npot > kMaxComp) return -1;
  const int* tp = pot_type;
  const double* p = pot_args;
  return count_entries(planar, npot, tp, p, 0);
}

// Compile n entries of galpy's streams into out from record `rec` on
// (advancing the streams and rec).
inline int compile_entries(int planar, int n, const int*& tp, const double*& p, GpComp* out,
                           int& rec, int depth)
{
  for (int k = 0; k < n; k++) {
    const int type = *tp++;
    if (is_wrapper(type)) {
      // the wrapper's record, then its wrapped entries' records; galpy's
      // stream: (nwrapped, wrapped args, the wrapper's own args)
      if (depth > 0) return -3;  // nested wrappers are not carried
      const int nw = (int)*p++;
      if (nw < 1 || nw > kMaxComp) return -1;
      const int w = rec++;
      const int rc = compile_entries(planar, nw, tp, p, out, rec, depth + 1);
      if (rc) return rc;
      GpComp& c = out[w];
      memset(&c, 0, sizeof(c));
      c.type = type;
      c.c[0] = p[0];
      c.c[1] = p[1];
      c.c[2] = p[2];
      if (type == T_WRAP_COROT) {  // (amp, vpo, beta, pa, to)
        c.c[3] = p[3];
        c.c[4] = p[4];
      }
      if (type == T_WRAP_SMOOTH) {  // (amp, tform, tsteady, grow)
        if (p[2] < p[1]) return -1;
        c.c[3] = p[3];
        c.c[4] = p[2] > p[1] ? 1.0 / (p[2] - p[1]) : 0.0;
      } else if (type == T_WRAP_GAUSS && !(p[2] > 0.0)) {  // (amp, to, sigma^2)
        return -1;
      } else if (type == T_WRAP_KUZMIN && !(p[1] >= 0.0 && p[2] >= 0.0)) {  // (amp, a, b^2)
        return -1;
      }
      c.c[15] = rec - w - 1;
      p += wrapper_nargs(type);
      continue;
    }
    const int na = galpy_nargs(type, planar, p);
    if (na < 0) return -3;
    const int nrec = comp_records(type, p);
    GpComp c;
    memset(&c, 0, sizeof(c));
    c.type = type;
    const double amp = na > 0 ? p[0] : 0.0;
    c.c[0] = amp;
    switch (type) {
      case T_PSWC: {
        const double alpha = p[1], rc = p[2];
        const double a = 1.5 - 0.5 * alpha;
        if (!(a > 0.0) || !(rc > 0.0)) return -1;
        const double mnorm = 2.0 * M_PI * pow(rc, 3.0 - alpha) * (double)tgammal((long double)a);
        c.c[1] = 1.0 / (rc * rc);
        c.c[2] = mnorm * pow(rc, -2.0 * a);
        c.c[3] = -0.5 * alpha;
        c.c[4] = mnorm;
        const double U = gamma_star_cutoff(a);
        c.c[5] = U;
        c.c[6] = kChebN / U;
        c.c[7] = 4.0 * M_PI;
        build_gamma_star_table(a, U, c.cheb);
        {  // (r^2)^(-alpha/2) = m^(-alpha/2) 2^(-alpha/2 e)
          const long double pw = -0.5L * (long double)alpha;
          build_binade_table([pw](long double m) { return powl(m, pw); }, c.bin);
          build_power_exponent_tables(pw, c.e2hi, c.e2lo);
        }
        // potential energy: gamma(1 - alpha/2, u) and gamma(1.5 - alpha/2, u)
        c.c[8] = 2.0 * M_PI * pow(rc, 3.0 - alpha);
        c.c[9] = rc;
        c.c[10] = 1.0 - 0.5 * alpha;
        c.c[11] = c.c[10] > 0.0 ? tgamma(c.c[10]) : NAN;  // alpha >= 2: energy undefined here
        c.c[12] = c.c[10] > 0.0 ? lgamma(c.c[10]) : NAN;
        c.c[13] = a;
        c.c[14] = tgamma(a);
        c.c[15] = lgamma(a);
        break;
      }
      case T_MN:
        c.c[1] = p[1];
        c.c[2] = p[2] * p[2];
        break;
      case T_HERNQUIST:
      case T_NFW:
        if (!(p[1] > 0.0)) return -1;
        c.c[1] = p[1];
        c.c[2] = 1.0 / p[1];
        if (type == T_NFW)  // log(m) / (m - 1); the nodes never fall on m = 1
          build_binade_table([](long double m) { return logl(m) / (m - 1.0L); }, c.bin);
        break;
      case T_LOGHALO: {
        const double q = p[1], core2 = p[2], om = p[3];
        if (!(q > 0.0)) return -1;
        c.c[1] = 1.0 / (q * q);
        c.c[2] = core2;
        // galpy passes 1 - 1/b^2 for a triaxial halo and 2.0 (> 1) when
        // axisymmetric (integrateFullOrbit.py:69-73)
        c.c[3] = om < 1.0 ? 1.0 - om : 1.0;
        break;
      }
      case T_POWER:
        c.c[1] = -0.5 * p[1];
        c.c[2] = 1.0 - p[1];
        c.c[3] = p[1];
        break;
      case T_JAFFE:
      case T_DEHNENCORE:
        if (!(p[1] > 0.0)) return -1;
        c.c[1] = p[1];
        break;
      case T_ISOCHRONE:
        if (!(p[1] > 0.0)) return -1;
        c.c[1] = p[1];
        c.c[2] = p[1] * p[1];
        break;
      case T_PLUMMER:
        c.c[1] = p[1] * p[1];
        break;
      case T_PSEUDOISO:
        if (!(p[1] > 0.0)) return -1;
        c.c[1] = p[1];
        c.c[2] = 1.0 / p[1];
        break;
      case T_BURKERT:
        if (!(p[1] > 0.0)) return -1;
        c.c[1] = p[1];
        c.c[2] = 1.0 / p[1];
        c.c[3] = M_PI * p[1] * p[1] * p[1];
        break;
      case T_DEHNEN:
        if (!(p[1] > 0.0) || !(p[2] < 3.0)) return -1;
        c.c[1] = p[1];
        c.c[2] = p[2];
        c.c[3] = 1.0 / (3.0 - p[2]);
        break;
      case T_HOMSPHERE:  // galpy passes R^2 and R^3
        c.c[1] = p[1];
        c.c[2] = p[2];
        break;
      case T_NULL:
        break;
      case T_EXPTRUNCNFW: {  // (amp, a, rc); the reference's series coefficients
        const double a = p[1], rc = p[2];
        if (!(a > 0.0) || !(rc > 0.0)) return -1;
        const double alpha = a / rc, ea = exp(alpha) * (1.0 + alpha);
        c.c[1] = a;
        c.c[2] = 1.0 / rc;
        c.c[3] = ea;
        c.c[4] = ea * expint_E1(alpha);
        c.c[5] = 1e-3 * (a < rc ? a : rc);
        c.c[6] = 0.5;
        c.c[7] = -(1.0 / rc + 2.0 / a) / 3.0;
        c.c[8] = (0.5 / (rc * rc) + 2.0 / (rc * a) + 3.0 / (a * a)) / 4.0;
        c.c[9] = -(1.0 / (6.0 * rc * rc * rc) + 1.0 / (rc * rc * a) + 3.0 / (rc * a * a) +
                   4.0 / (a * a * a)) / 5.0;
        c.c[10] = exp(alpha) / rc;
        break;
      }
      case T_EINASTO: {  // (amp, h, n)
        const double h = p[1], n = p[2];
        if (!(h > 0.0) || !(n > 0.0)) return -1;
        c.c[1] = h;
        c.c[2] = 1.0 / n;
        c.c[3] = 3.0 * n;
        c.c[4] = lgamma(3.0 * n);
        c.c[5] = 4.0 * M_PI * n * h * h * h * tgamma(3.0 * n);
        c.c[6] = 4.0 * M_PI * n * tgamma(3.0 * n);
        c.c[7] = 2.0 * n;
        c.c[8] = lgamma(2.0 * n);
        c.c[9] = 4.0 * M_PI * h * h * n * tgamma(2.0 * n);
        break;
      }
      case T_KKS: {  // (amp, ac, Delta)
        const double ac = p[1], Delta = p[2];
        if (!(Delta > 0.0) || ac == 1.0) return -1;
        const double gamma = Delta * Delta / (1.0 - ac * ac), alpha = gamma - Delta * Delta;
        c.c[1] = Delta * Delta;
        c.c[2] = alpha + gamma;
        break;
      }
      case T_TRIHERNQUIST: case T_TRINFW: case T_TRIJAFFE: case T_PERFECTELL: case T_TRIGAUSS:
      case T_POWERTRI: case T_TWOPOWERTRI: {
        // (amp, 15 cache slots, npsi, psi args, b^2, c^2, aligned, rot[9],
        // n, x_k[n], w_k[n]), integrateFullOrbit.py:214-290; x_k are the
        // Gauss-Legendre nodes of the integral over tau = 1/x^2 - 1
        const int npsi = (int)p[16];
        const double* ps = p + 17;
        const double* e = ps + npsi;
        const double b2 = e[0], c2 = e[1];
        const int order = (int)e[12];
        if (order > kEllMaxOrder) return -3;  // more nodes than the record holds
        switch (type) {
          case T_TWOPOWERTRI:  // (a, alpha, beta, beta - alpha, ...)
            c.c[1] = ps[0];
            c.c[2] = ps[1];
            c.c[3] = ps[2];
            c.c[4] = ps[3];
            break;
          case T_PERFECTELL: case T_TRIGAUSS: case T_POWERTRI:  // one parameter
            c.c[1] = ps[0];
            break;
          default:  // (a, a^k)
            c.c[1] = ps[0];
            c.c[2] = ps[1];
            break;
        }
        c.c[5] = order;
        c.c[6] = e[2] != 0.0 ? 0.0 : 1.0;  // galpy passes "aligned"
        for (int j = 0; j < 9; j++) c.bin[0][j] = e[3 + j];
        double* nd = &c.cheb[0][0];
        for (int k = 0; k < order; k++) {
          const long double xk = e[13 + k], tau = 1.0L / (xk * xk) - 1.0L;
          nd[4 * k] = e[13 + order + k];
          nd[4 * k + 1] = (double)(1.0L / (1.0L + tau));
          nd[4 * k + 2] = (double)(1.0L / ((long double)b2 + tau));
          nd[4 * k + 3] = (double)(1.0L / ((long double)c2 + tau));
        }
        break;
      }
      case T_KUZMINDISK:  // (amp, a)
        c.c[1] = p[1];
        break;
      case T_TRANSPIRAL: case T_STEADYSPIRAL: case T_ELLDISK: case T_LOPSIDED:
      case T_COSMPHI: {  // galpy's args as they are; the growth factor's 1 / (tsteady - tform)
        for (int j = 1; j < na; j++) c.c[j] = p[j];
        if ((type == T_STEADYSPIRAL || type == T_ELLDISK) && p[1] == p[1])
          c.c[9] = p[2] > p[1] ? 1.0 / (p[2] - p[1]) : 0.0;
        if (type == T_COSMPHI && (int)p[4] == 0) return -1;
        break;
      }
      case T_SPIRALARMS: {
        for (int j = 0; j < 9; j++) c.c[j] = p[1 + j];
        c.c[9] = p[0];
        for (int n = 0; n < (int)p[0]; n++) c.c[10 + n] = p[10 + n];
        if (!(p[3] != 0.0) || !(p[4] != 0.0) || !(p[7] > 0.0)) return -1;
        break;
      }
      case T_NEEDLEBAR: {  // (amp, a, b, c^2, pa, omegab, cache)
        if (!(p[1] > 0.0) || !(p[3] >= 0.0) || !(p[2] >= 0.0)) return -1;
        for (int j = 0; j < 6; j++) c.c[j] = p[j];
        c.c[6] = 0.5 / p[1];
        break;
      }
      case T_DEHNENBAR: {  // (amp * af, tform, tsteady, rb, omegab, barphi)
        if (!(p[3] > 0.0) || p[2] < p[1]) return -1;
        for (int j = 1; j < 6; j++) c.c[j] = p[j];
        c.c[6] = p[3] * p[3] * p[3];
        c.c[7] = p[2] > p[1] ? 1.0 / (p[2] - p[1]) : 0.0;
        break;
      }
      case T_SCF: {  // (a, isNonAxi, N, L, M, 0, Acos[N][L][M], Asin, cache)
        const int nonaxi = (int)p[1], N = (int)p[2], L = (int)p[3], M = (int)p[4];
        const int Me = nonaxi ? L : 1;
        if (!(p[0] > 0.0)) return -1;
        c.c[0] = p[0];
        c.c[1] = nonaxi;
        c.c[2] = N;
        c.c[3] = L;
        c.c[4] = Me;
        std::vector<double> pay;
        pay.reserve(scf_payload_len(p));
        const double s4 = sqrt(4.0 * M_PI);
        const double* Ac = p + 6;
        const double* As = p + 6 + N * L * M;
        for (int m = 0; m < Me; m++)
          for (int l = m; l < L; l++)
            for (int n = 0; n < N; n++) {
              const int ci = (n * L + l) * M + m;
              pay.push_back(s4 * Ac[ci]);
              if (nonaxi) pay.push_back(s4 * As[ci]);
            }
        c.c[5] = (double)pay.size();  // the recurrence table's offset
        for (int l = 0; l < L; l++) {
          const long double al = 2.0L * l + 1.5L;
          for (int n = 0; n + 1 < N; n++) {
            const long double n1 = n + 1.0L;
            pay.push_back((double)(2.0L * (n + al) / n1));
            pay.push_back((double)((n + 2.0L * al - 1.0L) / n1));
            pay.push_back((double)(2.0L * (n + al + 1.0L) / n1));
            pay.push_back((double)((n + 2.0L * al + 1.0L) / n1));
            pay.push_back((double)(2.0L * (n + al + 2.0L) / n1));
            pay.push_back((double)((n + 2.0L * al + 3.0L) / n1));
          }
        }
        for (int r = 1; r < nrec; r++) {  // continuation records
          GpComp& q = out[rec + r];
          memset(&q, 0, sizeof(q));
          q.type = T_PAYLOAD;
          double* d = &q.c[0];
          for (int j = 0; j < kPayloadDoubles; j++) {
            const size_t i = (size_t)(r - 1) * kPayloadDoubles + j;
            d[j] = i < pay.size() ? pay[i] : 0.0;
          }
        }
        break;
      }
      case T_FLATPOWER: {  // (amp, alpha, q^2, core^2); planar (amp, alpha, core^2)
        const double alpha = p[1], q2 = planar ? 1.0 : p[2], core2 = planar ? p[2] : p[3];
        if (!(q2 > 0.0)) return -1;
        c.c[1] = 1.0 / q2;
        c.c[2] = core2;
        c.c[3] = -0.5 * alpha - 1.0;
        c.c[4] = alpha;
        c.c[5] = alpha + 2.0;
        break;
      }
    }
    for (int i = 0; i < kChebN; i++)
      for (int j = 0; j < kChebC; j++) c.chebf[i][j] = (float)c.cheb[i][j];
    for (int i = 0; i < kBinSub; i++)
      for (int j = 0; j < kChebC; j++) c.binf[i][j] = (float)c.bin[i][j];
    out[rec] = c;
    rec += nrec;
    p += na;
  }
  return 0;
}

// Compile one group (npot top-level entries of galpy's streams) into its
// group_records(...) records.  Returns 0, -3 (unsupported type) or -1 (bad
// args).  *consumed receives the number of pot_args read.
inline int compile_group(int planar, int npot, const int* pot_type, const double* pot_args,
                         GpComp* out, int* consumed)
{
  if (npot < 1 || npot > kMaxComp) return -1;
  const int* tp = pot_type;
  const double* p = pot_args;
  int rec = 0;
  const int rc = compile_entries(planar, npot, tp, p, out, rec, 0);
  if (rc) return rc;
  if (consumed) *consumed = (int)(p - pot_args);
  return 0;
}

}  // namespace gpc
