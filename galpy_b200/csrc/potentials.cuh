// galpy_b200/csrc/potentials.cuh
//
// Device-side forces and tidal tensors of the potentials the engine supports:
// PowerSphericalPotentialwCutoff (galpy type 15), MiyamotoNagaiPotential (5),
// NFWPotential (9), HernquistPotential (8), LogarithmicHaloPotential (0,
// axisymmetric or triaxial), and the spherical PowerSpherical (7), Jaffe
// (10), Isochrone (14), Plummer (17), PseudoIsothermal (18), Burkert (20),
// DehnenCoreSpherical (33), DehnenSpherical (34), HomogeneousSphere (35) and
// Null (40) and Einasto (41) potentials, and the axisymmetric FlattenedPower
// (12) and KuzminKutuzovStaeckel (16), the planar HenonHeiles (29), and
// KuzminDisk (19), the EllipsoidalPotential family: TriaxialHernquist (21),
// TriaxialNFW (22),
// TriaxialJaffe (23), PerfectEllipsoid (30), TriaxialGaussian (37),
// PowerTriaxial (38) and TwoPowerTriaxial (43).  Reference formulas:
// galpy/potential/potential_c_ext/<name>.c.
//
// Design (not a translation of the reference's cylindrical route):
//  * Every component is evaluated directly in Cartesian coordinates.  The
//    axisymmetric terms are written as a_i = x_i * g(R, z), so neither
//    R = sqrt(x^2+y^2), acos(x/R), nor the 1/R conversions of
//    evalRectForce (integrateFullOrbit.c:1307-1325) are needed.
//  * The host compiles galpy's (pot_type, pot_args) once into GpComp records
//    holding the derived constants (compile_potential.h).
//  * The bulge mass M(r) = 2 pi rc^(3-alpha) Gamma(a) P(a, r^2/rc^2),
//    a = 1.5 - alpha/2, is evaluated as
//        M(r) / r^3 = Mnorm rc^(-2a) (r^2)^(-alpha/2) gamma*(a, u),
//        gamma*(a, u) = P(a, u) / u^a = e^-u sum_n u^n / Gamma(a+n+1),
//    where gamma* -- an entire, slowly varying function -- comes from a
//    piecewise Chebyshev table built on the host in extended precision
//    (kChebN intervals on [0, U]; P = 1 to double precision beyond U).
//    This replaces the reference's GSL series / continued fraction
//    (PowerSphericalPotentialwCutoff.c:9-11), whose dependent divisions made
//    it the latency bottleneck of every force evaluation.
//  * A component list is walked at run time (any combination of the
//    supported types), or fixed at compile time (FixedPot) so that the components of
//    a known potential such as MWPotential2014 are inlined side by side and
//    their latencies overlap.
//  * The Cartesian tidal tensor K = -grad grad Phi (variational runs) is
//    built from each component's own radial / meridional derivatives and
//    equals the reference's cylindrical-to-Cartesian assembly
//    (integrateFullOrbit.c:1570-1596).
#pragma once
#include "gpc_common.cuh"

namespace gpc {

enum : int { T_LOGHALO = 0, T_MN = 5, T_HERNQUIST = 8, T_NFW = 9, T_PSWC = 15 };
// spherical potentials (potential_c_ext/<name>.c): PowerSpherical (galpy's
// KeplerPotential is alpha = 3), Jaffe, Isochrone, Plummer,
// PseudoIsothermal, Burkert, DehnenCoreSpherical, DehnenSpherical,
// HomogeneousSphere, Null (no force)
enum : int { T_POWER = 7, T_JAFFE = 10, T_ISOCHRONE = 14, T_PLUMMER = 17, T_PSEUDOISO = 18,
             T_BURKERT = 20, T_DEHNENCORE = 33, T_DEHNEN = 34, T_HOMSPHERE = 35, T_NULL = 40,
             T_EINASTO = 41, T_EXPTRUNCNFW = 46 };
// axisymmetric FlattenedPowerPotential (FlattenedPowerPotential.c) and
// KuzminKutuzovStaeckelPotential (KuzminKutuzovStaeckelPotential.c)
enum : int { T_FLATPOWER = 12, T_KKS = 16 };
// planar, non-axisymmetric HenonHeilesPotential (HenonHeilesPotential.c)
enum : int { T_HENONHEILES = 29 };
// KuzminDiskPotential (KuzminDiskPotential.c): Phi = -amp / sqrt(R^2 + (a + |z|)^2)
enum : int { T_KUZMINDISK = 19 };
// EllipsoidalPotential.c with the density functions m -> rho(m) of
// TwoPowerTriaxialPotential.c (TriaxialHernquist, TriaxialNFW,
// TriaxialJaffe, TwoPowerTriaxial), PerfectEllipsoidPotential.c,
// TriaxialGaussianPotential.c and PowerTriaxialPotential.c
enum : int { T_TRIHERNQUIST = 21, T_TRINFW = 22, T_TRIJAFFE = 23, T_PERFECTELL = 30,
             T_TRIGAUSS = 37, T_POWERTRI = 38, T_TWOPOWERTRI = 43 };
GPC_HD GPC_FI constexpr bool is_ellipsoidal(int t)
{
  return t == T_TRIHERNQUIST || t == T_TRINFW || t == T_TRIJAFFE || t == T_PERFECTELL ||
         t == T_TRIGAUSS || t == T_POWERTRI || t == T_TWOPOWERTRI;
}

constexpr int kMaxComp = 16;  // components per potential group
constexpr int kChebN = 32;    // Chebyshev intervals of gamma*(a, u) on [0, U]
constexpr int kChebC = 12;    // coefficients per interval (degree 11)
constexpr int kBinSub = 8;    // sub-intervals of a binade [1, 2) in the binade tables

// One compiled potential component.  c[] by type:
//   PSwC:      c0 amp, c1 1/rc^2, c2 Mnorm rc^(-2a), c3 -alpha/2,
//              c4 Mnorm (total-mass factor, P = 1), c5 U, c6 kChebN / U,
//              c7 4 pi
//   MN:        c0 amp, c1 a, c2 b^2
//   Hernquist: c0 amp, c1 a
//   NFW:       c0 amp, c1 a, c2 1/a
//   LogHalo:   c0 amp, c1 1/q^2, c2 core^2, c3 1 - e (y-axis factor; 1 when
//              axisymmetric)
//   PowerSpherical: c1 -alpha/2, c2 1 - alpha, c3 alpha
//   Jaffe, DehnenCore: c1 a      Isochrone: c1 b, c2 b^2      Plummer: c1 b^2
//   PseudoIsothermal: c1 a, c2 1/a       Burkert: c1 a, c2 1/a, c3 pi a^3
//   DehnenSpherical: c1 a, c2 alpha, c3 1/(3 - alpha)
//   HomogeneousSphere: c1 R^2, c2 R^3    Null: -
//   Einasto: c1 h, c2 1/n, c3 3n, c4 lgamma(3n), c5 4 pi n h^3 Gamma(3n),
//              c6 4 pi n Gamma(3n), c7 2n, c8 lgamma(2n), c9 4 pi h^2 n Gamma(2n)
//   ExpTruncNFW: c1 a, c2 1/rc, c3 e^alpha (1 + alpha), c4 c3 E1(alpha),
//              c5 small-r threshold 1e-3 min(a, rc), c6..c9 its series
//              coefficients, c10 e^alpha / rc (alpha = a / rc)
//   FlattenedPower: c1 1/q^2 (1 in the plane), c2 core^2, c3 -alpha/2 - 1,
//              c4 alpha, c5 alpha + 2
//   KuzminKutuzovStaeckel: c1 Delta^2, c2 alpha + gamma with
//              gamma = Delta^2 / (1 - ac^2), alpha = gamma - Delta^2
//   PSwC potential (energy evaluation only): c8 2 pi rc^(3-alpha), c9 rc,
//              c10 a1 = 1 - alpha/2, c11 Gamma(a1), c12 lgamma(a1),
//              c13 a2 = 1.5 - alpha/2, c14 Gamma(a2), c15 lgamma(a2)
//
// Binade tables (FP64 force path): a function of x > 0 is evaluated from
// x = m 2^e, m in [1, 2), as g(m) * h(e), with g from a degree-11 polynomial
// on each eighth of [1, 2) (power basis of the local variable t in [-1, 1])
// and h(e) from two small tables indexed by e + 1024 = 64 hi + lo.
//   PSwC: bin = m^(-alpha/2), e2hi[hi] = 2^(-alpha/2 * 64 (hi - 16)),
//         e2lo[lo] = 2^(-alpha/2 * lo)  -> (r^2)^(-alpha/2)
//   NFW:  bin = log(m) / (m - 1)         -> log1p(r/a)
//
// tab: offset, in records, of the record that holds this component's
// tables (0: its own).  Parameter groups whose tables are identical (the
// gamma* and power tables depend only on alpha, the NFW table on nothing)
// share one copy, which keeps a ragged launch's table working set in L1.
struct GpComp {
  int type;
  int tab;
  double c[16];
  double cheb[kChebN][kChebC];  // PSwC only: power-basis coefficients per interval
  double bin[kBinSub][kChebC];  // PSwC, NFW: binade polynomial
  double e2hi[32];              // PSwC only
  double e2lo[64];              // PSwC only
  float chebf[kChebN][kChebC];  // single-precision copies for the FP32 force path
  float binf[kBinSub][kChebC];
};

// --------------------------------------------- branch-free FP64 helpers ---
// The force of an orbit step is a dependent chain of special functions; the
// library versions of log, exp, log1p, division and rsqrt carry branches for
// special operands, which also keep the compiler from interleaving the
// components of a potential.  These replacements are straight-line code for
// the positive, normal operands of the force path (not for 0, inf, NaN or
// subnormals).
//
// 1/sqrt(x) and 1/x: the hardware's approximate double-precision result
// (PTX rsqrt.approx.f64 / rcp.approx.ftz.f64, about 2^-22 relative) as a
// seed and one third-order Newton correction, y <- y (1 + e/2 + 3e^2/8) with
// e = 1 - x y^2 (resp. y (1 + e + e^2), e = 1 - x y), the residual formed
// with a fused multiply-add: error O(e^3) ~ 1e-20, so the result is within a
// few ulp (tests/test_gpu_parity.py checks it against 1/sqrt and 1/x).
GPC_HD GPC_FI double rsqrt_nr(double x)
{
#if defined(__CUDA_ARCH__)
  double y;
  asm("rsqrt.approx.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
#else
  return 1.0 / sqrt(x);
#endif
}

GPC_HD GPC_FI double rcp_nr(double x)
{
#if defined(__CUDA_ARCH__)
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
#else
  return 1.0 / x;
#endif
}

GPC_HD GPC_FI long long bits_of(double x)
{
#if defined(__CUDA_ARCH__)
  return __double_as_longlong(x);
#else
  long long b;
  memcpy(&b, &x, sizeof(b));
  return b;
#endif
}

GPC_HD GPC_FI double double_of(long long b)
{
#if defined(__CUDA_ARCH__)
  return __longlong_as_double(b);
#else
  double x;
  memcpy(&x, &b, sizeof(x));
  return x;
#endif
}

// ---------------------------------------------------------------- math ---
template <typename T> struct Num;
template <> struct Num<double> {
  GPC_HD static double lg(double x) { return log(x); }
  GPC_HD static double ex(double x) { return exp(x); }
  GPC_HD static double rsq(double x) { return rsqrt_nr(x); }
  GPC_HD static double rcp(double x) { return rcp_nr(x); }
};
// FP32 evaluation: hardware approximations (SFU) for log/exp/rsqrt/rcp.
template <> struct Num<float> {
#if defined(__CUDA_ARCH__)
  __device__ static float lg(float x) { return __logf(x); }
  __device__ static float ex(float x) { return __expf(x); }
  __device__ static float rcp(float x) { return __frcp_rn(x); }
#else
  static float lg(float x) { return logf(x); }
  static float ex(float x) { return expf(x); }
  static float rcp(float x) { return 1.0f / x; }
#endif
  GPC_HD static float rsq(float x) { return gpc::rsqf(x); }
};

// The record holding a component's tables.
GPC_HD GPC_FI const GpComp* tables(const GpComp* cp) { return cp + ldg(&cp->tab); }

// Interval index of s in [0, kChebN] without float<->int conversions (their
// latency sat on the force's critical path): adding 1.5 * 2^52 (resp.
// 1.5 * 2^23 in single precision) to s - 1/2 rounds it to an integer held in
// the low mantissa bits; at exact ties either neighbouring interval is
// valid.  Returns the index (clamped to the last interval) and sets the
// interval's start as a floating-point number.
template <typename T>
GPC_HD GPC_FI int interval_of(T s, T& start);
template <>
GPC_HD GPC_FI int interval_of<double>(double s, double& start)
{
  constexpr double M = 6755399441055744.0;  // 1.5 * 2^52
  const double r = (s - 0.5) + M;
  int k = (int)(bits_of(r) & 63);
  k = k < kChebN - 1 ? k : kChebN - 1;
  start = fmin(r - M, (double)(kChebN - 1));
  return k;
}
template <>
GPC_HD GPC_FI int interval_of<float>(float s, float& start)
{
  constexpr float M = 12582912.0f;  // 1.5 * 2^23
  const float r = (s - 0.5f) + M;
  int b;
#if defined(__CUDA_ARCH__)
  b = __float_as_int(r);
#else
  memcpy(&b, &r, sizeof(b));
#endif
  int k = b & 63;
  k = k < kChebN - 1 ? k : kChebN - 1;
  start = fminf(r - M, (float)(kChebN - 1));
  return k;
}

// Degree-11 polynomial sum_k c[k] x^k, |x| <= 1, by Estrin's scheme: the
// twelve coefficients pair up as (c0 + c1 x) + x^2 (c2 + c3 x) + ... and the
// pairs combine with x^2, x^4, x^8, so the dependency chain is 5 operations
// deep instead of Horner's 11 (FP64 operations have long latencies and the
// force is one dependent chain per step).  The coefficients of the tables
// decay, and the result stays within a few ulp (tests/test_harness.py).
template <typename T>
GPC_HD GPC_FI T poly12(const T* __restrict__ c, T x)
{
  const T x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
  const T p01 = fma(ldg(c + 1), x, ldg(c + 0)), p23 = fma(ldg(c + 3), x, ldg(c + 2));
  const T p45 = fma(ldg(c + 5), x, ldg(c + 4)), p67 = fma(ldg(c + 7), x, ldg(c + 6));
  const T p89 = fma(ldg(c + 9), x, ldg(c + 8)), pab = fma(ldg(c + 11), x, ldg(c + 10));
  const T q0 = fma(p23, x2, p01), q1 = fma(p67, x2, p45), q2 = fma(pab, x2, p89);
  return fma(q2, x8, fma(q1, x4, q0));
}

// gamma*(a, u) from the component's table, u in [0, U): on each interval
// the degree-11 Chebyshev interpolant is stored in the power basis of the
// interval's local variable x in [-1, 1] (tests/test_harness.py checks the
// values against mpmath).

// tp: the component's table record (tables(cp); cp itself in a launch with a
// single potential, where every record holds its own tables).
template <typename T>
GPC_HD GPC_FI T gamma_star(const GpComp* __restrict__ tp, T u, T scale)
{
  const T s = u * scale;
  T start;
  const int k = interval_of<T>(s, start);
  const T x = T(2) * (s - start) - T(1);
  // the FP32 path reads the single-precision copy (no conversions)
  const T* c;
  if constexpr (sizeof(T) == sizeof(double))
    c = tp->cheb[k];
  else
    c = tp->chebf[k];
  return poly12<T>(c, x);
}

// x = m 2^e (x > 0 normal): the binade-table polynomial at m, e + 1024 and
// the table row.
struct Binade {
  int ebias;  // e + 1024, in [1, 2047] for normal x
  int j;      // m's eighth of [1, 2): the table row
  const double* row;
  double t;   // local variable of m's eighth of [1, 2), in [-1, 1)
  double m1;  // m - 1 (exact)
};

GPC_HD GPC_FI Binade binade(const GpComp* __restrict__ tp, double x)
{
  const long long b = bits_of(x);
  Binade r;
  r.ebias = (int)((b >> 52) & 0x7ff) + 1;
  const int j = (int)((b >> 49) & 7);
  const double m = double_of((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
  // m with its top three fraction bits cleared: 1 + (m - (1 + j/8)), so the
  // local variable 16 (m - 1 - j/8) - 1 needs no integer conversion
  const double mlow = double_of((b & 0x0001ffffffffffffLL) | 0x3ff0000000000000LL);
  r.t = 16.0 * mlow - 17.0;  // exact
  r.m1 = m - 1.0;            // exact
  r.j = j;
  r.row = tp->bin[j];
  return r;
}

GPC_HD GPC_FI double horner12(const double* c, double t) { return poly12<double>(c, t); }

// The same polynomial with its tail in single precision:
//   p(x) = sum_{k<K} c_k x^k + x^K q(x),  q = sum_{k>=K} c_k x^(k-K),
// the leading K terms in float64 and q (from the single-precision copy of
// the coefficients, cf) in float32.  K = 4 on the binade tables (local
// variable over an eighth of [1, 2): |c4 / c0| ~ 1e-5, so q's rounding moves
// p by ~1e-12 relative), K = 6 on the wider gamma* intervals (|c6 / c0|
// ~ 1e-5); tests/test_harness.py bounds the resulting force against the
// float64 one.  Six (K = 4) or nine (K = 6) float64 operations instead of
// fourteen.
template <int K>
GPC_HD GPC_FI double poly12_tail32(const double* __restrict__ c, const float* __restrict__ cf,
                                   double x)
{
  static_assert(K == 4 || K == 6, "float64 head of 4 or 6 terms");
  const double x2 = x * x;
  const float xf = (float)x, x2f = xf * xf;
  if constexpr (K == 4) {
    const double lead = fma(fma(ldg(c + 3), x, ldg(c + 2)), x2, fma(ldg(c + 1), x, ldg(c + 0)));
    const float x4f = x2f * x2f;
    const float q01 = fmaf(ldg(cf + 5), xf, ldg(cf + 4));
    const float q23 = fmaf(ldg(cf + 7), xf, ldg(cf + 6));
    const float q45 = fmaf(ldg(cf + 9), xf, ldg(cf + 8));
    const float q67 = fmaf(ldg(cf + 11), xf, ldg(cf + 10));
    const float q = fmaf(fmaf(q67, x2f, q45), x4f, fmaf(q23, x2f, q01));
    return fma(x2 * x2, (double)q, lead);
  } else {
    const double x4 = x2 * x2;
    const double p01 = fma(ldg(c + 1), x, ldg(c + 0)), p23 = fma(ldg(c + 3), x, ldg(c + 2));
    const double p45 = fma(ldg(c + 5), x, ldg(c + 4));
    const double lead = fma(p45, x4, fma(p23, x2, p01));
    const float q01 = fmaf(ldg(cf + 7), xf, ldg(cf + 6));
    const float q23 = fmaf(ldg(cf + 9), xf, ldg(cf + 8));
    const float q45 = fmaf(ldg(cf + 11), xf, ldg(cf + 10));
    const float q = fmaf(q45, x2f * x2f, fmaf(q23, x2f, q01));
    return fma(x4 * x2, (double)q, lead);
  }
}

// (r^2)^(-alpha/2) from the PowerSphericalwCutoff component's tables
// (TAIL32: the polynomial's tail in single precision, poly12_tail32)
template <bool TAIL32 = false>
GPC_HD GPC_FI double pswc_power(const GpComp* __restrict__ tp, double r2)
{
  const Binade q = binade(tp, r2);
  const double s = ldg(&tp->e2hi[q.ebias >> 6]) * ldg(&tp->e2lo[q.ebias & 63]);
  if constexpr (TAIL32)
    return s * poly12_tail32<4>(q.row, tp->binf[q.j], q.t);
  else
    return s * horner12(q.row, q.t);
}

// log1p(x), x >= 0, from the NFW component's table of log(m) / (m - 1)
// (smooth, 1 at m = 1, so small arguments keep their relative accuracy):
// u = 1 + x rounded, log1p(x) = log(u) + (x - (u - 1)) / u to first order in
// the rounding of u.
template <bool TAIL32 = false>
GPC_HD GPC_FI double nfw_log1p(const GpComp* __restrict__ tp, double x)
{
  // ln 2 = ln2_hi + ln2_lo, the head rounded to 32 significant bits so that
  // e * ln2_hi is exact for every binade e
  constexpr double ln2_hi = 0.6931471803691238;
  constexpr double ln2_lo = 1.9082149292705877e-10;
  const double u = 1.0 + x;
  const double corr = (x - (u - 1.0)) * rcp_nr(u);
  const Binade q = binade(tp, u);
  // e as a double without a conversion: 2^52 + ebias, minus 2^52 + 1024
  const double e = double_of(0x4330000000000000LL | (long long)q.ebias) - 4503599627371520.0;
  double p;
  if constexpr (TAIL32)
    p = poly12_tail32<4>(q.row, tp->binf[q.j], q.t);
  else
    p = horner12(q.row, q.t);
  return fma(e, ln2_hi, fma(q.m1, p, fma(e, ln2_lo, corr)));
}

// The same log1p in single precision from the float copy of the table.
GPC_HD GPC_FI float f32_of_bits(int b)
{
#if defined(__CUDA_ARCH__)
  return __int_as_float(b);
#else
  float x;
  memcpy(&x, &b, sizeof(x));
  return x;
#endif
}

GPC_HD GPC_FI float nfw_log1pf(const GpComp* __restrict__ tp, float x)
{
  const float u = 1.0f + x;
  int b;
#if defined(__CUDA_ARCH__)
  b = __float_as_int(u);
#else
  memcpy(&b, &u, sizeof(b));
#endif
  const int eb = (b >> 23) & 0xff;
  // the rounding correction of u divided by u to within a factor 2
  // (2^-e): it is below single-precision resolution of the result already
  const float corr = (x - (u - 1.0f)) * f32_of_bits((254 - eb) << 23);
  const int j = (b >> 20) & 7;
  const float m = f32_of_bits((b & 0x7fffff) | 0x3f800000);
  const float mlow = f32_of_bits((b & 0xfffff) | 0x3f800000);  // top 3 fraction bits cleared
  const float t = 16.0f * mlow - 17.0f;
  const float e = f32_of_bits(0x4b000000 | eb) - 8388735.0f;  // (2^23 + eb) - (2^23 + 127)
  const float p = poly12<float>(tp->binf[j], t);
  return fmaf(e, 0.69314718f, fmaf(m - 1.0f, p, corr));
}

// Regularised lower incomplete gamma P(a, x), a > 0 (series, A&S 6.5.29;
// Legendre continued fraction for Q, A&S 6.5.31, modified Lentz).  The
// bulge's potential energy and the Einasto profile use it; the bulge force
// uses the gamma* table.
GPC_HD inline double inc_gamma_P(double a, double x, double lga)
{
  if (!(x > 0.0)) return 0.0;
  const double lpref = a * log(x) - x - lga;
  if (x < a + 1.0) {
    double ap = a, term = 1.0 / a, sum = term;
    for (int n = 0; n < 1000; n++) {
      ap += 1.0;
      term *= x / ap;
      sum += term;
      if (fabs(term) < fabs(sum) * 1e-17) break;
    }
    return sum * exp(lpref);
  }
  double b = x + 1.0 - a, c = 1.0 / 1e-300, d = 1.0 / b, h = d;
  for (int i = 1; i < 1000; i++) {
    const double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (fabs(d) < 1e-300) d = 1e-300;
    c = b + an / c;
    if (fabs(c) < 1e-300) c = 1e-300;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (fabs(del - 1.0) < 1e-17) break;
  }
  return 1.0 - exp(lpref) * h;
}

// Exponential integral E1(x), x > 0 (ExpTruncNFW): the power series
// -gamma_E - ln x - sum_k (-x)^k / (k k!) for x <= 1 (A&S 5.1.11), the
// continued fraction e^-x / (x + 1 - 1 / (x + 3 - 4 / (x + 5 - ...))) for
// x > 1 (A&S 5.1.22, modified Lentz).
GPC_HD inline double expint_E1(double x)
{
  if (x <= 1.0) {
    double term = 1.0, sum = 0.0;
    for (int k = 1; k < 200; k++) {
      term *= -x / k;
      const double d = term / k;
      sum += d;
      if (fabs(d) < 1e-17 * fabs(sum)) break;
    }
    return -0.57721566490153286061 - log(x) - sum;
  }
  double b = x + 1.0, c = 1e300, d = 1.0 / b, h = d;
  for (int i = 1; i < 1000; i++) {
    const double an = -(double)i * i;
    b += 2.0;
    d = 1.0 / (an * d + b);
    c = b + an / c;
    const double del = c * d;
    h *= del;
    if (fabs(del - 1.0) < 1e-16) break;
  }
  return h * exp(-x);
}

// ExpTruncNFW's enclosed-mass function F(r) (ExpTruncNFWPotential.c): a
// series below the small-r threshold, else e^alpha (1 + alpha) (E1(alpha) -
// E1(beta)) - 1 + a e^(-r/rc) / (a + r), beta = (a + r) / rc.
// S: the component's scalar accessor (sc[j] = c[j]).
template <class S>
GPC_HD inline double exptruncnfw_F(const S& sc, double r)
{
  const double a = sc[1], irc = sc[2];
  if (r < sc[5]) return (r * r / (a * a)) * (sc[6] + r * (sc[7] + r * (sc[8] + r * sc[9])));
  return sc[4] - sc[3] * expint_E1((a + r) * irc) - 1.0 + a * exp(-r * irc) / (a + r);
}

// ------------------------------------------------------------- forces ---
// Add one component's contribution to the radial factors: the acceleration
// is a = (x gR, y (gR + gyx), z gz) + a0, where a0 takes the terms that are
// not of that form (Henon-Heiles' -amp x^2 in a_y, ellipsoidal components).
// TYPE < 0: read the type at run time, any supported type (kRunTimeAll) or
// any but the ellipsoidal family (kRunTimeCommon).
constexpr int kRunTimeAll = -1, kRunTimeCommon = -2;
// Scalar parameters of a component: from the compiled record in global
// memory (read-only path), or from a copy passed as a kernel parameter
// (constant bank: no load instruction when the index is a compile-time
// constant) when every orbit of a launch uses the same potential.
struct ScalarsGlobal {
  static constexpr bool kDirect = false;
  const GpComp* cp;
  GPC_HD GPC_FI double operator[](int j) const { return ldg(&cp->c[j]); }
};
struct ScalarsDirect {
  static constexpr bool kDirect = true;  // one potential: records hold their own tables
  const double* p;
  GPC_HD GPC_FI double operator[](int j) const { return p[j]; }
};

// Acceleration terms that are not of the radial-factor form (Henon-Heiles'
// -amp x^2 in a_y, the ellipsoidal components' full vectors).
template <typename T>
struct AddAcc {
  T x, y, z;
};

// ---- ellipsoidal components -------------------------------------------
// Record: c[0] amp, c[1..4] the density's parameters (TriaxialHernquist
// (a, a^4), TriaxialNFW (a, a^3), TriaxialJaffe (a, a^2), TwoPowerTriaxial
// (a, alpha, beta, beta - alpha), PerfectEllipsoid (a^2), TriaxialGaussian
// (-2 sigma^2), PowerTriaxial (alpha)), c[5] the Gauss-Legendre order n,
// c[6] 1 if the principal axes are not the coordinate axes; the rotation
// (row-major, x' = rot x) in bin[0][0..8]; per node k of the integral over
// tau, cheb[] holds (w_k, 1/(1+tau_k), 1/(b^2+tau_k), 1/(c^2+tau_k)) with
// galpy's weights w_k (the -4 pi b c / sqrt(...) factor included).
// Force per unit amp: F' = sum_k w_k rho(m_k) (x'/(1+tau_k), y'/(b^2+tau_k),
// z'/(c^2+tau_k)), m_k^2 = x'^2/(1+tau_k) + y'^2/(b^2+tau_k) + z'^2/(c^2+tau_k),
// F = rot^T F'.
constexpr int kEllMaxOrder = kChebN * kChebC / 4;

GPC_HD GPC_FI double ell_rho(int type, const GpComp* cp, double m2, double& m)
{
  const double p1 = ldg(&cp->c[1]);
  switch (type) {
    case T_PERFECTELL: {
      const double d = 1.0 / (p1 + m2);
      return d * d;
    }
    case T_TRIGAUSS: return exp(m2 / p1);
    case T_POWERTRI: return exp(-0.5 * p1 * log(m2));
    default: break;
  }
  m = sqrt(m2);
  const double mpa = m + p1, p2 = ldg(&cp->c[2]);
  switch (type) {
    case T_TRIHERNQUIST: return p2 / (m * mpa * mpa * mpa);
    case T_TRINFW: return p2 / (m * mpa * mpa);
    case T_TRIJAFFE: {
      const double d = 1.0 / (m * mpa);
      return p2 * p2 * d * d;
    }
    default:  // TwoPowerTriaxial: (a/m)^alpha (1 + m/a)^-(beta - alpha)
      return exp(p2 * log(p1 / m) - ldg(&cp->c[4]) * log1p(m / p1));
  }
}

// rho'(m) / m, given rho(m) and m (set by ell_rho for the types that use it)
GPC_HD GPC_FI double ell_drho_over_m(int type, const GpComp* cp, double m2, double m, double rho)
{
  const double p1 = ldg(&cp->c[1]);
  switch (type) {
    case T_PERFECTELL: return -4.0 * rho / (p1 + m2);
    case T_TRIGAUSS: return 2.0 * rho / p1;
    case T_POWERTRI: return -p1 * rho / m2;
    case T_TRIHERNQUIST: return -rho * (p1 + 4.0 * m) / (m2 * (m + p1));
    case T_TRINFW: return -rho * (p1 + 3.0 * m) / (m2 * (m + p1));
    case T_TRIJAFFE: return -2.0 * rho * (p1 + 2.0 * m) / (m2 * (m + p1));
    default:  // TwoPowerTriaxial
      return -rho * (p1 * ldg(&cp->c[2]) + ldg(&cp->c[3]) * m) / (m2 * (m + p1));
  }
}

// Acceleration of one ellipsoidal component (amp included), FP64.
GPC_HD GPC_FI void ell_accel(const GpComp* __restrict__ cp, int type, double x, double y,
                             double z, double& ax, double& ay, double& az)
{
  const double* rot = &cp->bin[0][0];
  const bool rotated = ldg(&cp->c[6]) != 0.0;
  if (rotated) {
    const double xr = ldg(rot + 0) * x + ldg(rot + 1) * y + ldg(rot + 2) * z;
    const double yr = ldg(rot + 3) * x + ldg(rot + 4) * y + ldg(rot + 5) * z;
    const double zr = ldg(rot + 6) * x + ldg(rot + 7) * y + ldg(rot + 8) * z;
    x = xr;
    y = yr;
    z = zr;
  }
  const int n = (int)ldg(&cp->c[5]);
  const double* nd = &cp->cheb[0][0];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int k = 0; k < n; k++, nd += 4) {
    const double w = ldg(nd), i1 = ldg(nd + 1), i2 = ldg(nd + 2), i3 = ldg(nd + 3);
    const double xs = x * i1, ys = y * i2, zs = z * i3;
    const double m2 = x * xs + y * ys + z * zs;
    double m = 0.0;
    const double td = w * ell_rho(type, cp, m2, m);
    fx += td * xs;
    fy += td * ys;
    fz += td * zs;
  }
  if (rotated) {
    const double gx = ldg(rot + 0) * fx + ldg(rot + 3) * fy + ldg(rot + 6) * fz;
    const double gy = ldg(rot + 1) * fx + ldg(rot + 4) * fy + ldg(rot + 7) * fz;
    const double gz = ldg(rot + 2) * fx + ldg(rot + 5) * fy + ldg(rot + 8) * fz;
    fx = gx;
    fy = gy;
    fz = gz;
  }
  const double amp = ldg(&cp->c[0]);
  ax = amp * fx;
  ay = amp * fy;
  az = amp * fz;
}

// Tidal tensor K = -amp d^2 Phi / dx dx of one ellipsoidal component,
// evaluated in the principal-axis form at the given (unrotated) point as
// the reference's EllipsoidalPotential_2ndderiv_xyz_all is called; K[i] is
// added to (xx, xy, yy, xz, yz, zz).
GPC_HD GPC_FI void ell_tidal(const GpComp* __restrict__ cp, int type, double x, double y,
                             double z, double K[6])
{
  const int n = (int)ldg(&cp->c[5]);
  const double* nd = &cp->cheb[0][0];
  double h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // xx, xy, xz, yy, yz, zz per unit amp
  for (int k = 0; k < n; k++, nd += 4) {
    const double w = ldg(nd), i1 = ldg(nd + 1), i2 = ldg(nd + 2), i3 = ldg(nd + 3);
    const double xs = x * i1, ys = y * i2, zs = z * i3;
    const double m2 = x * xs + y * ys + z * zs;
    double m = sqrt(m2);
    const double rho = ell_rho(type, cp, m2, m);
    const double dv = w * rho, dd = w * ell_drho_over_m(type, cp, m2, m, rho);
    h[0] -= dd * xs * xs + dv * i1;
    h[1] -= dd * xs * ys;
    h[2] -= dd * xs * zs;
    h[3] -= dd * ys * ys + dv * i2;
    h[4] -= dd * ys * zs;
    h[5] -= dd * zs * zs + dv * i3;
  }
  const double amp = ldg(&cp->c[0]);
  K[0] -= amp * h[0];
  K[1] -= amp * h[1];
  K[2] -= amp * h[3];
  K[3] -= amp * h[2];
  K[4] -= amp * h[4];
  K[5] -= amp * h[5];
}

// KuzminKutuzovStaeckel: Phi = -amp V, V = 1 / (sqrt(l) + sqrt(n)) with the
// prolate spheroidal coordinates l, n = (R^2 + z^2 - alpha - gamma +- sqrt(D))
// / 2, D = (R^2 + z^2 - Delta^2)^2 + 4 Delta^2 R^2.  kks_parts returns the
// pieces the force and the tidal tensor share.
struct KksParts {
  double isd, l, n, srl, srn, isln2, dVdl, dVdn;
};
GPC_HD GPC_FI KksParts kks_parts(double D2, double apg, double R2, double z2)
{
  KksParts k;
  const double r2 = R2 + z2, rzm = r2 - D2;
  const double sd = sqrt(rzm * rzm + 4.0 * D2 * R2);
  k.isd = 1.0 / sd;
  k.l = 0.5 * (r2 - apg + sd);
  k.n = 0.5 * (r2 - apg - sd);
  k.srl = sqrt(k.l);
  k.srn = sqrt(k.n);
  const double sln = k.srl + k.srn;
  k.isln2 = 1.0 / (sln * sln);
  k.dVdl = 0.5 / k.srl * k.isln2;  // -dV/dl
  k.dVdn = 0.5 / k.srn * k.isln2;  // -dV/dn
  return k;
}

// The spherical potentials' acceleration factor -Phi'(r)/r (a = f x), for
// the run-time component list; FP32 and FP64 alike.
template <typename T, class S>
GPC_HD GPC_FI T sph_force_factor(int type, const S& sc, T r2)
{
  const T amp = T(sc[0]);
  switch (type) {
    case T_POWER:  // Phi' = amp r^(1-alpha)
      return -amp * Num<T>::ex(T(sc[1]) * Num<T>::lg(r2));
    case T_JAFFE: {  // Phi' = amp / (r (r + a))
      const T ir = Num<T>::rsq(r2);
      return -amp * ir * ir * Num<T>::rcp(r2 * ir + T(sc[1]));
    }
    case T_ISOCHRONE: {  // Phi' = amp r / (rb (b + rb)^2), rb = sqrt(r^2 + b^2)
      const T rb2 = r2 + T(sc[2]), irb = Num<T>::rsq(rb2);
      const T ib = Num<T>::rcp(T(sc[1]) + rb2 * irb);
      return -amp * irb * ib * ib;
    }
    case T_PLUMMER: {  // Phi' = amp r (r^2 + b^2)^(-3/2)
      const T i = Num<T>::rsq(r2 + T(sc[1]));
      return -amp * i * i * i;
    }
    case T_PSEUDOISO: {  // Phi' = amp (1/r - a atan(r/a) / r^2) / a
      const T ir = Num<T>::rsq(r2), r = r2 * ir;
      return -amp * T(sc[2]) * ir * ir * (T(1) - T(sc[1]) * atan(r * T(sc[2])) * ir);
    }
    case T_BURKERT: {  // Phi' = -amp pi a^3 / r^2 (2 atan x - 2 ln(1+x) - ln(1+x^2)), x = r/a
      const T ir = Num<T>::rsq(r2), x = r2 * ir * T(sc[2]);
      const T B = T(2) * atan(x) - T(2) * log1p(x) - log1p(x * x);
      return amp * T(sc[3]) * ir * ir * ir * B;
    }
    case T_DEHNENCORE: {  // Phi' = amp r / (3 (a + r)^3)
      const T ia = Num<T>::rcp(r2 * Num<T>::rsq(r2) + T(sc[1]));
      return -amp * ia * ia * ia / T(3);
    }
    case T_DEHNEN: {  // Phi' = amp r (1 + a/r)^alpha / ((a + r)^3 (3 - alpha))
      const T ir = Num<T>::rsq(r2), ia = Num<T>::rcp(r2 * ir + T(sc[1]));
      const T w = Num<T>::ex(T(sc[2]) * Num<T>::lg(T(1) + T(sc[1]) * ir));
      return -amp * T(sc[3]) * w * ia * ia * ia;
    }
    case T_HOMSPHERE: {  // Phi' = 2 amp r inside R, 2 amp R^3 / r^2 outside
      const T ir = Num<T>::rsq(r2);
      return r2 < T(sc[1]) ? T(-2) * amp : T(-2) * amp * T(sc[2]) * ir * ir * ir;
    }
    case T_EXPTRUNCNFW: {  // Phi'/r = amp F(r) / r^3 (in float64)
      const double r = sqrt((double)r2);
      return T(-(double)amp * exptruncnfw_F(sc, r) / (r * r * r));
    }
    case T_EINASTO: {  // Phi'/r = amp 4 pi n h^3 gamma(3n, (r/h)^(1/n)) / r^3 (in float64)
      const double r = sqrt((double)r2), x = pow(r / sc[1], sc[2]);
      const double P = inc_gamma_P(sc[3], x, sc[4]);
      return T(-(double)amp * sc[5] * P / (r * r * r));
    }
    default:  // T_NULL
      return T(0);
  }
}

// MIX (float64 path only): 0 plain float64; MIX_TAIL32 the table
// polynomials' tails in float32 (poly12_tail32); MIX_F32BULGE in addition the
// whole bulge (PowerSphericalwCutoff) term in float32.
enum : int { MIX_NONE = 0, MIX_TAIL32 = 1, MIX_F32BULGE = 2 };

// gamma*(a, u) with the interpolant's tail in float32 (poly12_tail32).
}  // namespace gpc
#include "potentials_td.cuh"
namespace gpc {

GPC_HD GPC_FI double gamma_star_tail32(const GpComp* __restrict__ tp, double u, double scale)
{
  const double s = u * scale;
  double start;
  const int k = interval_of<double>(s, start);
  const double x = 2.0 * (s - start) - 1.0;
  return poly12_tail32<6>(tp->cheb[k], tp->chebf[k], x);
}

template <typename T, bool PLANAR, int TYPE, class S, int MIX = MIX_NONE>
GPC_HD GPC_FI void comp_accel(const GpComp* __restrict__ cp, const S& sc, T x, T y, T z, T z2,
                              T R2, T r2, T& gR, T& gz, T& gyx, AddAcc<T>& a0, double t)
{
  const int type = TYPE >= 0 ? TYPE : ldg(&cp->type);
  const T amp = T(sc[0]);
  constexpr bool F64 = sizeof(T) == sizeof(double);  // FP64: branch-free helpers
  const GpComp* tp = S::kDirect ? cp : tables(cp);
  switch (type) {
    case T_PSWC: {
      // F = -amp M(r)/r^3 r_vec
      const T u = r2 * T(sc[1]);
      T f;
      if constexpr (F64 && MIX == MIX_F32BULGE) {
        // the bulge term in float32 (as the FP32-force path), the rest of the
        // force in float64
        const float r2f = (float)r2, uf = (float)u;
        const float pw = Num<float>::ex((float)sc[3] * Num<float>::lg(r2f));
        const float ir = Num<float>::rsq(r2f);
        const float inner = (float)sc[2] * pw *
                            gamma_star<float>(tp, uf < (float)sc[5] ? uf : (float)sc[5],
                                              (float)sc[6]);
        const float outer = (float)sc[4] * (ir * ir * ir);
        f = -amp * (double)(uf < (float)sc[5] ? inner : outer);
      } else if constexpr (F64) {
        // both forms, then a select: no branch in the force chain
        const double ir = rsqrt_nr(r2);
        const double g = MIX == MIX_TAIL32 ? gamma_star_tail32(tp, fmin(u, sc[5]), sc[6])
                                           : gamma_star<double>(tp, fmin(u, sc[5]), sc[6]);
        const double inner = sc[2] * pswc_power<MIX == MIX_TAIL32>(tp, r2) * g;
        const double outer = sc[4] * (ir * ir * ir);
        f = -amp * (u < sc[5] ? inner : outer);
      } else {  // single precision: hardware log2/exp2 for the power, same select
        const T pw = Num<T>::ex(T(sc[3]) * Num<T>::lg(r2));  // (r^2)^(-alpha/2)
        const T ir = Num<T>::rsq(r2);
        const T inner = T(sc[2]) * pw * gamma_star<T>(tp, u < T(sc[5]) ? u : T(sc[5]), T(sc[6]));
        const T outer = T(sc[4]) * (ir * ir * ir);
        f = -amp * (u < T(sc[5]) ? inner : outer);
      }
      gR += f;
      gz += f;
      break;
    }
    case T_MN: {
      const T a = T(sc[1]);
      const T zb2 = z2 + T(sc[2]);
      const T izb = Num<T>::rsq(zb2);
      const T s = a + zb2 * izb;  // a + sqrt(z^2 + b^2)
      const T iD = Num<T>::rsq(R2 + s * s);
      const T iD3 = iD * iD * iD;
      gR -= amp * iD3;
      if (!PLANAR) gz -= amp * s * izb * iD3;
      break;
    }
    case T_NFW: {
      // Phi = -amp ln(1 + r/a)/r ; F = amp (1/(r^2 (a+r)) - ln(1+r/a)/r^3) r_vec
      const T a = T(sc[1]);
      T f;
      if constexpr (F64) {
        const double ir = rsqrt_nr(r2);
        const double r = r2 * ir;
        f = amp * ir * ir * (rcp_nr(a + r) - nfw_log1p<(MIX > MIX_NONE)>(tp, r * sc[2]) * ir);
      } else {
        const T ir = Num<T>::rsq(r2);
        const T r = r2 * ir;
        f = amp * ir * ir * (Num<T>::rcp(a + r) - nfw_log1pf(tp, r * T(sc[2])) * ir);
      }
      gR += f;
      gz += f;
      break;
    }
    case T_HERNQUIST: {
      // Phi = -amp / (2 (r + a)) ; F = -amp / (2 r (r + a)^2) r_vec
      const T a = T(sc[1]);
      const T ir = Num<T>::rsq(r2);
      const T ira = Num<T>::rcp(r2 * ir + a);
      const T f = -T(0.5) * amp * ir * ira * ira;
      gR += f;
      gz += f;
      break;
    }
    case T_KKS: {  // in float64: a = -amp (x g_R, y g_R, z g_z)
      const double D2 = sc[1];
      const KksParts k = kks_parts(D2, sc[2], (double)R2, (double)z2);
      const double r2d = (double)R2 + (double)z2;
      const double fR = (1.0 + (r2d + D2) * k.isd) * k.dVdl + (1.0 - (r2d + D2) * k.isd) * k.dVdn;
      const double fz = (1.0 + (r2d - D2) * k.isd) * k.dVdl + (1.0 - (r2d - D2) * k.isd) * k.dVdn;
      gR -= amp * T(fR);
      if (!PLANAR) gz -= amp * T(fz);
      break;
    }
    case T_FLATPOWER: {
      // Phi = -amp m^(-alpha) / alpha (alpha = 0: amp/2 ln m^2),
      // m^2 = R^2 + z^2/q^2 + core^2: a = -amp (m^2)^(-alpha/2-1) (x, y, z/q^2)
      const T iq2 = T(sc[1]);
      const T m2 = R2 + z2 * iq2 + T(sc[2]);
      const T g = -amp * Num<T>::ex(T(sc[3]) * Num<T>::lg(m2));
      gR += g;
      if (!PLANAR) gz += g * iq2;
      break;
    }
    case T_LOGHALO: {
      // Phi = amp/2 ln(x^2 + (1-e) y^2 + z^2/q^2 + core^2)
      const T iq2 = T(sc[1]);
      const T ye = T(sc[3]);
      const T D = x * x + ye * y * y + z2 * iq2 + T(sc[2]);
      const T g = -amp * Num<T>::rcp(D);
      gR += g;
      gyx += g * (ye - T(1));
      if (!PLANAR) gz += g * iq2;
      break;
    }
    case T_HENONHEILES: {
      // Phi = amp ((x^2 + y^2)/2 + x^2 y - y^3/3) (planar only):
      // a = -amp (x (1 + 2y), y (1 - y) + x^2)
      gR -= amp * (T(1) + T(2) * y);
      gyx += T(3) * amp * y;
      a0.y -= amp * x * x;
      break;
    }
    case T_KUZMINDISK: {
      // a = -amp D^(-3/2) (x, y, sign(z) (a + |z|)), D = R^2 + (a + |z|)^2;
      // a_z through a0 (sign(0) = 0, as the reference's zforce)
      const T az = T(sc[1]) + (PLANAR ? T(0) : (z < T(0) ? -z : z));
      const T iD = Num<T>::rsq(R2 + az * az);
      const T g = -amp * iD * iD * iD;
      gR += g;
      if (!PLANAR) a0.z += z > T(0) ? g * az : (z < T(0) ? -g * az : T(0));
      break;
    }
    case T_PAYLOAD:  // an SCF component's coefficients
      break;
    case T_WRAP_SMOOTH:
    case T_WRAP_ROTATE:
    case T_WRAP_GAUSS:  // opened by the full list's loop; no other list carries one
      gR = T(NAN);
      break;
    case T_SPIRALARMS: {  // in float64, full list only
      if constexpr (TYPE == kRunTimeAll) {
        double ax = 0.0, ay = 0.0, az = 0.0;
        spiral_accel<PLANAR>(cp, (double)x, (double)y, (double)z, t, ax, ay, az, nullptr);
        a0.x += T(ax);
        a0.y += T(ay);
        if (!PLANAR) a0.z += T(az);
      } else {
        gR = T(NAN);
      }
      break;
    }
    case T_TRANSPIRAL: case T_STEADYSPIRAL: case T_ELLDISK: case T_LOPSIDED:
    case T_COSMPHI: {  // planar only, in float64, full list only
      if constexpr (TYPE == kRunTimeAll && PLANAR) {
        double ax = 0.0, ay = 0.0;
        disk_pert_accel(cp, type, (double)x, (double)y, t, ax, ay, nullptr);
        a0.x += T(ax);
        a0.y += T(ay);
      } else {
        gR = T(NAN);
      }
      break;
    }
    case T_DEHNENBAR:
    case T_NEEDLEBAR:
    case T_SCF: {  // in float64; carried by the full run-time list only
      if constexpr (TYPE == kRunTimeAll) {
        double ax, ay, az;
        if (type == T_DEHNENBAR) {
          dbar_accel<PLANAR>(cp, t, (double)x, (double)y, (double)z, ax, ay, az);
        } else if (type == T_NEEDLEBAR) {
          ax = ay = az = 0.0;
          needle_accel<PLANAR>(cp, t, (double)x, (double)y, (double)z, ax, ay, az, nullptr);
        } else
          scf_accel<PLANAR>(cp, (double)x, (double)y, (double)z, ax, ay, az);
        a0.x += T(ax);
        a0.y += T(ay);
        if (!PLANAR) a0.z += T(az);
      } else {
        gR = T(NAN);
      }
      break;
    }
    case T_TRIHERNQUIST: case T_TRINFW: case T_TRIJAFFE: case T_PERFECTELL: case T_TRIGAUSS:
    case T_POWERTRI: case T_TWOPOWERTRI: {  // in float64
      if constexpr (TYPE == kRunTimeCommon) {
        // not carried by the common run-time list (the host never selects it
        // for such a potential): a non-finite force stops the orbit, err 3
        gR = T(NAN);
      } else {
        double ax, ay, az;
        ell_accel(tp, type, (double)x, (double)y, PLANAR ? 0.0 : (double)z, ax, ay, az);
        a0.x += T(ax);
        a0.y += T(ay);
        if (!PLANAR) a0.z += T(az);
      }
      break;
    }
    default: {
      const T f = sph_force_factor<T>(type, sc, r2);
      gR += f;
      gz += f;
      break;
    }
  }
}

// Run-time component list (any combination of the supported types).
// The full list also carries the time-dependent DehnenBar, the SCF
// expansion and the wrappers: its force reads the evaluation time
// (kTimeDep).  A wrapper opens a frame over the records it wraps: the
// accumulators are set aside, the wrapped components are evaluated at the
// point rotated by -alpha, and at the frame's end their acceleration,
// rotated back by alpha and scaled by the wrapper's factor, joins a0 (R^2
// and r^2 do not change under the rotation about z).  A KuzminLike frame
// evaluates them at (xi, 0, 0) instead and adds fac a_x' grad xi.
struct DynPot {
  static constexpr bool kDirectScalars = false;
  static constexpr bool kAdditive = true;  // a component may add to a0
  static constexpr bool kTimeDep = true;
  template <typename T, bool PLANAR>
  GPC_HD GPC_FI static void sum(const GpComp* __restrict__ comp, const double* /*scal*/, int ncomp,
                                T x, T y, T z, T z2, T R2, T r2, T& gR, T& gz, T& gyx,
                                AddAcc<T>& a0, double t)
  {
    int wend = -1;  // one past the open frame's last record
    T xw = x, yw = y, zw = z, z2w = z2, R2w = R2, r2w = r2, sR = T(0), sz = T(0), syx = T(0);
    AddAcc<T> sa{T(0), T(0), T(0)};
    WrapFrame fr{1.0, 1.0, 0.0, false, false, 0.0, 0.0, 0.0};
    for (int k = 0; k <= ncomp; k++) {
      if (k == wend) {  // close the frame
        const T fc = T(fr.c), fs = T(fr.s), ff = T(fr.fac);
        const T axw = xw * gR + a0.x, ayw = yw * (gR + gyx) + a0.y, azw = zw * gz + a0.z;
        gR = sR;
        gz = sz;
        gyx = syx;
        if (fr.kz) {  // fac dPhi/dxi grad xi, the wrapped force taken along x'
          const T g = ff * axw / T(fr.xi);
          a0.x = sa.x + g * x;
          a0.y = sa.y + g * y;
          if (!PLANAR) a0.z = sa.z + g * T(fr.q);
        } else {
          // a rotation by alpha(R) adds -fac tau' grad alpha, tau' the wrapped
          // torque about z, grad alpha = (alpha'/R) (x, y, 0)
          const T tq = fr.co ? ff * T(fr.q) * (xw * ayw - yw * axw) : T(0);
          a0.x = sa.x + ff * (fc * axw - fs * ayw) - tq * x;
          a0.y = sa.y + ff * (fs * axw + fc * ayw) - tq * y;
          if (!PLANAR) a0.z = sa.z + ff * azw;
        }
        xw = x;
        yw = y;
        zw = z;
        z2w = z2;
        R2w = R2;
        r2w = r2;
        wend = -1;
      }
      if (k == ncomp) break;
      const int type = ldg(&comp[k].type);
      if (is_wrapper(type)) {  // open a frame (wrappers do not nest)
        fr = wrap_frame(comp + k, type, t);
        wend = k + 1 + (int)ldg(&comp[k].c[15]);
        sR = gR;
        sz = gz;
        syx = gyx;
        sa = a0;
        gR = gz = gyx = T(0);
        a0 = AddAcc<T>{T(0), T(0), T(0)};
        if (fr.kz) {
          kuzmin_map<PLANAR>(comp + k, (double)R2, (double)z, fr);
          xw = T(fr.xi);
          yw = zw = z2w = T(0);
          R2w = r2w = xw * xw;
        } else {
          if (fr.co) corot_map(comp + k, (double)R2, t, fr);
          xw = T(fr.c) * x + T(fr.s) * y;
          yw = T(fr.c) * y - T(fr.s) * x;
        }
        continue;
      }
      comp_accel<T, PLANAR, kRunTimeAll>(comp + k, ScalarsGlobal{comp + k}, xw, yw, zw, z2w, R2w,
                                         r2w, gR, gz, gyx, a0, t);
    }
  }
};

// Run-time component list without the ellipsoidal family, whose
// Gauss-Legendre shell integral costs every kernel of the full list 5-30
// registers (and some kernels a resident block): the host selects it for
// potentials without such a component (GALPY_CUDA_SIG_COMMON).
struct DynPotCommon {
  static constexpr bool kDirectScalars = false;
  static constexpr bool kAdditive = true;
  static constexpr bool kTimeDep = false;
  template <typename T, bool PLANAR>
  GPC_HD GPC_FI static void sum(const GpComp* __restrict__ comp, const double* /*scal*/, int ncomp,
                                T x, T y, T z, T z2, T R2, T r2, T& gR, T& gz, T& gyx,
                                AddAcc<T>& a0, double /*t*/)
  {
    for (int k = 0; k < ncomp; k++)
      comp_accel<T, PLANAR, kRunTimeCommon>(comp + k, ScalarsGlobal{comp + k}, x, y, z, z2, R2,
                                            r2, gR, gz, gyx, a0, 0.0);
  }
};

// Compile-time component list: the components are inlined side by side.
// DIRECT: the scalars come from `scal` (kScalarStride doubles per component,
// a kernel-parameter copy), else from the records in global memory.
constexpr int kScalarStride = 16;
template <bool DIRECT, int... TYPES>
struct FixedPot {
  static constexpr bool kDirectScalars = DIRECT;
  static constexpr bool kAdditive =
      ((TYPES == T_HENONHEILES || TYPES == T_KUZMINDISK || is_ellipsoidal(TYPES)) || ...);
  static constexpr bool kTimeDep = false;
  template <typename T, bool PLANAR>
  GPC_HD GPC_FI static void sum(const GpComp* __restrict__ comp, const double* scal, int /*ncomp*/,
                                T x, T y, T z, T z2, T R2, T r2, T& gR, T& gz, T& gyx,
                                AddAcc<T>& a0, double /*t*/)
  {
    int k = 0;
    if (DIRECT) {
      ((comp_accel<T, PLANAR, TYPES>(comp + k, ScalarsDirect{scal + kScalarStride * k}, x, y, z,
                                     z2, R2, r2, gR, gz, gyx, a0, 0.0),
        ++k),
       ...);
    } else {
      ((comp_accel<T, PLANAR, TYPES>(comp + k, ScalarsGlobal{comp + k}, x, y, z, z2, R2, r2, gR,
                                     gz, gyx, a0, 0.0),
        ++k),
       ...);
    }
  }
};
// galpy's MWPotential2014 order; MW14Pot takes the scalars as kernel
// parameters (one potential per launch), MW14GroupPot from the records
// (parameter groups).
using MW14Pot = FixedPot<true, T_PSWC, T_MN, T_NFW>;
using MW14GroupPot = FixedPot<false, T_PSWC, T_MN, T_NFW>;

// A compile-time list evaluated in one of the mixed float64 / float32 forms
// (MIX_TAIL32, MIX_F32BULGE; float64 state and force accumulation).
template <bool DIRECT, int MIX, int... TYPES>
struct MixedPot {
  static constexpr bool kDirectScalars = DIRECT;
  static constexpr bool kAdditive = false;
  static constexpr bool kTimeDep = false;
  template <typename T, bool PLANAR>
  GPC_HD GPC_FI static void sum(const GpComp* __restrict__ comp, const double* scal, int /*ncomp*/,
                                T x, T y, T z, T z2, T R2, T r2, T& gR, T& gz, T& gyx,
                                AddAcc<T>& a0, double /*t*/)
  {
    int k = 0;
    if (DIRECT) {
      ((comp_accel<T, PLANAR, TYPES, ScalarsDirect, MIX>(
            comp + k, ScalarsDirect{scal + kScalarStride * k}, x, y, z, z2, R2, r2, gR, gz, gyx,
            a0, 0.0),
        ++k),
       ...);
    } else {
      ((comp_accel<T, PLANAR, TYPES, ScalarsGlobal, MIX>(comp + k, ScalarsGlobal{comp + k}, x,
                                                         y, z, z2, R2, r2, gR, gz, gyx, a0, 0.0),
        ++k),
       ...);
    }
  }
};
template <bool DIRECT, int MIX>
using MW14MixedPot = MixedPot<DIRECT, MIX, T_PSWC, T_MN, T_NFW>;

// Acceleration at (x, y, z) and time t (read by time-dependent components
// only); PLANAR evaluates galpy's planar potential (the 3D potential in the
// plane z = 0) and leaves az untouched.
template <typename T, bool PLANAR, class POT = DynPot>
GPC_HD GPC_FI void accel(const GpComp* __restrict__ comp, int ncomp, T x, T y, T z, T& ax, T& ay,
                         T& az, const double* scal = nullptr, double t = 0.0)
{
  const T R2 = x * x + y * y;
  const T z2 = PLANAR ? T(0) : z * z;
  const T r2 = R2 + z2;
  T gR = T(0), gz = T(0), gyx = T(0);
  AddAcc<T> a0{T(0), T(0), T(0)};
  POT::template sum<T, PLANAR>(comp, scal, ncomp, x, y, z, z2, R2, r2, gR, gz, gyx, a0, t);
  ax = x * gR;
  ay = y * (gR + gyx);
  if (!PLANAR) az = z * gz;
  if constexpr (POT::kAdditive) {  // compile-time lists without such terms skip the adds
    ax += a0.x;
    ay += a0.y;
    if (!PLANAR) az += a0.z;
  }
}

// ------------------------------------------------------ tidal tensor ---
// Acceleration and the symmetric Cartesian tidal tensor K = d a / d x
// (K[0]=xx, K[1]=xy, K[2]=yy, K[3]=xz, K[4]=yz, K[5]=zz), FP64.
// Spherical components use Phi'(r), Phi''(r):
//   K_ij = -(Phi'' - Phi'/r) x_i x_j / r^2 - Phi'/r delta_ij.
GPC_HD GPC_FI void add_spherical(double dphi_over_r, double d2phi, double x, double y, double z,
                                 double r2, double& gR, double& gz, double K[6])
{
  const double c = (d2phi - dphi_over_r) / r2;
  gR -= dphi_over_r;
  gz -= dphi_over_r;
  K[0] -= c * x * x + dphi_over_r;
  K[1] -= c * x * y;
  K[2] -= c * y * y + dphi_over_r;
  K[3] -= c * x * z;
  K[4] -= c * y * z;
  K[5] -= c * z * z + dphi_over_r;
}

// Phi'(r)/r and Phi''(r) of the spherical potentials (zero for Null).
GPC_HD inline void sph_derivs(const GpComp* __restrict__ cp, int type, double amp, double r2,
                              double& dpr, double& d2)
{
  const double r = sqrt(r2), ir = 1.0 / r, c1 = ldg(&cp->c[1]);
  dpr = d2 = 0.0;
  switch (type) {
    case T_POWER:
      dpr = amp * exp(ldg(&cp->c[1]) * log(r2));
      d2 = ldg(&cp->c[2]) * dpr;  // (1 - alpha) amp r^-alpha
      break;
    case T_JAFFE: {
      const double ira = 1.0 / (r + c1);
      dpr = amp * ir * ir * ira;
      d2 = -amp * (c1 + 2.0 * r) * ir * ir * ira * ira;
      break;
    }
    case T_ISOCHRONE: {
      const double b = c1, rb = sqrt(r2 + ldg(&cp->c[2])), ib = 1.0 / (b + rb);
      dpr = amp / rb * ib * ib;
      const double q = 1.0 / (rb * (b + rb));
      d2 = -amp * (-b * b * b - b * b * rb + 2.0 * r2 * rb) * q * q * q;
      break;
    }
    case T_PLUMMER: {
      const double i = 1.0 / sqrt(r2 + c1);
      dpr = amp * i * i * i;
      d2 = amp * (c1 - 2.0 * r2) * i * i * i * i * i;
      break;
    }
    case T_PSEUDOISO: {
      const double a = c1, at = atan(r / a);
      dpr = amp / a * (ir * ir - a * at * ir * ir * ir);
      d2 = amp * ir * ir * (2.0 * a * ir * at - (2.0 * a * a + r2) / (a * a + r2)) / a;
      break;
    }
    case T_BURKERT: {
      const double a = c1, x = r / a, pa3 = ldg(&cp->c[3]);
      const double B = 2.0 * atan(x) - 2.0 * log1p(x) - log1p(x * x);
      dpr = -amp * pa3 * ir * ir * ir * B;
      d2 = amp * pa3 * (4.0 / ((a * a + r2) * (a + r)) + 2.0 * B * ir * ir * ir);
      break;
    }
    case T_DEHNENCORE: {
      const double ia = 1.0 / (c1 + r);
      dpr = amp * ia * ia * ia / 3.0;
      d2 = -amp * (2.0 * r - c1) * ia * ia * ia * ia / 3.0;
      break;
    }
    case T_DEHNEN: {
      const double a = c1, alpha = ldg(&cp->c[2]), i3a = ldg(&cp->c[3]);
      const double ia = 1.0 / (a + r), w = pow(1.0 + a * ir, alpha);
      dpr = amp * i3a * w * ia * ia * ia;
      d2 = -amp * i3a * w * (2.0 * r + a * (alpha - 1.0)) * ia * ia * ia * ia;
      break;
    }
    case T_HOMSPHERE:
      if (r2 < c1) {
        dpr = d2 = 2.0 * amp;
      } else {
        dpr = 2.0 * amp * ldg(&cp->c[2]) * ir * ir * ir;
        d2 = -2.0 * dpr;
      }
      break;
    case T_EXPTRUNCNFW: {  // Phi'' = amp (e^(-r/rc) / (r (a + r)^2) - 2 F / r^3)
      const double F = exptruncnfw_F(ScalarsGlobal{cp}, r), ar = c1 + r;
      dpr = amp * F * ir * ir * ir;
      d2 = amp * (exp(-r * ldg(&cp->c[2])) * ir / (ar * ar) - 2.0 * F * ir * ir * ir);
      break;
    }
    case T_EINASTO: {  // Phi'' = amp (4 pi e^-x - 2 * 4 pi n Gamma(3n) P / s^3)
      const double x = pow(r / c1, ldg(&cp->c[2]));
      const double P = inc_gamma_P(ldg(&cp->c[3]), x, ldg(&cp->c[4]));
      const double s = r / c1;
      dpr = amp * ldg(&cp->c[5]) * P * ir * ir * ir;
      d2 = amp * (4.0 * M_PI * exp(-x) - 2.0 * ldg(&cp->c[6]) * P / (s * s * s));
      break;
    }
    default:
      break;
  }
}

// One component's acceleration terms and its part of K = d a / d x at
// (x, y, z) (the full list's cases; wrappers are opened by accel_tidal).
template <bool PLANAR>
GPC_HD GPC_FI void comp_tidal(const GpComp* __restrict__ cp, int type, double x, double y,
                              double z, double R2, double z2, double r2, double& gR, double& gz,
                              double& gyx, double& ax0, double& ay0, double& az0, double K[6],
                              double t)
{
  const double amp = ldg(&cp->c[0]);
  switch (type) {
    case T_PSWC: {
      const double u = r2 * ldg(&cp->c[1]);
      const double pw = exp(ldg(&cp->c[3]) * log(r2));  // (r^2)^(-alpha/2)
      double Mr3;                                         // M(r) / r^3
      if (u < ldg(&cp->c[5])) {
        Mr3 = ldg(&cp->c[2]) * pw * gamma_star<double>(tables(cp), u, ldg(&cp->c[6]));
      } else {
        const double ir = rsq(r2);
        Mr3 = ldg(&cp->c[4]) * ir * ir * ir;
      }
      const double dpr = amp * Mr3;  // Phi'/r
      // Phi'' = amp (4 pi r^-alpha exp(-r^2/rc^2) - 2 M / r^3)
      const double d2 = amp * (ldg(&cp->c[7]) * pw * exp(-u) - 2.0 * Mr3);
      add_spherical(dpr, d2, x, y, z, r2, gR, gz, K);
      break;
    }
    case T_NFW: {
      const double a = ldg(&cp->c[1]);
      const double ir = rsq(r2), r = r2 * ir;
      const double L = log1p(r * ldg(&cp->c[2]));
      const double iar = 1.0 / (a + r);
      const double dpr = amp * (L * ir - iar) * ir * ir;  // Phi'/r
      const double d2 = amp * (r * (2.0 * a + 3.0 * r) * iar * iar - 2.0 * L) * ir * ir * ir;
      add_spherical(dpr, d2, x, y, z, r2, gR, gz, K);
      break;
    }
    case T_HERNQUIST: {
      const double a = ldg(&cp->c[1]);
      const double ir = rsq(r2), r = r2 * ir;
      const double ira = 1.0 / (r + a);
      const double dpr = 0.5 * amp * ir * ira * ira;  // Phi'/r
      const double d2 = -amp * ira * ira * ira;       // Phi''
      add_spherical(dpr, d2, x, y, z, r2, gR, gz, K);
      break;
    }
    case T_MN: {
      // Phi = -amp (R^2 + s^2)^-1/2, s = a + zeta, zeta = sqrt(z^2 + b^2)
      const double a = ldg(&cp->c[1]);
      const double zb2 = z2 + ldg(&cp->c[2]);
      const double izb = rsq(zb2), zeta = zb2 * izb, s = a + zeta;
      const double iD = rsq(R2 + s * s), iD3 = iD * iD * iD, iD5 = iD3 * iD * iD;
      const double sz = s * izb;  // s / zeta
      gR -= amp * iD3;
      gz -= amp * sz * iD3;
      K[0] -= amp * (iD3 - 3.0 * x * x * iD5);
      K[1] += 3.0 * amp * x * y * iD5;
      K[2] -= amp * (iD3 - 3.0 * y * y * iD5);
      K[3] += 3.0 * amp * x * z * sz * iD5;
      K[4] += 3.0 * amp * y * z * sz * iD5;
      // d2Phi/dz2 = amp [ iD3 (s/zeta - a z^2/zeta^3) - 3 z^2 (s/zeta)^2 iD5 ]
      K[5] -= amp * (iD3 * (sz - a * z2 * izb * izb * izb) - 3.0 * z2 * sz * sz * iD5);
      break;
    }
    case T_KKS: {
      // Phi_R / R, Phi_RR, Phi_zz, Phi_Rz in (l, n) by the chain rule
      // (KuzminKutuzovStaeckelPotential.c R2deriv / z2deriv / Rzderiv),
      // then the axisymmetric Cartesian Hessian
      const double D2 = ldg(&cp->c[1]);
      const KksParts k = kks_parts(D2, ldg(&cp->c[2]), R2, z2);
      const double r2 = R2 + z2, rzp = r2 + D2, rzm = r2 - D2, isd = k.isd;
      const double id = isd * isd, id15 = isd * id;
      const double isln3 = k.isln2 / (k.srl + k.srn);
      const double d2l = (-3.0 * k.srl - k.srn) / (4.0 * k.l * k.srl) * isln3;
      const double d2n = (-k.srl - 3.0 * k.srn) / (4.0 * k.n * k.srn) * isln3;
      const double d2ln = -0.5 / (k.srl * k.srn) * isln3;
      // first derivatives per unit R (resp. z) of l and n
      const double lR = 1.0 + rzp * isd, nR = 1.0 - rzp * isd;
      const double lz = 1.0 + rzm * isd, nz = 1.0 - rzm * isd;
      const double gRk = -amp * (lR * k.dVdl + nR * k.dVdn);  // a_R / R
      const double gzk = -amp * (lz * k.dVdl + nz * k.dVdn);  // a_z / z
      const double offR = (3.0 * R2 + z2 + D2) * isd, cubR = 2.0 * R2 * rzp * rzp * id15;
      const double offz = (R2 + 3.0 * z2 - D2) * isd, cubz = 2.0 * z2 * rzm * rzm * id15;
      const double PRR = amp * ((1.0 + offR - cubR) * k.dVdl + (1.0 - offR + cubR) * k.dVdn +
                                R2 * (lR * lR * d2l + nR * nR * d2n + 2.0 * lR * nR * d2ln));
      const double Pzz = amp * ((1.0 + offz - cubz) * k.dVdl + (1.0 - offz + cubz) * k.dVdn +
                                z2 * (lz * lz * d2l + nz * nz * d2n + 2.0 * lz * nz * d2ln));
      const double mixRz = 2.0 * isd * (1.0 - (r2 * r2 - D2 * D2) * id);  // / (R z)
      const double PRz_Rz = amp * (mixRz * (k.dVdl - k.dVdn) + lR * lz * d2l + nR * nz * d2n +
                                   (lR * nz + lz * nR) * d2ln);  // Phi_Rz / (R z)
      const double PR_R = -gRk;
      gR += gRk;
      gz += gzk;
      const double iR2 = R2 > 0.0 ? 1.0 / R2 : 0.0;
      K[0] -= PRR * x * x * iR2 + PR_R * y * y * iR2;
      K[1] -= (PRR - PR_R) * x * y * iR2;
      K[2] -= PRR * y * y * iR2 + PR_R * x * x * iR2;
      K[3] -= PRz_Rz * x * z;
      K[4] -= PRz_Rz * y * z;
      K[5] -= Pzz;
      break;
    }
    case T_FLATPOWER: {  // the logarithmic halo's structure with weight (alpha+2) m2^(-alpha/2-2)
      const double iq2 = ldg(&cp->c[1]);
      const double m2 = R2 + z2 * iq2 + ldg(&cp->c[2]);
      const double pw = exp(ldg(&cp->c[3]) * log(m2)), g = -amp * pw;
      const double h = amp * ldg(&cp->c[5]) * pw / m2;
      const double ux = x, uy = y, uz = iq2 * z;
      gR += g;
      gz += g * iq2;
      K[0] += g + h * ux * ux;
      K[1] += h * ux * uy;
      K[2] += g + h * uy * uy;
      K[3] += h * ux * uz;
      K[4] += h * uy * uz;
      K[5] += g * iq2 + h * uz * uz;
      break;
    }
    case T_LOGHALO: {
      const double iq2 = ldg(&cp->c[1]), ye = ldg(&cp->c[3]);
      const double D = x * x + ye * y * y + z2 * iq2 + ldg(&cp->c[2]);
      const double iDl = 1.0 / D, g = -amp * iDl;
      const double ux = x, uy = ye * y, uz = iq2 * z;  // grad of D / 2
      gR += g;
      gyx += g * (ye - 1.0);
      gz += g * iq2;
      const double h = 2.0 * amp * iDl * iDl;
      K[0] += g + h * ux * ux;
      K[1] += h * ux * uy;
      K[2] += g * ye + h * uy * uy;
      K[3] += h * ux * uz;
      K[4] += h * uy * uz;
      K[5] += g * iq2 + h * uz * uz;
      break;
    }
    case T_HENONHEILES: {  // planar only; K = -amp ((1 + 2y, 2x), (2x, 1 - 2y))
      gR -= amp * (1.0 + 2.0 * y);
      gyx += 3.0 * amp * y;
      ay0 -= amp * x * x;
      K[0] -= amp * (1.0 + 2.0 * y);
      K[1] -= 2.0 * amp * x;
      K[2] -= amp * (1.0 - 2.0 * y);
      break;
    }
    case T_KUZMINDISK: {  // Cartesian Hessian of -amp D^(-1/2), D = x^2 + y^2 + (a + |z|)^2
      const double zs = (z > 0.0) - (z < 0.0), az = ldg(&cp->c[1]) + fabs(z);
      const double D = R2 + az * az, iD = rsq(D), d15 = iD * iD * iD, d25 = d15 / D;
      gR -= amp * d15;
      az0 -= zs * amp * d15 * az;
      if (PLANAR) {
        // the reference's planar second derivative (KuzminDiskPotential.c,
        // PlanarR2deriv) is amp (-D^(-3/2) + 3 R^2 D^(-5/2)), the opposite
        // sign of d^2 Phi / dR^2 of its planar potential; planar
        // variational runs follow it: K = -(Phi_RR c^2 + Phi_R/R s^2, ...)
        const double PRR = -amp * (d15 - 3.0 * R2 * d25), PR_R = amp * d15;
        const double iR2 = R2 > 0.0 ? 1.0 / R2 : 0.0;
        K[0] -= (PRR * x * x + PR_R * y * y) * iR2;
        K[1] -= (PRR - PR_R) * x * y * iR2;
        K[2] -= (PRR * y * y + PR_R * x * x) * iR2;
        break;
      }
      K[0] -= amp * (d15 - 3.0 * x * x * d25);
      K[1] += 3.0 * amp * x * y * d25;
      K[2] -= amp * (d15 - 3.0 * y * y * d25);
      K[3] += 3.0 * amp * x * az * zs * d25;
      K[4] += 3.0 * amp * y * az * zs * d25;
      K[5] -= amp * (d15 - 3.0 * az * az * d25);
      break;
    }
    case T_PAYLOAD:
      break;
    case T_DEHNENBAR:
      dbar_tidal<PLANAR>(cp, t, x, y, z, ax0, ay0, az0, K);
      break;
    case T_NEEDLEBAR:
      needle_accel<PLANAR>(cp, t, x, y, z, ax0, ay0, az0, K);
      break;
    case T_SCF:
      scf_tidal<PLANAR>(cp, x, y, z, ax0, ay0, az0, K);
      break;
    case T_TRANSPIRAL: case T_STEADYSPIRAL: case T_ELLDISK: case T_LOPSIDED: case T_COSMPHI:
      if (PLANAR)
        disk_pert_accel(cp, type, x, y, t, ax0, ay0, K);
      else
        gR = NAN;
      break;
    case T_SPIRALARMS:
      spiral_accel<PLANAR>(cp, x, y, z, t, ax0, ay0, az0, K);
      break;
    case T_TRIHERNQUIST: case T_TRINFW: case T_TRIJAFFE: case T_PERFECTELL: case T_TRIGAUSS:
    case T_POWERTRI: case T_TWOPOWERTRI: {
      double fx, fy, fz;
      ell_accel(cp, type, x, y, z, fx, fy, fz);
      ax0 += fx;
      ay0 += fy;
      az0 += fz;
      ell_tidal(cp, type, x, y, z, K);
      break;
    }
    default: {
      double dpr, d2;  // Phi'/r, Phi''
      sph_derivs(cp, type, amp, r2, dpr, d2);
      add_spherical(dpr, d2, x, y, z, r2, gR, gz, K);
      break;
    }
  }
}

template <bool PLANAR>
GPC_HD GPC_FI void accel_tidal(const GpComp* __restrict__ comp, int ncomp, double x, double y,
                               double z, double& ax, double& ay, double& az, double K[6],
                               double t = 0.0)
{
  if (PLANAR) z = 0.0;
  const double R2 = x * x + y * y, z2 = z * z, r2 = R2 + z2;
  double gR = 0.0, gz = 0.0, gyx = 0.0, ax0 = 0.0, ay0 = 0.0, az0 = 0.0;
#pragma unroll
  for (int i = 0; i < 6; i++) K[i] = 0.0;
  // wrapper frames as in DynPot::sum; K of the wrapped records, taken in the
  // rotated frame, returns as fac R(alpha) K' R(alpha)^T
  int wend = -1;
  double xw = x, yw = y, zw = z, z2w = z2, R2w = R2, r2w = r2;
  double sR = 0.0, sz = 0.0, syx = 0.0, sx0 = 0.0, sy0 = 0.0, sz0 = 0.0, sK[6];
  WrapFrame fr{1.0, 1.0, 0.0, false, false, 0.0, 0.0, 0.0};
  for (int k = 0; k <= ncomp; k++) {
    if (k == wend) {
      const double c = fr.c, s = fr.s, f = fr.fac;
      const double axw = xw * gR + ax0, ayw = yw * (gR + gyx) + ay0, azw = zw * gz + az0;
      gR = sR;
      gz = sz;
      gyx = syx;
      if (fr.kz) {
        // Phi = fac f(xi): -Hessian = fac (K'_xx g g^T + a'_x grad grad xi),
        // g = grad xi = (x, y, q) / xi, grad grad xi = (I' - g g^T) / xi with
        // I' = diag(1, 1, dq)
        const double ix = 1.0 / fr.xi, gx = x * ix, gy = y * ix, gz3 = fr.q * ix;
        const double kp = K[0], ap = axw * ix;
        ax0 = sx0 + f * axw * gx;
        ay0 = sy0 + f * axw * gy;
        az0 = sz0 + (PLANAR ? 0.0 : f * axw * gz3);
        K[0] = sK[0] + f * ((kp - ap) * gx * gx + ap);
        K[1] = sK[1] + f * (kp - ap) * gx * gy;
        K[2] = sK[2] + f * ((kp - ap) * gy * gy + ap);
        K[3] = sK[3] + f * (kp - ap) * gx * gz3;
        K[4] = sK[4] + f * (kp - ap) * gy * gz3;
        K[5] = sK[5] + f * ((kp - ap) * gz3 * gz3 + ap * fr.dq);
      } else {
        ax0 = sx0 + f * (c * axw - s * ayw);
        ay0 = sy0 + f * (s * axw + c * ayw);
        az0 = sz0 + (PLANAR ? 0.0 : f * azw);
        const double kxx = K[0], kxy = K[1], kyy = K[2], kxz = K[3], kyz = K[4], kzz = K[5];
        K[0] = sK[0] + f * (c * c * kxx - 2.0 * c * s * kxy + s * s * kyy);
        K[1] = sK[1] + f * (c * s * (kxx - kyy) + (c * c - s * s) * kxy);
        K[2] = sK[2] + f * (s * s * kxx + 2.0 * c * s * kxy + c * c * kyy);
        K[3] = sK[3] + f * (c * kxz - s * kyz);
        K[4] = sK[4] + f * (s * kxz + c * kyz);
        K[5] = sK[5] + f * kzz;
        if (fr.co) {
          // Phi = fac Phi'(R(-alpha) x), alpha = alpha(R): with tau' = -dPhi'/dphi',
          // u = R(alpha) grad'(dPhi'/dphi'), P2 = d2Phi'/dphi'2 and g = grad alpha,
          // -Hessian gains fac (u g^T + g u^T - P2 g g^T - tau' grad grad alpha),
          // grad grad alpha = (alpha'' - alpha'/R) R^ R^T + (alpha'/R) I_2; the
          // acceleration gains -fac tau' g.  Primed Hessian H' = -K'.
          const double hxx = -kxx, hxy = -kxy, hyy = -kyy, hxz = -kxz, hyz = -kyz;
          const double px = -axw, py = -ayw, tq = xw * ayw - yw * axw;
          const double ux = py + xw * hxy - yw * hxx, uy = xw * hyy - px - yw * hxy;
          const double uz = xw * hyz - yw * hxz;
          const double P2 = xw * xw * hyy - 2.0 * xw * yw * hxy + yw * yw * hxx - xw * px - yw * py;
          const double uix = c * ux - s * uy, uiy = s * ux + c * uy;
          const double gx = fr.q * x, gy = fr.q * y, iR2 = 1.0 / R2, e = fr.dq - fr.q;
          ax0 -= f * tq * gx;
          ay0 -= f * tq * gy;
          K[0] += f * (2.0 * uix * gx - P2 * gx * gx - tq * (e * x * x * iR2 + fr.q));
          K[1] += f * (uix * gy + uiy * gx - P2 * gx * gy - tq * e * x * y * iR2);
          K[2] += f * (2.0 * uiy * gy - P2 * gy * gy - tq * (e * y * y * iR2 + fr.q));
          K[3] += f * uz * gx;
          K[4] += f * uz * gy;
        }
      }
      xw = x;
      yw = y;
      zw = z;
      z2w = z2;
      R2w = R2;
      r2w = r2;
      wend = -1;
    }
    if (k == ncomp) break;
    const GpComp* cp = comp + k;
    const int type = ldg(&cp->type);
    if (is_wrapper(type)) {
      fr = wrap_frame(cp, type, t);
      wend = k + 1 + (int)ldg(&cp->c[15]);
      sR = gR;
      sz = gz;
      syx = gyx;
      sx0 = ax0;
      sy0 = ay0;
      sz0 = az0;
#pragma unroll
      for (int i = 0; i < 6; i++) {
        sK[i] = K[i];
        K[i] = 0.0;
      }
      gR = gz = gyx = ax0 = ay0 = az0 = 0.0;
      if (fr.kz) {
        kuzmin_map<PLANAR>(cp, R2, z, fr);
        xw = fr.xi;
        yw = zw = z2w = 0.0;
        R2w = r2w = xw * xw;
      } else {
        if (fr.co) corot_map(cp, R2, t, fr);
        xw = fr.c * x + fr.s * y;
        yw = fr.c * y - fr.s * x;
      }
      continue;
    }
    comp_tidal<PLANAR>(cp, type, xw, yw, zw, R2w, z2w, r2w, gR, gz, gyx, ax0, ay0, az0, K, t);
  }
  ax = x * gR + ax0;
  ay = y * (gR + gyx) + ay0;
  az = PLANAR ? 0.0 : z * gz + az0;
}

// -------------------------------------------------- potential values ---
// Potential of the spherical potentials at r^2 (0 for Null, whose constant
// value galpy adds on the Python side only).
GPC_HD inline double sph_value(const GpComp* __restrict__ cp, int type, double amp, double r2)
{
  const double r = sqrt(r2), c1 = ldg(&cp->c[1]);
  switch (type) {
    case T_POWER: {
      const double alpha = ldg(&cp->c[3]);
      if (alpha == 2.0) return 0.5 * amp * log(r2);
      return -amp * pow(r2, 1.0 - 0.5 * alpha) / (alpha - 2.0);
    }
    case T_JAFFE: return -amp * log1p(c1 / r) / c1;
    case T_ISOCHRONE: return -amp / (c1 + sqrt(r2 + ldg(&cp->c[2])));
    case T_PLUMMER: return -amp / sqrt(r2 + c1);
    case T_PSEUDOISO: return amp * (0.5 * log1p(r2 / (c1 * c1)) + c1 / r * atan(r / c1)) / c1;
    case T_BURKERT: {
      const double x = r / c1;
      return -amp * c1 * c1 * M_PI / x *
             (-M_PI + 2.0 * (1.0 + x) * atan(1.0 / x) + 2.0 * (1.0 + x) * log1p(x) +
              (1.0 - x) * log1p(x * x));
    }
    case T_DEHNENCORE: {
      const double u = r / (r + c1);
      return -amp * (1.0 - u * u) / (6.0 * c1);
    }
    case T_DEHNEN: {
      const double alpha = ldg(&cp->c[2]);
      return -amp * (1.0 - pow(r / (r + c1), 2.0 - alpha)) / (c1 * (2.0 - alpha) * (3.0 - alpha));
    }
    case T_HOMSPHERE:
      return r2 < c1 ? amp * (r2 - 3.0 * c1) : -2.0 * amp * ldg(&cp->c[2]) / r;
    case T_EXPTRUNCNFW: {  // -amp (F / r + e^(-r/rc) / (a + r) - e^alpha E1(beta) / rc)
      const double irc = ldg(&cp->c[2]);
      const double G = exp(-r * irc) / (c1 + r) - ldg(&cp->c[10]) * expint_E1((c1 + r) * irc);
      return -amp * (exptruncnfw_F(ScalarsGlobal{cp}, r) / r + G);
    }
    case T_EINASTO: {  // -amp 4 pi h^2 n [Gamma(3n) P(3n, x) / s + Gamma(2n) Q(2n, x)]
      const double s = r / c1, x = pow(s, ldg(&cp->c[2]));
      const double P3 = inc_gamma_P(ldg(&cp->c[3]), x, ldg(&cp->c[4]));
      const double Q2 = 1.0 - inc_gamma_P(ldg(&cp->c[7]), x, ldg(&cp->c[8]));
      return -amp * (ldg(&cp->c[6]) * c1 * c1 * P3 / s + ldg(&cp->c[9]) * Q2);
    }
    default:
      return 0.0;
  }
}

// Phi of an ellipsoidal component: -amp/2 sum_k w_k psi(m_k) in the
// rotated frame (EllipsoidalPotentialEval), psi of each density:
// TriaxialHernquist -a^4/(m+a)^2, TriaxialNFW -2 a^3/(m+a), TriaxialJaffe
// 2 a^2 (a/(m+a) + ln(m/(m+a))), PerfectEllipsoid -1/(a^2+m^2),
// TriaxialGaussian s e^(m^2/s) (s = -2 sigma^2), PowerTriaxial
// 2/(2-alpha) m^(2-alpha).
GPC_HD inline double ell_value(const GpComp* __restrict__ cp, int type, double x, double y,
                               double z)
{
  const double* rot = &cp->bin[0][0];
  if (ldg(&cp->c[6]) != 0.0) {
    const double xr = ldg(rot + 0) * x + ldg(rot + 1) * y + ldg(rot + 2) * z;
    const double yr = ldg(rot + 3) * x + ldg(rot + 4) * y + ldg(rot + 5) * z;
    const double zr = ldg(rot + 6) * x + ldg(rot + 7) * y + ldg(rot + 8) * z;
    x = xr;
    y = yr;
    z = zr;
  }
  const int n = (int)ldg(&cp->c[5]);
  const double* nd = &cp->cheb[0][0];
  const double p1 = ldg(&cp->c[1]), p2 = ldg(&cp->c[2]);
  double out = 0.0;
  for (int k = 0; k < n; k++, nd += 4) {
    const double m2 = x * x * ldg(nd + 1) + y * y * ldg(nd + 2) + z * z * ldg(nd + 3);
    const double m = sqrt(m2);
    double psi;
    switch (type) {
      case T_TRIHERNQUIST: psi = -p2 / ((m + p1) * (m + p1)); break;
      case T_TRINFW: psi = -2.0 * p2 / (m + p1); break;
      case T_TRIJAFFE: psi = 2.0 * p2 * (p1 / (m + p1) + log(m / (m + p1))); break;
      case T_PERFECTELL: psi = -1.0 / (p1 + m2); break;
      case T_TRIGAUSS: psi = p1 * exp(m2 / p1); break;
      default: psi = 2.0 / (2.0 - p1) * pow(m2, 1.0 - 0.5 * p1); break;  // PowerTriaxial
    }
    out += ldg(nd) * psi;
  }
  return -0.5 * ldg(&cp->c[0]) * out;
}

// Potential Phi(x, y, z) summed over one group's components, FP64
// (the *PotentialEval functions of potential_c_ext/*.c).
// One component's potential at (x, y, z) (wrappers are opened by
// potential_value).
GPC_HD inline double comp_value(const GpComp* __restrict__ cp, double x, double y, double z,
                                double R2, double z2, double r2)
{
  const double amp = ldg(&cp->c[0]);
  double phi = 0.0;
  switch (ldg(&cp->type)) {
    case T_PSWC: {
      // amp 2 pi rc^(3-alpha) / r [ r/rc gamma(a1, u) - gamma(a2, u) ]
      const double r = sqrt(r2), u = r2 * ldg(&cp->c[1]);
      const double a1 = ldg(&cp->c[10]), a2 = ldg(&cp->c[13]);
      const double g1 = ldg(&cp->c[11]) * inc_gamma_P(a1, u, ldg(&cp->c[12]));
      const double g2 = ldg(&cp->c[14]) * inc_gamma_P(a2, u, ldg(&cp->c[15]));
      phi += amp * ldg(&cp->c[8]) / r * (r / ldg(&cp->c[9]) * g1 - g2);
      break;
    }
    case T_MN: {
      const double s = ldg(&cp->c[1]) + sqrt(z2 + ldg(&cp->c[2]));
      phi -= amp / sqrt(R2 + s * s);
      break;
    }
    case T_NFW: {
      const double r = sqrt(r2);
      phi -= amp * log1p(r * ldg(&cp->c[2])) / r;
      break;
    }
    case T_HERNQUIST: {
      phi -= amp / (2.0 * (sqrt(r2) + ldg(&cp->c[1])));
      break;
    }
    case T_LOGHALO: {
      const double D = x * x + ldg(&cp->c[3]) * y * y + z2 * ldg(&cp->c[1]) + ldg(&cp->c[2]);
      phi += 0.5 * amp * log(D);
      break;
    }
    case T_KKS: {  // n clipped at 0 as the reference's Eval does
      const double D2 = ldg(&cp->c[1]), r2 = R2 + z2, rzm = r2 - D2;
      const double sd = sqrt(rzm * rzm + 4.0 * D2 * R2);
      const double l = 0.5 * (r2 - ldg(&cp->c[2]) + sd), n = 0.5 * (r2 - ldg(&cp->c[2]) - sd);
      phi -= amp / (sqrt(l) + sqrt(n > 0.0 ? n : 0.0));
      break;
    }
    case T_FLATPOWER: {
      const double m2 = R2 + z2 * ldg(&cp->c[1]) + ldg(&cp->c[2]), alpha = ldg(&cp->c[4]);
      phi += alpha == 0.0 ? 0.5 * amp * log(m2) : -amp * pow(m2, -0.5 * alpha) / alpha;
      break;
    }
    case T_HENONHEILES:  // amp (R^2/2 + R^3 sin(3 phi)/3)
      phi += amp * (0.5 * R2 + x * x * y - y * y * y / 3.0);
      break;
    case T_KUZMINDISK: {
      const double az = ldg(&cp->c[1]) + fabs(z);
      phi -= amp / sqrt(R2 + az * az);
      break;
    }
    case T_TRIHERNQUIST: case T_TRINFW: case T_TRIJAFFE: case T_PERFECTELL: case T_TRIGAUSS:
    case T_POWERTRI:
      phi += ell_value(cp, ldg(&cp->type), x, y, z);
      break;
    case T_TWOPOWERTRI:  // psi needs the Gauss hypergeometric function 2F1: not carried
      phi += NAN;
      break;
    case T_PAYLOAD:
      break;
    case T_SCF: {
      double ax, ay, az, p;
      scf_accel<false>(cp, x, y, z, ax, ay, az, &p);
      phi += p;
      break;
    }
    case T_SPIRALARMS:  // at t = 0 (time-dependent: the hooks keep galpy's path)
      phi += spiral_potential<false>(cp, sqrt(R2), z, atan2(y, x), 0.0).v;
      break;
    case T_NEEDLEBAR:  // at t = 0, likewise
      phi += needle_value(cp, 0.0, x, y, z);
      break;
    case T_TRANSPIRAL: case T_STEADYSPIRAL: case T_ELLDISK: case T_LOPSIDED: case T_COSMPHI:
    case T_DEHNENBAR:  // no evaluation in the reference's C (the hooks keep galpy's)
      phi += NAN;
      break;
    default:
      phi += sph_value(cp, ldg(&cp->type), amp, r2);
      break;
  }
  return phi;
}

// Potential summed over one group's records; a wrapper scales the sum over
// the records it wraps (evaluated at t = 0 as the reference's potential
// evaluation does; the rotation wrapper has none: NaN).
GPC_HD inline double potential_value(const GpComp* __restrict__ comp, int ncomp, double x,
                                     double y, double z)
{
  const double R2 = x * x + y * y, z2 = z * z, r2 = R2 + z2;
  double phi = 0.0;
  for (int k = 0; k < ncomp; k++) {
    const GpComp* cp = comp + k;
    const int type = ldg(&cp->type);
    if (is_wrapper(type)) {
      const int nw = (int)ldg(&cp->c[15]);
      WrapFrame fr = wrap_frame(cp, type, 0.0);
      double w = 0.0;
      if (fr.kz) {  // the wrapped list at (xi, 0, 0)
        kuzmin_map<false>(cp, R2, z, fr);
        const double xi2 = fr.xi * fr.xi;
        for (int j = 1; j <= nw; j++) w += comp_value(cp + j, fr.xi, 0.0, 0.0, xi2, 0.0, xi2);
      } else {
        for (int j = 1; j <= nw; j++) w += comp_value(cp + j, x, y, z, R2, z2, r2);
      }
      phi += type == T_WRAP_ROTATE || type == T_WRAP_COROT ? NAN : fr.fac * w;
      k += nw;
      continue;
    }
    phi += comp_value(cp, x, y, z, R2, z2, r2);
  }
  return phi;
}

}  // namespace gpc
