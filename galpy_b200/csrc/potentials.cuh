// galpy_b200/csrc/potentials.cuh
//
// Device-side forces and tidal tensors of the potentials the engine supports:
// PowerSphericalPotentialwCutoff (galpy type 15), MiyamotoNagaiPotential (5),
// NFWPotential (9), HernquistPotential (8) and LogarithmicHaloPotential (0,
// axisymmetric or triaxial).  Reference formulas:
// galpy/potential/potential_c_ext/{PowerSphericalPotentialwCutoff,
// MiyamotoNagaiPotential,NFWPotential,HernquistPotential,
// LogarithmicHaloPotential}.c.
//
// Design (not a translation of the reference's cylindrical route):
//  * Every component is evaluated directly in Cartesian coordinates.  The
//    axisymmetric terms are written as a_i = x_i * g(R, z), so neither
//    R = sqrt(x^2+y^2), acos(x/R), nor the 1/R conversions of
//    evalRectForce (integrateFullOrbit.c:1307-1325) are needed.
//  * The host compiles galpy's (pot_type, pot_args) once into GpComp records
//    holding the derived constants (1/rc^2, Gamma(a), b^2, 1/a ...), so no
//    per-evaluation tgamma/pow(rc, 3-alpha) as in
//    PowerSphericalPotentialwCutoff.c:10.
//  * One component list per potential group; a launch may hold many groups
//    (ragged multi-potential batches).  The component loop is warp-uniform
//    whenever the lanes of a warp integrate orbits of the same group.
//  * The Cartesian tidal tensor K = -grad grad Phi (for variational and
//    adjoint integration) is built from each component's own radial /
//    meridional derivatives, equal to the reference's cylindrical-to-
//    Cartesian assembly (integrateFullOrbit.c:1570-1596).
//  * The regularised incomplete gamma function of the bulge mass is this
//    project's own implementation of the published series (Abramowitz &
//    Stegun 6.5.29) and Legendre continued fraction (A&S 6.5.31, modified
//    Lentz evaluation), with host-precomputed reciprocals 1/(a+n) so the
//    series needs no division.
#pragma once
#include "gpc_common.cuh"

namespace gpc {

enum : int { T_LOGHALO = 0, T_MN = 5, T_HERNQUIST = 8, T_NFW = 9, T_PSWC = 15 };

constexpr int kMaxComp = 16;      // components per potential group
constexpr int kSeriesTerms = 48;  // tabulated 1/(a+n), n = 1..kSeriesTerms

// One compiled potential component: 8 scalars + the series table.  The
// meaning of c[] depends on the type (see compile_potential in the host code):
//   PSwC:      c0 amp, c1 1/rc^2, c2 a = 1.5 - alpha/2, c3 lgamma(a),
//              c4 Mnorm = 2 pi rc^(3-alpha) Gamma(a), c5 -alpha/2,
//              c6 4 pi, c7 alpha
//   MN:        c0 amp, c1 a, c2 b^2
//   Hernquist: c0 amp, c1 a, c2 1/a
//   NFW:       c0 amp, c1 a, c2 1/a
//   LogHalo:   c0 amp, c1 1/q^2, c2 core^2, c3 1 - e (y-axis factor; 1 when
//              axisymmetric), c4 triaxial flag
struct GpComp {
  int type;
  int pad;
  double c[8];
  double inv_ap[kSeriesTerms];  // PSwC: 1/(a+n), n = 1..kSeriesTerms
};

// ---------------------------------------------------------------- math ---
template <typename T> struct Num;
template <> struct Num<double> {
  GPC_HD static double eps() { return 1.0e-16; }
  GPC_HD static double tiny() { return 1.0e-300; }
  GPC_HD static double lg(double x) { return log(x); }
  GPC_HD static double ex(double x) { return exp(x); }
  GPC_HD static double lg1p(double x) { return log1p(x); }
  GPC_HD static double rsq(double x) { return gpc::rsq(x); }
  GPC_HD static double rcp(double x) { return 1.0 / x; }
  GPC_HD static int maxit() { return 400; }
};
// FP32 evaluation: hardware approximations (SFU) for log/exp/rsqrt/rcp.
template <> struct Num<float> {
  GPC_HD static float eps() { return 6.0e-8f; }
  GPC_HD static float tiny() { return 1.0e-37f; }
#if defined(__CUDA_ARCH__)
  __device__ static float lg(float x) { return __logf(x); }
  __device__ static float ex(float x) { return __expf(x); }
  __device__ static float rcp(float x) { return __frcp_rn(x); }
#else
  static float lg(float x) { return logf(x); }
  static float ex(float x) { return expf(x); }
  static float rcp(float x) { return 1.0f / x; }
#endif
  GPC_HD static float lg1p(float x) { return log1pf(x); }
  GPC_HD static float rsq(float x) { return gpc::rsqf(x); }
  GPC_HD static int maxit() { return 200; }
};

// Regularised lower incomplete gamma P(a, x), a > 0, x >= 0 (see header).
// lga = lgamma(a); inv_ap[n-1] = 1/(a+n).
template <typename T>
GPC_HD GPC_FI T inc_gamma_P(T a, T x, T lga, const double* __restrict__ inv_ap)
{
  if (x <= T(0)) return T(0);
  const T lpref = a * Num<T>::lg(x) - x - lga;
  if (x < a + T(1)) {
    // series: P = pref * sum_n x^n / (a (a+1) ... (a+n))
    T term = Num<T>::rcp(a), sum = term;
    int n = 0;
    for (; n < kSeriesTerms; n++) {
      term *= x * T(ldg(inv_ap + n));
      sum += term;
      if (fabs(term) < fabs(sum) * Num<T>::eps()) break;
    }
    if (n == kSeriesTerms) {  // only for x very close to a+1 with large a
      T ap = a + T(kSeriesTerms);
      for (int m = 0; m < Num<T>::maxit(); m++) {
        ap += T(1);
        term *= x / ap;
        sum += term;
        if (fabs(term) < fabs(sum) * Num<T>::eps()) break;
      }
    }
    return sum * Num<T>::ex(lpref);
  }
  // continued fraction for Q, modified Lentz
  T b = x + T(1) - a, c = T(1) / Num<T>::tiny(), d = Num<T>::rcp(b), h = d;
  for (int i = 1; i < Num<T>::maxit(); i++) {
    const T an = -T(i) * (T(i) - a);
    b += T(2);
    d = an * d + b;
    if (fabs(d) < Num<T>::tiny()) d = Num<T>::tiny();
    c = b + an / c;
    if (fabs(c) < Num<T>::tiny()) c = Num<T>::tiny();
    d = Num<T>::rcp(d);
    const T del = d * c;
    h *= del;
    if (fabs(del - T(1)) < Num<T>::eps()) break;
  }
  return T(1) - Num<T>::ex(lpref) * h;
}

// ------------------------------------------------------------- forces ---
// Acceleration at (x, y, z) summed over one group's components; PLANAR
// evaluates galpy's planar potential (the 3D potential in the plane z = 0)
// and leaves az untouched.  T is the arithmetic type of the evaluation.
template <typename T, bool PLANAR>
GPC_HD GPC_FI void accel(const GpComp* __restrict__ comp, int ncomp, T x, T y, T z,
                                      T& ax, T& ay, T& az)
{
  const T R2 = x * x + y * y;
  const T z2 = PLANAR ? T(0) : z * z;
  const T r2 = R2 + z2;
  T gR = T(0), gz = T(0), gy_extra = T(0);
  for (int k = 0; k < ncomp; k++) {
    const GpComp* cp = comp + k;
    const int type = ldg(&cp->type);
    const T amp = T(ldg(&cp->c[0]));
    switch (type) {
      case T_PSWC: {
        // F = -amp M(r)/r^3 * r_vec, M(r) = Mnorm P(a, r^2/rc^2)
        const T a = T(ldg(&cp->c[2]));
        const T P = inc_gamma_P<T>(a, r2 * T(ldg(&cp->c[1])), T(ldg(&cp->c[3])), cp->inv_ap);
        const T ir = Num<T>::rsq(r2);
        const T f = -amp * T(ldg(&cp->c[4])) * P * (ir * ir * ir);
        gR += f;
        gz += f;
        break;
      }
      case T_MN: {
        const T a = T(ldg(&cp->c[1]));
        const T zb2 = z2 + T(ldg(&cp->c[2]));
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
        const T a = T(ldg(&cp->c[1]));
        const T ir = Num<T>::rsq(r2);
        const T r = r2 * ir;
        const T f = amp * ir * ir * (Num<T>::rcp(a + r) - Num<T>::lg1p(r * T(ldg(&cp->c[2]))) * ir);
        gR += f;
        gz += f;
        break;
      }
      case T_HERNQUIST: {
        // Phi = -amp / (2 (r + a)) ; F = -amp / (2 r (r + a)^2) r_vec
        const T a = T(ldg(&cp->c[1]));
        const T ir = Num<T>::rsq(r2);
        const T ira = Num<T>::rcp(r2 * ir + a);
        const T f = -T(0.5) * amp * ir * ira * ira;
        gR += f;
        gz += f;
        break;
      }
      case T_LOGHALO: {
        // Phi = amp/2 ln(x^2 + (1-e) y^2 + z^2/q^2 + core^2)
        const T iq2 = T(ldg(&cp->c[1]));
        const T ye = T(ldg(&cp->c[3]));
        const T D = x * x + ye * y * y + z2 * iq2 + T(ldg(&cp->c[2]));
        const T g = -amp * Num<T>::rcp(D);
        gR += g;
        gy_extra += g * (ye - T(1));
        if (!PLANAR) gz += g * iq2;
        break;
      }
      default:
        break;
    }
  }
  ax = x * gR;
  ay = y * (gR + gy_extra);
  if (!PLANAR) az = z * gz;
}

// ------------------------------------------------------ tidal tensor ---
// Acceleration and the symmetric Cartesian tidal tensor K = d a / d x
// (K[0]=xx, K[1]=xy, K[2]=yy, K[3]=xz, K[4]=yz, K[5]=zz), FP64.
// Spherical components use Phi'(r), Phi''(r):
//   K_ij = -(Phi'' - Phi'/r) x_i x_j / r^2 - Phi'/r delta_ij.
GPC_HD GPC_FI void add_spherical(double dphi_over_r, double d2phi, double x, double y,
                                              double z, double r2, double& gR, double& gz,
                                              double K[6])
{
  // dphi_over_r = Phi'/r, d2phi = Phi''
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

template <bool PLANAR>
GPC_HD GPC_FI void accel_tidal(const GpComp* __restrict__ comp, int ncomp, double x,
                                            double y, double z, double& ax, double& ay, double& az,
                                            double K[6])
{
  if (PLANAR) z = 0.0;
  const double R2 = x * x + y * y, z2 = z * z, r2 = R2 + z2;
  double gR = 0.0, gz = 0.0, gyx = 0.0;
#pragma unroll
  for (int i = 0; i < 6; i++) K[i] = 0.0;
  for (int k = 0; k < ncomp; k++) {
    const GpComp* cp = comp + k;
    const int type = ldg(&cp->type);
    const double amp = ldg(&cp->c[0]);
    switch (type) {
      case T_PSWC: {
        const double a = ldg(&cp->c[2]), irc2 = ldg(&cp->c[1]);
        const double P = inc_gamma_P<double>(a, r2 * irc2, ldg(&cp->c[3]), cp->inv_ap);
        const double ir = rsq(r2);
        const double M = ldg(&cp->c[4]) * P;
        const double dpr = amp * M * ir * ir * ir;  // Phi'/r = amp M / r^3
        // Phi'' = amp (4 pi r^-alpha exp(-r^2/rc^2) - 2 M / r^3)
        const double d2 = amp * (ldg(&cp->c[6]) * pow(r2, ldg(&cp->c[5])) * exp(-r2 * irc2) -
                                 2.0 * M * ir * ir * ir);
        add_spherical(dpr, d2, x, y, z, r2, gR, gz, K);
        break;
      }
      case T_NFW: {
        const double a = ldg(&cp->c[1]);
        const double ir = rsq(r2), r = r2 * ir;
        const double L = log1p(r * ldg(&cp->c[2]));
        const double iar = 1.0 / (a + r);
        const double dpr = amp * (L * ir - iar) * ir * ir;                      // Phi'/r
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
        // dPhi/dR = amp R iD3, dPhi/dz = amp z s/zeta iD3
        const double sz = s * izb;  // s / zeta
        gR -= amp * iD3;
        gz -= amp * sz * iD3;
        // d2Phi/dR2 = amp (iD3 - 3 R^2 iD5); with x_i/R factors:
        //   K_xx = -(amp iD3 - 3 amp x^2 iD5), K_xy = 3 amp x y iD5
        K[0] -= amp * (iD3 - 3.0 * x * x * iD5);
        K[1] += 3.0 * amp * x * y * iD5;
        K[2] -= amp * (iD3 - 3.0 * y * y * iD5);
        // d2Phi/dRdz = -3 amp R z s/zeta iD5  -> K_xz = 3 amp x z sz iD5
        K[3] += 3.0 * amp * x * z * sz * iD5;
        K[4] += 3.0 * amp * y * z * sz * iD5;
        // d2Phi/dz2 = amp [ iD3 (s/zeta - a z^2/zeta^3) - 3 z^2 sz^2 iD5 ]
        //   (d/dz (z s/zeta) = s/zeta + z d(s/zeta)/dz = s/zeta - a z^2/zeta^3)
        K[5] -= amp * (iD3 * (sz - a * z2 * izb * izb * izb) - 3.0 * z2 * sz * sz * iD5);
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
      default:
        break;
    }
  }
  ax = x * gR;
  ay = y * (gR + gyx);
  az = PLANAR ? 0.0 : z * gz;
}

}  // namespace gpc
