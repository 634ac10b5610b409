// galpy_b200/csrc/potentials_td.cuh
//
// Device forces of the time-dependent DehnenBarPotential (galpy type 1,
// potential_c_ext/DehnenBarPotential.c) and of the SCFPotential with static
// coefficients (type 24, potential_c_ext/SCFPotential.c), evaluated in
// Cartesian form.  Included by potentials.cuh; used by the full run-time
// component list only.
//
// DehnenBar.  Phi = A s(t) cos 2(phi - Omega t - phi_b) (R/r)^2 g(r), with
// g = (r/rb)^3 - 2 inside rb and -(rb/r)^3 outside, and s(t) the quintic
// growth factor between tform and tsteady.  Since R^2 cos 2(phi - B/2) =
// cB (x^2 - y^2) + 2 sB x y with B = 2 (Omega t + phi_b), the potential is
// A s h(r) Q(x, y): h = g / r^2 (r/rb^3 - 2/r^2 inside, -rb^3/r^5 outside)
// times a quadratic form -- no angle, no division by R, and its Cartesian
// gradient and Hessian follow in closed form.
//
// SCF.  Phi = sum_{n,l,m} (Acos cos m phi + Asin sin m phi) P_l^m(cos theta)
// phiTilde_nl(r), phiTilde_nl = -(a r)^l / (a + r)^(2l+1) C_n^(2l+3/2)(xi),
// xi = (r - a) / (r + a) (Hernquist & Ostriker 1992).  The sums run m
// outer, l inner, n innermost, each family by its three-term recurrence, so
// no array is held per thread: cos / sin m phi by the angle-addition
// recurrence from (x, y) / R; P_l^m and dP_l^m / dtheta upward in l from
// P_m^m = -(2m - 1) sin(theta) P_{m-1}^{m-1} (Condon-Shortley phase) and its
// theta derivative; C_n^alpha and C_n^(alpha+1) (dC_n^alpha / dxi = 2 alpha
// C_{n-1}^(alpha+1)) upward in n with the coefficients tabulated on the host.
#pragma once
#include <cstddef>

namespace gpc {

enum : int { T_DEHNENBAR = 1, T_SCF = 24 };
// Wrappers (DehnenSmoothWrapperPotential.c, SolidBodyRotationWrapperPotential.c,
// GaussianAmplitudeWrapperPotential.c): a wrapper record is followed by the
// records of the components it wraps (c15 holds their count).
// KuzminLikeWrapperPotential.c: the wrapped list on the plane at
// xi = sqrt(R^2 + (a + sqrt(z^2 + b^2))^2).
// CorotatingRotationWrapperPotential.c: the wrapped list rotated by
// alpha(R, t) = vpo R^(beta - 1) (t - to) + pa.
enum : int { T_WRAP_SMOOTH = -1, T_WRAP_ROTATE = -2, T_WRAP_COROT = -4, T_WRAP_GAUSS = -5,
             T_WRAP_KUZMIN = -10 };
GPC_HD GPC_FI constexpr bool is_wrapper(int t)
{
  return t == T_WRAP_SMOOTH || t == T_WRAP_ROTATE || t == T_WRAP_GAUSS || t == T_WRAP_KUZMIN ||
         t == T_WRAP_COROT;
}
// Planar-only disk perturbations: TransientLogSpiral, SteadyLogSpiral,
// EllipticalDisk, LopsidedDisk, CosmphiDisk (potential_c_ext/<name>.c)
enum : int { T_TRANSPIRAL = 2, T_STEADYSPIRAL = 3, T_ELLDISK = 4, T_LOPSIDED = 6,
             T_COSMPHI = 28 };
// SpiralArmsPotential (SpiralArmsPotential.c): 3D and planar
enum : int { T_SPIRALARMS = 27 };
constexpr int kSpiralMaxTerms = 6;  // Cn terms a record holds
// SoftenedNeedleBarPotential (SoftenedNeedleBarPotential.c): 3D and planar
enum : int { T_NEEDLEBAR = 25 };

GPC_HD GPC_FI constexpr bool is_disk_pert(int t)
{
  return t == T_TRANSPIRAL || t == T_STEADYSPIRAL || t == T_ELLDISK || t == T_LOPSIDED ||
         t == T_COSMPHI;
}
// Continuation record of a component whose data does not fit one record
// (an SCF expansion's coefficients): skipped by every component loop.
enum : int { T_PAYLOAD = -100 };

// Types that only the full run-time component list carries.
GPC_HD GPC_FI constexpr bool needs_full_list(int t)
{
  return is_ellipsoidal(t) || t == T_DEHNENBAR || t == T_SCF || t == T_PAYLOAD || is_wrapper(t) ||
         is_disk_pert(t) || t == T_SPIRALARMS || t == T_NEEDLEBAR;
}

// Doubles of payload per continuation record: the record after its
// (type, tab) header.
constexpr int kPayloadDoubles = (int)((sizeof(GpComp) - offsetof(GpComp, c)) / sizeof(double));
static_assert(offsetof(GpComp, c) == 8 && (sizeof(GpComp) - 8) % sizeof(double) == 0,
              "continuation records are read as a run of doubles");

// Payload value j of the component record cp (its continuation records
// follow it).
GPC_HD GPC_FI double payload(const GpComp* __restrict__ cp, int j)
{
  const int rec = j / kPayloadDoubles, off = j - rec * kPayloadDoubles;
  return ldg(&cp[1 + rec].c[0] + off);
}

// ---- DehnenBar ------------------------------------------------------------
// Record: c0 amp (galpy's amp * af), c1 tform, c2 tsteady, c3 rb, c4 omegab,
// c5 barphi, c6 rb^3, c7 1 / (tsteady - tform).
// Growth factor of the bar and of DehnenSmoothWrapper (dehnenBarSmooth,
// dehnenSmooth): 0 before tform, the quintic 3/16 xi^5 - 5/8 xi^3 + 15/16 xi
// + 1/2 of xi = 2 (t - tform) / (tsteady - tform) - 1 until tsteady, 1 after
// (inv: 1 / (tsteady - tform)).
GPC_HD GPC_FI double dehnen_smooth(double t, double tform, double tsteady, double inv)
{
  if (t < tform) return 0.0;
  if (t >= tsteady) return 1.0;
  const double xi = 2.0 * (t - tform) * inv - 1.0, x2 = xi * xi;
  return ((3.0 / 16.0 * x2 - 5.0 / 8.0) * x2 + 15.0 / 16.0) * xi + 0.5;
}

// A wrapper's effect at time t: the wrapped components' forces are scaled
// by fac and evaluated in a frame rotated by alpha (cos c, sin s): at
// phi - alpha, rotated back by alpha.  DehnenSmooth: fac = amp s(t) (1 - s
// when not growing); GaussianAmplitude: amp exp(-(t - to)^2 / (2 sigma^2));
// SolidBodyRotation: amp, alpha = omega t + pa.
// Records: c0 amp; smooth c1 tform, c2 tsteady, c3 grow, c4 1/(tsteady -
// tform); Gaussian c1 to, c2 sigma^2; rotation c1 omega, c2 pa.
// A wrapper's frame: its factor and, for the rotations, cos / sin of the
// angle; for KuzminLike (kz) the point map x -> (xi, 0, 0) with
// grad xi = (x, y, q) / xi, q = (a + zeta) z / zeta, zeta = sqrt(z^2 + b^2),
// and dq = dq/dz = 1 + a b^2 / zeta^3 (for the tidal tensor); for
// CorotatingRotation (co) the angle at the point's R, with q = alpha'(R) / R
// and dq = alpha''(R).
struct WrapFrame {
  double fac, c, s;
  bool kz, co;
  double xi, q, dq;
};

GPC_HD GPC_FI WrapFrame wrap_frame(const GpComp* __restrict__ cp, int type, double t)
{
  WrapFrame f{ldg(&cp->c[0]), 1.0, 0.0, false, false, 0.0, 0.0, 0.0};
  if (type == T_WRAP_KUZMIN) {
    f.kz = true;
  } else if (type == T_WRAP_COROT) {
    f.co = true;
  } else if (type == T_WRAP_SMOOTH) {
    const double sm = dehnen_smooth(t, ldg(&cp->c[1]), ldg(&cp->c[2]), ldg(&cp->c[4]));
    f.fac *= ldg(&cp->c[3]) != 0.0 ? sm : 1.0 - sm;
  } else if (type == T_WRAP_GAUSS) {
    const double d = t - ldg(&cp->c[1]);
    f.fac *= exp(-0.5 * d * d / ldg(&cp->c[2]));
  } else {
    sincos(ldg(&cp->c[1]) * t + ldg(&cp->c[2]), &f.s, &f.c);
  }
  return f;
}

// The KuzminLike point map at (R^2, z) (z = 0 in the plane).
template <bool PLANAR>
GPC_HD GPC_FI void kuzmin_map(const GpComp* __restrict__ cp, double R2, double z, WrapFrame& f)
{
  const double a = ldg(&cp->c[1]), b2 = ldg(&cp->c[2]);
  const double zeta = sqrt((PLANAR ? 0.0 : z * z) + b2), A = a + zeta;
  f.xi = sqrt(R2 + A * A);
  f.q = PLANAR ? 0.0 : A * z / zeta;
  f.dq = 1.0 + a * b2 / (zeta * zeta * zeta);
}

// The CorotatingRotation angle at R^2, time t (record c1 vpo, c2 beta,
// c3 pa, c4 to): alpha = w R^(beta-1) + pa, alpha'/R = w (beta-1) R^(beta-3),
// alpha'' = w (beta-1) (beta-2) R^(beta-3), w = vpo (t - to).
GPC_HD GPC_FI void corot_map(const GpComp* __restrict__ cp, double R2, double t, WrapFrame& f)
{
  const double beta = ldg(&cp->c[2]), w = ldg(&cp->c[1]) * (t - ldg(&cp->c[4]));
  const double Rb = pow(R2, 0.5 * (beta - 3.0));
  sincos(w * Rb * R2 + ldg(&cp->c[3]), &f.s, &f.c);
  f.q = w * (beta - 1.0) * Rb;
  f.dq = f.q * (beta - 2.0);
}

struct BarParts {
  double A;           // amp * s(t)
  double cB, sB;      // cos, sin of 2 (omegab t + barphi)
  double h, hp_r;     // h(r), h'(r) / r
  double hpp;         // h''(r)
};

GPC_HD GPC_FI BarParts dbar_parts(const GpComp* __restrict__ cp, double t, double r2)
{
  BarParts b;
  b.A = ldg(&cp->c[0]) * dehnen_smooth(t, ldg(&cp->c[1]), ldg(&cp->c[2]), ldg(&cp->c[7]));
  sincos(2.0 * (ldg(&cp->c[4]) * t + ldg(&cp->c[5])), &b.sB, &b.cB);
  const double rb = ldg(&cp->c[3]), rb3 = ldg(&cp->c[6]);
  const double ir2 = 1.0 / r2, ir = sqrt(ir2), ir4 = ir2 * ir2;
  if (r2 <= rb * rb) {
    const double r = r2 * ir;
    b.h = r / rb3 - 2.0 * ir2;
    b.hp_r = ir / rb3 + 4.0 * ir4;
    b.hpp = -12.0 * ir4;
  } else {
    const double ir5 = ir4 * ir;
    b.h = -rb3 * ir5;
    b.hp_r = 5.0 * rb3 * ir5 * ir2;
    b.hpp = -30.0 * rb3 * ir5 * ir2;
  }
  return b;
}

// Acceleration -grad Phi at time t (PLANAR: the 3D potential at z = 0).
template <bool PLANAR>
GPC_HD GPC_FI void dbar_accel(const GpComp* __restrict__ cp, double t, double x, double y,
                              double z, double& ax, double& ay, double& az)
{
  const double zz = PLANAR ? 0.0 : z;
  const BarParts b = dbar_parts(cp, t, x * x + y * y + zz * zz);
  const double Q = b.cB * (x * x - y * y) + 2.0 * b.sB * x * y;
  const double Qx = 2.0 * (b.cB * x + b.sB * y), Qy = 2.0 * (b.sB * x - b.cB * y);
  const double f = -b.A * b.hp_r * Q;
  ax = f * x - b.A * b.h * Qx;
  ay = f * y - b.A * b.h * Qy;
  az = PLANAR ? 0.0 : f * zz;
}

// Acceleration and K = -grad grad Phi (K[0] xx, 1 xy, 2 yy, 3 xz, 4 yz, 5 zz),
// added to ax.. and K.
template <bool PLANAR>
GPC_HD GPC_FI void dbar_tidal(const GpComp* __restrict__ cp, double t, double x, double y,
                              double z, double& ax, double& ay, double& az, double K[6])
{
  const double zz = PLANAR ? 0.0 : z;
  const double r2 = x * x + y * y + zz * zz;
  const BarParts b = dbar_parts(cp, t, r2);
  const double Q = b.cB * (x * x - y * y) + 2.0 * b.sB * x * y;
  const double Qx = 2.0 * (b.cB * x + b.sB * y), Qy = 2.0 * (b.sB * x - b.cB * y);
  const double f = -b.A * b.hp_r * Q;
  ax += f * x - b.A * b.h * Qx;
  ay += f * y - b.A * b.h * Qy;
  if (!PLANAR) az += f * zz;
  // Hessian: A [(h'' - h'/r) x_i x_j / r^2 Q + h'/r (delta_ij Q + x_i Q_j +
  // x_j Q_i) + h Q_ij], Q_xx = 2 cB, Q_xy = 2 sB, Q_yy = -2 cB
  const double c = b.A * (b.hpp - b.hp_r) * Q / r2, d = b.A * b.hp_r, e = b.A * b.h;
  const double dQ = d * Q;
  K[0] -= c * x * x + dQ + 2.0 * d * x * Qx + 2.0 * e * b.cB;
  K[1] -= c * x * y + d * (x * Qy + y * Qx) + 2.0 * e * b.sB;
  K[2] -= c * y * y + dQ + 2.0 * d * y * Qy - 2.0 * e * b.cB;
  if (!PLANAR) {
    K[3] -= c * x * zz + d * zz * Qx;
    K[4] -= c * y * zz + d * zz * Qy;
    K[5] -= c * zz * zz + dQ;
  }
}

// ---- planar disk perturbations ------------------------------------------
// Record: galpy's args in c0..c8 (TransientLogSpiral amp, A, to, sigma^2,
// alpha, m, omegas, gamma; SteadyLogSpiral amp, tform, tsteady, A, alpha, m,
// omegas, gamma; EllipticalDisk amp, tform, tsteady, twophio, p, phib;
// LopsidedDisk amp, phio, p, phib; CosmphiDisk amp, mphio, p, mphib, m, rb,
// rb^p, rb^2p, r1^p), c9 1 / (tsteady - tform).  Each is R-power (or log R)
// times a harmonic in phi; the parts below are -dPhi/dR (FR), -dPhi/dphi
// (tq) and the second derivatives (R2, p2, Rp), as the reference writes them.
struct CylParts {
  double FR, tq, R2, p2, Rp;
};

GPC_HD inline CylParts disk_pert_parts(const GpComp* __restrict__ cp, int type, double R,
                                       double phi, double t)
{
  double a[9];
#pragma unroll
  for (int k = 0; k < 9; k++) a[k] = ldg(&cp->c[k]);
  const double amp = a[0];
  CylParts P;
  if (type == T_TRANSPIRAL || type == T_STEADYSPIRAL) {
    double g, A, alpha, m, om, gam;
    if (type == T_TRANSPIRAL) {
      const double d = t - a[2];
      A = a[1];
      g = amp * A * exp(-0.5 * d * d / a[3]);
      alpha = a[4], m = a[5], om = a[6], gam = a[7];
    } else {  // tform NaN: always on
      A = a[3];
      const double sm = a[1] != a[1] ? 1.0 : dehnen_smooth(t, a[1], a[2], ldg(&cp->c[9]));
      g = amp * sm * A;
      alpha = a[4], m = a[5], om = a[6], gam = a[7];
    }
    double sc, cc;
    sincos(alpha * log(R) - m * (phi - om * t - gam), &sc, &cc);
    const double iR = 1.0 / R;
    P.FR = g * iR * sc;
    P.tq = -g / alpha * m * sc;
    P.R2 = g * iR * iR * (sc - alpha * cc);
    P.p2 = -g / alpha * m * m * cc;
    P.Rp = g * m * iR * cc;
    return P;
  }
  if (type == T_ELLDISK || type == T_LOPSIDED) {
    double k, p, harm;
    if (type == T_ELLDISK) {
      const double sm = a[1] != a[1] ? 1.0 : dehnen_smooth(t, a[1], a[2], ldg(&cp->c[9]));
      k = amp * sm * a[3];
      p = a[4];
      harm = 2.0;
    } else {
      k = amp * a[1];
      p = a[2];
      harm = 1.0;
    }
    const double phib = type == T_ELLDISK ? a[5] : a[3];
    double sn, cs;
    sincos(harm * (phi - phib), &sn, &cs);
    const double Rp1 = pow(R, p - 1.0), Rp0 = Rp1 * R;
    const double h = type == T_ELLDISK ? 0.5 : 1.0;  // the R-part's factor: twophio / 2, phio
    P.FR = -k * h * p * Rp1 * cs;
    P.tq = k * h * harm * Rp0 * sn;
    P.R2 = k * h * p * (p - 1.0) * Rp1 / R * cs;
    P.p2 = -k * h * harm * harm * Rp0 * cs;
    P.Rp = -k * h * harm * p * Rp1 * sn;
    return P;
  }
  // CosmphiDisk
  const double mphio = a[1], p = a[2], mphib = a[3], m = (double)(int)a[4], rb = a[5];
  const double rbp = a[6], rb2p = a[7], r1p = a[8];
  double sn, cs;
  sincos(m * phi - mphib, &sn, &cs);
  if (R <= rb) {
    const double iRp = pow(R, -p), inner = rbp * (2.0 * r1p - rbp * iRp);
    P.FR = -amp * p * mphio / m * rb2p * iRp / R * cs;
    P.tq = amp * mphio * inner * sn;
    P.R2 = -amp * p * (p + 1.0) * mphio / m * rb2p * iRp / (R * R) * cs;
    P.p2 = -amp * m * mphio * inner * cs;
    P.Rp = -amp * p * mphio / m * rb2p * iRp / R * sn;
  } else {
    const double Rp1 = pow(R, p - 1.0), Rp0 = Rp1 * R;
    P.FR = -amp * p * mphio / m * Rp1 * cs;
    P.tq = amp * mphio * Rp0 * sn;
    P.R2 = amp * p * (p - 1.0) * mphio / m * Rp1 / R * cs;
    P.p2 = -amp * m * mphio * Rp0 * cs;
    P.Rp = -amp * p * mphio * Rp1 * sn;
  }
  return P;
}

// Cartesian acceleration (and K = -grad grad Phi if K) in the plane from
// the cylindrical parts at (x, y), R > 0.
GPC_HD GPC_FI void disk_pert_accel(const GpComp* __restrict__ cp, int type, double x, double y,
                                   double t, double& ax, double& ay, double* K)
{
  const double R = sqrt(x * x + y * y), iR = 1.0 / R, c = x * iR, s = y * iR;
  const CylParts P = disk_pert_parts(cp, type, R, atan2(y, x), t);
  ax += c * P.FR - s * iR * P.tq;
  ay += s * P.FR + c * iR * P.tq;
  if (K) {
    const double PR = -P.FR, Pf = -P.tq, iR2 = iR * iR, cs = c * s, c2s2 = c * c - s * s;
    K[0] -= c * c * P.R2 - 2.0 * cs * iR * P.Rp + s * s * iR2 * P.p2 + s * s * iR * PR +
            2.0 * cs * iR2 * Pf;
    K[1] -= cs * P.R2 + c2s2 * iR * P.Rp - cs * iR2 * P.p2 - cs * iR * PR - c2s2 * iR2 * Pf;
    K[2] -= s * s * P.R2 + 2.0 * cs * iR * P.Rp + c * c * iR2 * P.p2 + c * c * iR * PR -
            2.0 * cs * iR2 * Pf;
  }
}

// ---- second-order forward differentiation over (R, z, phi) --------------
// A value with its gradient and (HESS) Hessian in three variables: the
// spiral arms' potential is written once, and its forces and second
// derivatives follow by the chain rule of each operation.
template <bool HESS>
struct Dual3 {
  double v, g[3], h[3][3];
};

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_var(double v, int i)
{
  Dual3<HESS> r;
  r.v = v;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    r.g[a] = a == i ? 1.0 : 0.0;
#pragma unroll
    for (int b = 0; b < 3; b++) r.h[a][b] = 0.0;
  }
  return r;
}

// f(u) from f(u.v), f'(u.v), f''(u.v)
template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_apply(const Dual3<HESS>& u, double f, double f1, double f2)
{
  Dual3<HESS> r;
  r.v = f;
#pragma unroll
  for (int a = 0; a < 3; a++) r.g[a] = f1 * u.g[a];
  if (HESS) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) r.h[a][b] = f1 * u.h[a][b] + f2 * u.g[a] * u.g[b];
  }
  return r;
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_mul(const Dual3<HESS>& x, const Dual3<HESS>& y)
{
  Dual3<HESS> r;
  r.v = x.v * y.v;
#pragma unroll
  for (int a = 0; a < 3; a++) r.g[a] = x.g[a] * y.v + x.v * y.g[a];
  if (HESS) {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++)
        r.h[a][b] = x.h[a][b] * y.v + x.g[a] * y.g[b] + x.g[b] * y.g[a] + x.v * y.h[a][b];
  }
  return r;
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_lin(double ca, const Dual3<HESS>& x, double c0)  // ca x + c0
{
  Dual3<HESS> r;
  r.v = ca * x.v + c0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    r.g[a] = ca * x.g[a];
    if (HESS)
#pragma unroll
      for (int b = 0; b < 3; b++) r.h[a][b] = ca * x.h[a][b];
  }
  return r;
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_rcp(const Dual3<HESS>& u)
{
  const double i = 1.0 / u.v;
  return dual_apply(u, i, -i * i, 2.0 * i * i * i);
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_exp(const Dual3<HESS>& u)
{
  const double e = exp(u.v);
  return dual_apply(u, e, e, e);
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_log(const Dual3<HESS>& u)
{
  const double i = 1.0 / u.v;
  return dual_apply(u, log(u.v), i, -i * i);
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_cos(const Dual3<HESS>& u)
{
  double s, c;
  sincos(u.v, &s, &c);
  return dual_apply(u, c, -s, -c);
}

template <bool HESS>
GPC_HD GPC_FI Dual3<HESS> dual_cosh(const Dual3<HESS>& u)
{
  const double c = cosh(u.v);
  return dual_apply(u, c, sinh(u.v), c);
}

// ---- SpiralArms -------------------------------------------------------------
// Phi = -amp H exp(-(R - r_ref)/Rs) sum_n Cn / (Kn Dn) cos(n gamma)
//       / cosh(Kn z / Bn)^Bn,  gamma = N (phi - omega t - phi_ref - ln(R/r_ref)
//       / tan alpha), Kn = n N / (R sin alpha), Bn = Kn H (1 + 0.4 Kn H),
//       Dn = (1 + Kn H + 0.3 (Kn H)^2) / (1 + 0.3 Kn H)
// (Cox & Gomez 2002).  Record: c0 amp, c1 N, c2 sin alpha, c3 tan alpha, c4
// r_ref, c5 phi_ref, c6 Rs, c7 H, c8 omega, c9 the number of terms, c10.. Cn.
template <bool HESS>
GPC_HD inline Dual3<HESS> spiral_potential(const GpComp* __restrict__ cp, double R, double z,
                                           double phi, double t)
{
  const double amp = ldg(&cp->c[0]), N = ldg(&cp->c[1]), sa = ldg(&cp->c[2]);
  const double ta = ldg(&cp->c[3]), rref = ldg(&cp->c[4]), phiref = ldg(&cp->c[5]);
  const double Rs = ldg(&cp->c[6]), H = ldg(&cp->c[7]), om = ldg(&cp->c[8]);
  const int nC = (int)ldg(&cp->c[9]);
  const Dual3<HESS> vR = dual_var<HESS>(R, 0), vz = dual_var<HESS>(z, 1);
  const Dual3<HESS> vf = dual_var<HESS>(phi, 2);
  const Dual3<HESS> iR = dual_rcp(vR);
  // gamma = N (phi - omega t - phi_ref) - N / tan(alpha) ln(R / r_ref)
  Dual3<HESS> gam = dual_lin(-N / ta, dual_log(dual_lin(1.0 / rref, vR, 0.0)), 0.0);
#pragma unroll
  for (int a = 0; a < 3; a++) gam.g[a] += N * vf.g[a];
  gam.v += N * (phi - om * t - phiref);
  Dual3<HESS> sum = dual_lin(0.0, vR, 0.0);
  for (int n = 1; n <= nC && n <= kSpiralMaxTerms; n++) {
    const double Cn = ldg(&cp->c[9 + n]);
    const Dual3<HESS> Kn = dual_lin(n * N / sa, iR, 0.0);   // n N / (R sin alpha)
    const Dual3<HESS> KH = dual_lin(H, Kn, 0.0);
    const Dual3<HESS> Bn = dual_mul(KH, dual_lin(0.4, KH, 1.0));
    const Dual3<HESS> Dn = dual_mul(dual_lin(1.0, dual_mul(KH, dual_lin(0.3, KH, 1.0)), 1.0),
                                    dual_rcp(dual_lin(0.3, KH, 1.0)));
    const Dual3<HESS> c = dual_cos(dual_lin((double)n, gam, 0.0));
    // cosh(Kn z / Bn)^(-Bn) = exp(-Bn log cosh(Kn z / Bn))
    const Dual3<HESS> arg = dual_mul(dual_mul(Kn, vz), dual_rcp(Bn));
    const Dual3<HESS> sech = dual_exp(dual_mul(dual_lin(-1.0, Bn, 0.0), dual_log(dual_cosh(arg))));
    const Dual3<HESS> term = dual_mul(dual_mul(c, sech), dual_rcp(dual_mul(Kn, Dn)));
    sum.v += Cn * term.v;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      sum.g[a] += Cn * term.g[a];
      if (HESS)
#pragma unroll
        for (int b = 0; b < 3; b++) sum.h[a][b] += Cn * term.h[a][b];
    }
  }
  const Dual3<HESS> pre = dual_exp(dual_lin(-1.0 / Rs, vR, rref / Rs));
  return dual_lin(-amp * H, dual_mul(pre, sum), 0.0);
}

// Acceleration (and K if K) of the spiral arms at (x, y, z), time t, R > 0.
template <bool PLANAR>
GPC_HD inline void spiral_accel(const GpComp* __restrict__ cp, double x, double y, double z,
                                double t, double& ax, double& ay, double& az, double* K)
{
  const double zz = PLANAR ? 0.0 : z;
  const double R = sqrt(x * x + y * y), iR = 1.0 / R, c = x * iR, s = y * iR;
  const double phi = atan2(y, x);
  if (!K) {
    const Dual3<false> P = spiral_potential<false>(cp, R, zz, phi, t);
    const double FR = -P.g[0], tq = -P.g[2];
    ax += c * FR - s * iR * tq;
    ay += s * FR + c * iR * tq;
    if (!PLANAR) az += -P.g[1];
    return;
  }
  const Dual3<true> P = spiral_potential<true>(cp, R, zz, phi, t);
  const double FR = -P.g[0], tq = -P.g[2];
  ax += c * FR - s * iR * tq;
  ay += s * FR + c * iR * tq;
  if (!PLANAR) az += -P.g[1];
  const double R2 = P.h[0][0], p2 = P.h[2][2], Rp = P.h[0][2];
  const double PR = -FR, Pf = -tq, iR2 = iR * iR, cs = c * s, c2s2 = c * c - s * s;
  K[0] -= c * c * R2 - 2.0 * cs * iR * Rp + s * s * iR2 * p2 + s * s * iR * PR + 2.0 * cs * iR2 * Pf;
  K[1] -= cs * R2 + c2s2 * iR * Rp - cs * iR2 * p2 - cs * iR * PR - c2s2 * iR2 * Pf;
  K[2] -= s * s * R2 + 2.0 * cs * iR * Rp + c * c * iR2 * p2 + c * c * iR * PR - 2.0 * cs * iR2 * Pf;
  if (!PLANAR) {
    const double Rz = P.h[0][1], zp = P.h[1][2];
    K[3] -= c * Rz - s * iR * zp;
    K[4] -= s * Rz + c * iR * zp;
    K[5] -= P.h[1][1];
  }
}

// ---- SoftenedNeedleBar ------------------------------------------------------
// In the frame turning with the bar (angle pa + omegab t):
// Phi = amp ln[(x - a + T-) / (x + a + T+)] / (2a), T+- = sqrt((a +- x)^2 +
// y^2 + u^2), u = b + sqrt(z^2 + c^2) (Long & Murali 1992).  Its gradient
// per amplitude, with G = (a - x)/T- + (a + x)/T+ and T+ - T- = 4ax/(T+ + T-)
// (no cancellation near x = 0):
//   dPhi/dx = 2x / (T+ T- (T+ + T-)),  G/(2a) = (S - 4x^2/S) / (2 T+ T-), S = T+ + T-,
//   dPhi/dy = y G/(2a s2),  dPhi/dz = w G/(2a s2),  s2 = y^2 + u^2, w = z u / sqrt(z^2 + c^2).
// The Hessian adds h = ((a - x)/T-^3 + (a + x)/T+^3)/(2a) and k = (1/T-^3 -
// 1/T+^3)/(2a) = 2x (T+^2 + T+ T- + T-^2) / (S T+^3 T-^3):
//   xx h, xy -y k, xz -w k, yy g (s2 - 2y^2)/s2^2 - y^2 h/s2,
//   yz -y w (2g/s2^2 + h/s2), zz (1 + b c^2/zc^3) g/s2 - w^2 (h/s2 + 2g/s2^2)
// with g = G/(2a).  Record: c0 amp, c1 a, c2 b, c3 c^2, c4 pa, c5 omegab,
// c6 1/(2a).
template <bool PLANAR>
GPC_HD inline void needle_accel(const GpComp* __restrict__ cp, double t, double X, double Y,
                                double Z, double& ax, double& ay, double& az, double* K)
{
  const double amp = ldg(&cp->c[0]), a = ldg(&cp->c[1]), b = ldg(&cp->c[2]);
  const double c2 = ldg(&cp->c[3]);
  double sn, cs;
  sincos(ldg(&cp->c[4]) + ldg(&cp->c[5]) * t, &sn, &cs);
  const double x = cs * X + sn * Y, y = cs * Y - sn * X, z = PLANAR ? 0.0 : Z;
  const double zc = sqrt(z * z + c2), u = b + zc, s2 = y * y + u * u, is2 = 1.0 / s2;
  const double Tp = sqrt((a + x) * (a + x) + s2), Tm = sqrt((a - x) * (a - x) + s2);
  const double S = Tp + Tm, iS = 1.0 / S, iPM = 1.0 / (Tp * Tm);
  const double g = 0.5 * (S - 4.0 * x * x * iS) * iPM;  // G / (2a)
  const double px = 2.0 * x * iPM * iS, py = y * g * is2;
  const double fx = -amp * px, fy = -amp * py;
  ax += cs * fx - sn * fy;
  ay += sn * fx + cs * fy;
  const double w = z * u / zc;
  if (!PLANAR) az -= amp * w * g * is2;
  if (!K) return;
  const double iP3 = iPM * iPM * iPM, i2a = ldg(&cp->c[6]);
  const double h = ((a - x) * Tp * Tp * Tp + (a + x) * Tm * Tm * Tm) * iP3 * i2a;
  const double k = 2.0 * x * (Tp * Tp + Tp * Tm + Tm * Tm) * iS * iP3;
  const double pxx = h, pxy = -y * k, pyy = g * (s2 - 2.0 * y * y) * is2 * is2 - y * y * h * is2;
  // rotate the bar-frame Hessian back: R H R^T with R = [[cs, -sn], [sn, cs]]
  const double c2r = cs * cs, s2r = sn * sn, csr = cs * sn;
  K[0] -= amp * (c2r * pxx - 2.0 * csr * pxy + s2r * pyy);
  K[1] -= amp * (csr * (pxx - pyy) + (c2r - s2r) * pxy);
  K[2] -= amp * (s2r * pxx + 2.0 * csr * pxy + c2r * pyy);
  if (!PLANAR) {
    const double pxz = -w * k, pyz = -y * w * (2.0 * g * is2 * is2 + h * is2);
    const double pzz = (1.0 + b * c2 / (zc * zc * zc)) * g * is2 - w * w * (h * is2 + 2.0 * g * is2 * is2);
    K[3] -= amp * (cs * pxz - sn * pyz);
    K[4] -= amp * (sn * pxz + cs * pyz);
    K[5] -= amp * pzz;
  }
}

// Potential of the needle bar at time t.
GPC_HD inline double needle_value(const GpComp* __restrict__ cp, double t, double X, double Y,
                                  double Z)
{
  const double amp = ldg(&cp->c[0]), a = ldg(&cp->c[1]), b = ldg(&cp->c[2]);
  double sn, cs;
  sincos(ldg(&cp->c[4]) + ldg(&cp->c[5]) * t, &sn, &cs);
  const double x = cs * X + sn * Y, y = cs * Y - sn * X;
  const double u = b + sqrt(Z * Z + ldg(&cp->c[3])), s2 = y * y + u * u;
  const double Tp = sqrt((a + x) * (a + x) + s2), Tm = sqrt((a - x) * (a - x) + s2);
  return amp * ldg(&cp->c[6]) * log((x - a + Tm) / (x + a + Tp));
}

// ---- SCF --------------------------------------------------------------------
// Record: c0 a, c1 1 if non-axisymmetric, c2 N, c3 L, c4 the number of m
// orders summed (L if non-axisymmetric, else 1), c5 the payload offset of
// the recurrence table.  Payload (continuation records): for m < c4, l in
// [m, L), n < N: sqrt(4 pi) Acos_nlm (and sqrt(4 pi) Asin_nlm next to it if
// non-axisymmetric); then for l < L, n < N - 1 the Gegenbauer recurrence
// C_{n+1} = p0 xi C_n - p1 C_{n-1} of alpha = 2l + 3/2 (p0, p1), of
// alpha + 1 (p2, p3) and of alpha + 2 (p4, p5): kScfTable doubles.
constexpr int kScfTable = 6;

// Derivatives of Phi in spherical coordinates (r, theta, phi); the second
// ones only with HESS.
struct ScfSums {
  double pot;                  // Phi
  double dr, dth, dph;         // first derivatives
  double drr, dthth, dphph;    // second derivatives
  double drth, drph, dthph;
};

template <bool HESS>
GPC_HD inline ScfSums scf_sums(const GpComp* __restrict__ cp, double r, double ct, double st,
                               double cph, double sph)
{
  const double a = ldg(&cp->c[0]);
  const bool nonaxi = ldg(&cp->c[1]) != 0.0;
  const int N = (int)ldg(&cp->c[2]), L = (int)ldg(&cp->c[3]), Me = (int)ldg(&cp->c[4]);
  const int rec0 = (int)ldg(&cp->c[5]);
  const double ar = a + r, iar = 1.0 / ar, xi = (r - a) * iar;
  const double q = r * a * iar * iar;  // the factor between l and l + 1
  const double ar2 = ar * ar, ar3 = ar2 * ar, ar4 = ar2 * ar2;
  ScfSums S{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double cm = 1.0, sm = 0.0;                   // cos, sin m phi
  double pmm = 1.0, dmm = 0.0, emm = 0.0;      // P_m^m and its first, second theta derivative
  // radial prefactors at l = m: -1/(a+r), 1/(r (a+r)^3), 1/(r^2 (a+r)^5), times q^m
  double rtm = -iar, rt1m = iar * iar * iar / r, rt2m = HESS ? rt1m * iar * iar / r : 0.0;
  int j = 0;  // payload cursor (coefficients)
  for (int m = 0; m < Me; m++) {
    if (m > 0) {
      const double f = -(2.0 * m - 1.0);
      const double pn = f * st * pmm, dn = f * (ct * pmm + st * dmm);
      if (HESS) emm = f * (-st * pmm + 2.0 * ct * dmm + st * emm);
      pmm = pn;
      dmm = dn;
      const double cn = cm * cph - sm * sph;
      sm = sm * cph + cm * sph;
      cm = cn;
      rtm *= q;
      rt1m *= q;
      rt2m *= q;
    }
    // P_l^m (p0), P_{l-1}^m (p1) and their theta derivatives (d, e)
    double p1 = 0.0, d1 = 0.0, e1 = 0.0, p0 = pmm, d0 = dmm, e0 = emm;
    double rt = rtm, rt1 = rt1m, rt2 = rt2m;
    for (int l = m; l < L; l++) {
      if (l > m) {
        double pn, dn, en = 0.0;
        if (l == m + 1) {
          const double c2 = 2.0 * m + 1.0;
          pn = c2 * ct * p0;
          dn = c2 * (ct * d0 - st * p0);
          if (HESS) en = c2 * (ct * e0 - 2.0 * st * d0 - ct * p0);
        } else {
          const double il = 1.0 / (double)(l - m), c2 = 2.0 * l - 1.0, c3 = l + m - 1.0;
          pn = (c2 * ct * p0 - c3 * p1) * il;
          dn = (c2 * (ct * d0 - st * p0) - c3 * d1) * il;
          if (HESS) en = (c2 * (ct * e0 - 2.0 * st * d0 - ct * p0) - c3 * e1) * il;
        }
        p1 = p0;
        d1 = d0;
        e1 = e0;
        p0 = pn;
        d0 = dn;
        e0 = en;
        rt *= q;
        rt1 *= q;
        rt2 *= q;
      }
      // radial sums over n with the Gegenbauer recurrences of alpha = 2l + 3/2:
      // C_n, dC_n = 2 alpha C_{n-1}^(alpha+1), d2C_n = 4 alpha (alpha+1) C_{n-2}^(alpha+2)
      const double alpha2 = 4.0 * l + 3.0;                         // 2 alpha
      const double alpha4 = (4.0 * l + 3.0) * (4.0 * l + 5.0);     // 4 alpha (alpha + 1)
      const int tb = rec0 + kScfTable * l * (N - 1);
      double Cp = 0.0, C = 1.0, Ep = 0.0, E = 1.0, Fp = 0.0, F = 1.0;
      double ac = payload(cp, j), as = nonaxi ? payload(cp, j + 1) : 0.0;
      j += nonaxi ? 2 : 1;
      double Sc = ac, Ss = as, Dc = 0.0, Ds = 0.0, Hc = 0.0, Hs = 0.0;
      for (int n = 1; n < N; n++) {
        const int k = tb + kScfTable * (n - 1);
        const double Cn = payload(cp, k) * xi * C - payload(cp, k + 1) * Cp;
        const double dC = alpha2 * E;
        const double En = payload(cp, k + 2) * xi * E - payload(cp, k + 3) * Ep;
        Cp = C;
        C = Cn;
        Ep = E;
        E = En;
        ac = payload(cp, j);
        as = nonaxi ? payload(cp, j + 1) : 0.0;
        j += nonaxi ? 2 : 1;
        Sc += ac * Cn;
        Ss += as * Cn;
        Dc += ac * dC;
        Ds += as * dC;
        if (HESS && n >= 2) {
          const double d2C = alpha4 * F;  // F = C_{n-2}^(alpha+2)
          Hc += ac * d2C;
          Hs += as * d2C;
          const int k2 = tb + kScfTable * (n - 2);
          const double Fn = payload(cp, k2 + 4) * xi * F - payload(cp, k2 + 5) * Fp;
          Fp = F;
          F = Fn;
        }
      }
      // azimuthal combinations and their phi derivatives
      const double U = cm * Sc + sm * Ss, V = cm * Dc + sm * Ds;
      const double Uf = (double)m * (cm * Ss - sm * Sc);
      const double c1 = (2.0 * l + 1.0) * r * ar - l * ar2, c0 = 2.0 * a * r;
      const double R1 = rt1 * (c1 * U - c0 * V);  // d/dr of the radial factor times U
      S.pot += p0 * rt * U;
      S.dr += p0 * R1;
      S.dth += d0 * rt * U;
      S.dph += p0 * rt * Uf;
      if (HESS) {
        const double H = cm * Hc + sm * Hs, Vf = (double)m * (cm * Ds - sm * Dc);
        const double u2 = l * (1.0 - l) * ar4 - (4.0 * l * l + 6.0 * l + 2.0) * r * r * ar2 +
                          l * (4.0 * l + 2.0) * r * ar3;
        const double v2 = a * r * (4.0 * r * r + 4.0 * a * r + (8.0 * l + 4.0) * r * ar -
                                   4.0 * l * ar2);
        const double w2 = 4.0 * a * a * r * r;
        S.drr += p0 * rt2 * (u2 * U + v2 * V - w2 * H);
        S.dthth += e0 * rt * U;
        S.dphph -= (double)(m * m) * p0 * rt * U;
        S.drth += d0 * R1;
        S.drph += p0 * rt1 * (c1 * Uf - c0 * Vf);
        S.dthph += d0 * rt * Uf;
      }
    }
  }
  return S;
}

// Acceleration -grad Phi (PLANAR: at z = 0); pot receives Phi if non-null.
template <bool PLANAR>
GPC_HD inline void scf_accel(const GpComp* __restrict__ cp, double x, double y, double z,
                             double& ax, double& ay, double& az, double* pot = nullptr)
{
  const double zz = PLANAR ? 0.0 : z;
  const double R2 = x * x + y * y, r2 = R2 + zz * zz, R = sqrt(R2), r = sqrt(r2);
  const double iR = R > 0.0 ? 1.0 / R : 0.0, ir = 1.0 / r;
  const double cph = R > 0.0 ? x * iR : 1.0, sph = R > 0.0 ? y * iR : 0.0;
  const ScfSums S = scf_sums<false>(cp, r, zz * ir, R * ir, cph, sph);
  if (pot) *pot = S.pot;
  // dPhi/dx_i = Phi_r x_i / r + Phi_theta dtheta/dx_i + Phi_phi dphi/dx_i,
  // theta = atan2(R, z): dtheta/dR = z / r^2, dtheta/dz = -R / r^2
  const double gr = S.dr * ir, gth = S.dth * ir * ir, gph = S.dph * iR;
  ax = -(gr * x + gth * zz * cph - gph * sph);
  ay = -(gr * y + gth * zz * sph + gph * cph);
  az = PLANAR ? 0.0 : -(gr * zz - gth * R);
}

// Acceleration and K = -grad grad Phi added to ax.. and K (PLANAR: at
// z = 0): the spherical second derivatives, then the cylindrical ones by the
// chain rule through r = sqrt(R^2 + z^2), theta = atan2(R, z) (as the
// reference's compute_scf_hessian_cyl), then the Cartesian tensor from the
// cylindrical derivatives (R > 0).
template <bool PLANAR>
GPC_HD inline void scf_tidal(const GpComp* __restrict__ cp, double x, double y, double z,
                             double& ax, double& ay, double& az, double K[6])
{
  const double zz = PLANAR ? 0.0 : z;
  const double R2 = x * x + y * y, r2 = R2 + zz * zz, R = sqrt(R2), r = sqrt(r2);
  const double iR = 1.0 / R, ir = 1.0 / r;
  const double c = x * iR, s = y * iR;
  const ScfSums S = scf_sums<true>(cp, r, zz * ir, R * ir, c, s);
  const double ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2;
  const double rR = R * ir, rz = zz * ir, thR = zz * ir2, thz = -R * ir2;
  const double rRR = zz * zz * ir3, rzz = R2 * ir3, rRz = -R * zz * ir3;
  const double thRR = -2.0 * R * zz * ir4, thzz = -thRR, thRz = (R2 - zz * zz) * ir4;
  const double PR = S.dr * rR + S.dth * thR, Pz = S.dr * rz + S.dth * thz, Pf = S.dph;
  const double HRR = S.drr * rR * rR + 2.0 * S.drth * rR * thR + S.dthth * thR * thR +
                     S.dr * rRR + S.dth * thRR;
  const double Hzz = S.drr * rz * rz + 2.0 * S.drth * rz * thz + S.dthth * thz * thz +
                     S.dr * rzz + S.dth * thzz;
  const double HRz = S.drr * rR * rz + S.drth * (rR * thz + rz * thR) + S.dthth * thR * thz +
                     S.dr * rRz + S.dth * thRz;
  const double Hff = S.dphph, HRf = S.drph * rR + S.dthph * thR, Hzf = S.drph * rz + S.dthph * thz;
  // gradient and Hessian of Phi(R, phi, z) in Cartesian coordinates
  ax -= c * PR - s * iR * Pf;
  ay -= s * PR + c * iR * Pf;
  if (!PLANAR) az -= Pz;
  const double iR2 = iR * iR, cs = c * s, c2s2 = c * c - s * s;
  K[0] -= c * c * HRR - 2.0 * cs * iR * HRf + s * s * iR2 * Hff + s * s * iR * PR +
          2.0 * cs * iR2 * Pf;
  K[1] -= cs * HRR + c2s2 * iR * HRf - cs * iR2 * Hff - cs * iR * PR - c2s2 * iR2 * Pf;
  K[2] -= s * s * HRR + 2.0 * cs * iR * HRf + c * c * iR2 * Hff + c * c * iR * PR -
          2.0 * cs * iR2 * Pf;
  if (!PLANAR) {
    K[3] -= c * HRz - s * iR * Hzf;
    K[4] -= s * HRz + c * iR * Hzf;
    K[5] -= Hzz;
  }
}

}  // namespace gpc
