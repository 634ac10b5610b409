/*
 * oracle/galpy_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of galpy's batched C orbit integration for the potential
 * types and integrators that the CUDA engine implements.  It is the checker
 * for the CUDA kernels (tests/, __graft_entry__.smoke(), bench.py's CPU
 * baseline leg) and is never linked into, or called by, the product path.
 *
 * What is restated (reference file:line in galpy):
 *   forces   PowerSphericalPotentialwCutoff.c:9-131, MiyamotoNagaiPotential.c:
 *            16-117, NFWPotential.c:16-106, HernquistPotential.c:15-100,
 *            LogarithmicHaloPotential.c:5-297, and the spherical
 *            PowerSpherical, Jaffe, Isochrone, Plummer, PseudoIsothermal,
 *            Burkert, DehnenCore, Dehnen, HomogeneousSphere potentials and
 *            ZeroForce, Einasto and ExpTruncNFW (through
 *            SphericalPotential.c),
 *            FlattenedPowerPotential.c, KuzminKutuzovStaeckelPotential.c,
 *            HenonHeilesPotential.c (planar), the time-dependent
            DehnenBarPotential.c and SCFPotential.c (static coefficients;
            the Gegenbauer and Legendre arrays by this file's own
            recurrences) (potential_c_ext/)
 *   sums     galpy_potentials.c:120-354 (sum over components, in order)
 *   RHS      orbit_c_ext/integrateFullOrbit.c:1307-1352 (evalRectForce,
 *            evalRectDeriv), :1496-1681 (the dxdv variants);
 *            orbit_c_ext/integratePlanarOrbit.c:1015-1055, :1124-1276
 *   steppers util/bovy_symplecticode.c:132-587 (leapfrog, symplec4,
 *            symplec6), :588-1052 (their step estimators), :1053-1400
 *            (*_dxdv); util/bovy_rk.c:66-480 (rk4, rk6 + estimators),
 *            :501-760 (dopr54); util/leung_dop853.c:231-517 (dop853)
 *   drivers  integrateFullOrbit.c:1046-1150, :1151-1233 (surface of
 *            section, with evalSOSDeriv :1353-1390), :1234-1306;
 *            integratePlanarOrbit.c:848-939 (planar surface of section,
 *            with evalPlanarSOSDerivx/y :1056-1123);
 *            integratePlanarOrbit.c:743-847, :940-1014
 *   coords   util/bovy_coords.c:57-148
 * Each force evaluation gets the time the reference's stepper hands it (its
 * own bookkeeping of `to`, t_current, t_old, or the state's time in a
 * surface of section), which only the time-dependent components read.
 * The arithmetic of each formula follows the reference term by term so that
 * this restatement agrees with the reference's own C (built from its sources
 * into oracle/_ref by oracle/Makefile) to the last bit or close to it; the
 * incomplete gamma function is the one in oracle/incgamma.c.
 *
 * Extras over the reference (test instrumentation only): per-orbit counts of
 * accepted steps and of force evaluations, an optional attempt budget, and a
 * stop (err 2) where the reference never returns (a DOP853 attempt rejected
 * at its smallest step repeats exactly).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "dop853_coeffs.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

double oracle_gamma_inc_P(double a, double x);
double oracle_gamma_inc_Q(double a, double x);
double oracle_expint_E1(double x);

/* ------------------------------------------------------------------ */
/* potentials                                                          */
/* ------------------------------------------------------------------ */
enum { PT_LOGHALO = 0, PT_MN = 5, PT_HERNQUIST = 8, PT_NFW = 9, PT_PSWC = 15 };
/* spherical potentials, each restated from potential_c_ext/<name>.c */
enum {
  PT_POWER = 7,       /* PowerSphericalPotential (KeplerPotential: alpha = 3) */
  PT_JAFFE = 10,      /* JaffePotential */
  PT_ISOCHRONE = 14,  /* IsochronePotential */
  PT_PLUMMER = 17,    /* PlummerPotential */
  PT_PSEUDOISO = 18,  /* PseudoIsothermalPotential */
  PT_BURKERT = 20,    /* BurkertPotential */
  PT_DEHNENCORE = 33, /* DehnenCoreSphericalPotential (DehnenCorePotential.c) */
  PT_DEHNEN = 34,     /* DehnenSphericalPotential (DehnenPotential.c) */
  PT_HOMSPHERE = 35,  /* HomogeneousSpherePotential */
  PT_NULL = 40,       /* NullPotential (ZeroForce) */
  PT_EINASTO = 41,    /* EinastoPotential (through SphericalPotential.c) */
  PT_EXPTRUNCNFW = 46 /* ExpTruncNFWPotential (through SphericalPotential.c) */
};
/* axisymmetric: FlattenedPowerPotential (FlattenedPowerPotential.c); args
   (amp, alpha, q^2, core^2) in 3D, (amp, alpha, core^2) in the plane */
enum { PT_FLATPOWER = 12 };
/* KuzminKutuzovStaeckelPotential (KuzminKutuzovStaeckelPotential.c); args
   (amp, ac, Delta) in 3D and in the plane */
enum { PT_KKS = 16 };
/* planar only: HenonHeilesPotential (HenonHeilesPotential.c), args (amp) */
enum { PT_HENONHEILES = 29 };
/* KuzminDiskPotential (KuzminDiskPotential.c), args (amp, a), 3D and planar */
enum { PT_KUZMINDISK = 19 };
/* the EllipsoidalPotential family (EllipsoidalPotential.c; densities of
   TwoPowerTriaxialPotential.c, PerfectEllipsoidPotential.c,
   TriaxialGaussianPotential.c, PowerTriaxialPotential.c), 3D and planar:
   args (amp, 15 cache slots, npsi, psi args [npsi], b2, c2, aligned,
   rot [9], glorder, glx [glorder], weights [glorder]) */
enum { PT_TRIHERNQUIST = 21, PT_TRINFW = 22, PT_TRIJAFFE = 23, PT_PERFECTELL = 30,
       PT_TRIGAUSS = 37, PT_POWERTRI = 38, PT_TWOPOWERTRI = 43 };
/* time-dependent DehnenBarPotential (DehnenBarPotential.c), args (amp * af,
   tform, tsteady, rb, omegab, barphi), 3D and planar */
enum { PT_DEHNENBAR = 1 };
/* SCFPotential (SCFPotential.c), static coefficients: args (a, isNonAxi, N,
   L, M, Nt = 0, Acos [N][L][M], Asin [N][L][M] if isNonAxi, 11 cache slots) */
enum { PT_SCF = 24 };
/* wrappers (DehnenSmoothWrapperPotential.c, SolidBodyRotationWrapperPotential.c,
   GaussianAmplitudeWrapperPotential.c): type followed by the wrapped
   components' types; args (nwrapped, the wrapped components' args, then
   (amp, tform, tsteady, grow), (amp, omega, pa) or (amp, to, sigma^2)) */
enum { PT_WRAP_SMOOTH = -1, PT_WRAP_ROTATE = -2, PT_WRAP_GAUSS = -5 };
/* KuzminLikeWrapperPotential.c: the wrapped potential at xi(R, z) =
   sqrt(R^2 + (a + sqrt(z^2 + b^2))^2) on the plane, args (amp, a, b^2) */
enum { PT_WRAP_KUZMIN = -10 };
/* CorotatingRotationWrapperPotential.c: the wrapped list at phi - vpo
   R^(beta - 1) (t - to) - pa, args (amp, vpo, beta, pa, to) */
enum { PT_WRAP_COROT = -4 };
/* planar-only disk perturbations: TransientLogSpiral (2; amp, A, to,
   sigma^2, alpha, m, omegas, gamma), SteadyLogSpiral (3; amp, tform,
   tsteady, A, alpha, m, omegas, gamma; tform NaN: no growth), EllipticalDisk
   (4; amp, tform, tsteady, twophio, p, phib), LopsidedDisk (6; amp, phio, p,
   phib), CosmphiDisk (28; amp, mphio, p, mphib, m, rb, rb^p, rb^2p, r1^p) */
enum { PT_TRANSPIRAL = 2, PT_STEADYSPIRAL = 3, PT_ELLDISK = 4, PT_LOPSIDED = 6,
       PT_COSMPHI = 28 };
/* SpiralArmsPotential (SpiralArmsPotential.c), 3D and planar: args (nCs,
   amp, N, sin alpha, tan alpha, r_ref, phi_ref, Rs, H, omega, Cs[nCs]) */
enum { PT_SPIRALARMS = 27 };
/* SoftenedNeedleBarPotential (SoftenedNeedleBarPotential.c), 3D and planar:
   args (amp, a, b, c^2, pa, omegab, 7 cache slots the reference fills) */
enum { PT_NEEDLEBAR = 25 };

static int is_ellipsoidal(int type)
{
  switch (type) {
  case PT_TRIHERNQUIST: case PT_TRINFW: case PT_TRIJAFFE: case PT_PERFECTELL:
  case PT_TRIGAUSS: case PT_POWERTRI: case PT_TWOPOWERTRI:
    return 1;
  }
  return 0;
}

/* argument count of an ellipsoidal component (integrateFullOrbit.c case 21) */
static int ell_nargs(const double *a)
{
  int np = (int)a[16];
  return 30 + np + 2 * (int)a[29 + np];
}

/* argument count of an SCF component (integrateFullOrbit.c case 24) with
   static coefficients (Nt = 0; time-dependent coefficients are not
   restated); -1 otherwise */
#define SCF_MAXN 64
#define SCF_MAXL 32
static int scf_nargs(const double *a)
{
  int nonaxi = (int)a[1], N = (int)a[2], L = (int)a[3], M = (int)a[4], Nt = (int)a[5];
  if (Nt != 0 || N < 1 || L < 1 || M < 1 || N > SCF_MAXN || L > SCF_MAXL) return -1;
  if (nonaxi && M != L) return -1; /* the reference sums m <= l over an [N][L][L] array */
  return 6 + (1 + nonaxi) * N * L * M + 11;
}

#define OMAXPOT 32

typedef struct {
  int type;
  double p[9];     /* the component's args as galpy passes them */
  const double *ea; /* all args (ellipsoidal and SCF components: the caller's array) */
  double t;        /* time of the current evaluation (time-dependent types) */
  int nsub;        /* a wrapper: the entries it wraps, which follow it */
} ocomp;

typedef struct {
  int n;
  int planar;
  ocomp c[OMAXPOT];
  long long nforce; /* force evaluations (instrumentation) */
  double t;         /* time at which the stepper evaluates the next force */
} opot;

static int nargs_of(int type, int planar)
{
  switch (type) {
  case PT_LOGHALO: return 4;
  case PT_MN: return 3;
  case PT_HERNQUIST: return 2;
  case PT_NFW: return 2;
  case PT_PSWC: return planar ? 3 : 5;
  case PT_POWER: case PT_JAFFE: case PT_ISOCHRONE: case PT_PLUMMER: case PT_PSEUDOISO:
  case PT_BURKERT: case PT_DEHNENCORE: return 2;
  case PT_DEHNEN: case PT_HOMSPHERE: case PT_EINASTO: case PT_EXPTRUNCNFW: return 3;
  case PT_NULL: return 0;
  case PT_FLATPOWER: return planar ? 3 : 4;
  case PT_KKS: return 3;
  case PT_HENONHEILES: return planar ? 1 : -1;
  case PT_KUZMINDISK: return 2;
  case PT_DEHNENBAR: return 6;
  case PT_NEEDLEBAR: return 13;
  case PT_TRANSPIRAL: case PT_STEADYSPIRAL: return planar ? 8 : -1;
  case PT_ELLDISK: return planar ? 6 : -1;
  case PT_LOPSIDED: return planar ? 4 : -1;
  case PT_COSMPHI: return planar ? 9 : -1;
  default: return -1;
  }
}

static int is_new_spherical(int type)
{
  switch (type) {
  case PT_POWER: case PT_JAFFE: case PT_ISOCHRONE: case PT_PLUMMER: case PT_PSEUDOISO:
  case PT_BURKERT: case PT_DEHNENCORE: case PT_DEHNEN: case PT_HOMSPHERE: case PT_NULL:
  case PT_EINASTO: case PT_EXPTRUNCNFW:
    return 1;
  }
  return 0;
}

/* ExpTruncNFWPotential.c, args (amp, a, rc): the enclosed-mass function F
   (a small-r series below 1e-3 min(a, rc)), G, and the radial functions;
   GSL's E1 restated in incgamma.c; SphericalPotential.c applies amp */
static double etnfw_F(double r, double a, double rc)
{
  double small_r_thresh = 1e-3 * (a < rc ? a : rc);
  if (r < small_r_thresh) {
    double c2 = 0.5;
    double c3 = -(1.0 / rc + 2.0 / a) / 3.0;
    double c4 = (0.5 / (rc * rc) + 2.0 / (rc * a) + 3.0 / (a * a)) / 4.0;
    double c5 = -(1.0 / (6.0 * rc * rc * rc) + 1.0 / (rc * rc * a) + 3.0 / (rc * a * a) +
                  4.0 / (a * a * a)) / 5.0;
    return (r * r / (a * a)) * (c2 + r * (c3 + r * (c4 + r * c5)));
  }
  double alpha = a / rc, beta = (a + r) / rc;
  return (exp(alpha) * (1.0 + alpha) * (oracle_expint_E1(alpha) - oracle_expint_E1(beta)) -
          1.0 + a * exp(-r / rc) / (a + r));
}
static double etnfw_G(double r, double a, double rc)
{
  double alpha = a / rc, beta = (a + r) / rc;
  return exp(-r / rc) / (a + r) - exp(alpha) * oracle_expint_E1(beta) / rc;
}
static double etnfw_rforce(const ocomp *c, double r) { return -etnfw_F(r, c->p[1], c->p[2]) / (r * r); }
static double etnfw_r2deriv(const ocomp *c, double r)
{
  double a = c->p[1], rc = c->p[2];
  double rdens = exp(-r / rc) / (4.0 * M_PI * a * a * r * pow(1.0 + r / a, 2));
  return 4.0 * M_PI * rdens - 2.0 * etnfw_F(r, a, rc) / (r * r * r);
}
static double etnfw_revaluate(const ocomp *c, double r)
{
  return -(etnfw_F(r, c->p[1], c->p[2]) / r + etnfw_G(r, c->p[1], c->p[2]));
}

/* its prolate spheroidal coordinates (l, n) and the derivatives of
   V = 1 / (sqrt(l) + sqrt(n)) the reference uses, as it writes them */
static double kks_Rz(const ocomp *c, double R, double z, int which)
{
  double amp = c->p[0], ac = c->p[1], Delta = c->p[2];
  double gamma = Delta * Delta / (1. - ac * ac);
  double alpha = gamma - Delta * Delta;
  double term = R * R + z * z - alpha - gamma;
  double discr = pow(R * R + z * z - Delta * Delta, 2.) + (4. * Delta * Delta * R * R);
  double l = 0.5 * (term + sqrt(discr));
  double n = 0.5 * (term - sqrt(discr));
  double dVdl = 0.5 / sqrt(l) / pow(sqrt(l) + sqrt(n), 2.);
  double dVdn = 0.5 / sqrt(n) / pow(sqrt(l) + sqrt(n), 2.);
  if (which == 0) { /* Rforce */
    double dldR = R * (1. + (R * R + z * z + Delta * Delta) / sqrt(discr));
    double dndR = R * (1. - (R * R + z * z + Delta * Delta) / sqrt(discr));
    return -amp * (dldR * dVdl + dndR * dVdn);
  }
  /* zforce */
  double dldz = z * (1. + (R * R + z * z - Delta * Delta) / sqrt(discr));
  double dndz = z * (1. - (R * R + z * z - Delta * Delta) / sqrt(discr));
  return -amp * (dldz * dVdl + dndz * dVdn);
}

/* second derivatives: which = 0 R2deriv, 1 z2deriv, 2 Rzderiv */
static double kks_hess(const ocomp *c, double R, double z, int which)
{
  double amp = c->p[0], ac = c->p[1], Delta = c->p[2];
  double D2 = Delta * Delta, D4 = D2 * D2;
  double gamma = D2 / (1. - ac * ac);
  double alpha = gamma - D2;
  double R2 = R * R, z2 = z * z, rz2 = R2 + z2;
  double rzD2p = rz2 + D2, rzmD2 = rz2 - D2;
  double term = rz2 - alpha - gamma;
  double discr = rzmD2 * rzmD2 + (4. * D2 * R2);
  double sdiscr = sqrt(discr), isdiscr = 1. / sdiscr;
  double idiscr15 = isdiscr / discr, idiscr = 1. / discr;
  double l = 0.5 * (term + sdiscr), n = 0.5 * (term - sdiscr);
  double srl = sqrt(l), srn = sqrt(n), sln = srl + srn;
  double isln2 = 1. / (sln * sln), isln3 = isln2 / sln;
  double dVdl = 0.5 / srl * isln2, dVdn = 0.5 / srn * isln2;
  double d2Vdl2 = (-3. * srl - srn) / (4. * l * srl) * isln3;
  double d2Vdn2 = (-srl - 3. * srn) / (4. * n * srn) * isln3;
  double d2Vdln = -0.5 / (srl * srn) * isln3;
  if (which == 0) {
    double rzD2p_isd = rzD2p * isdiscr;
    double dldR = R * (1. + rzD2p_isd), dndR = R * (1. - rzD2p_isd);
    double hess_off = (3. * R2 + z2 + D2) * isdiscr;
    double hess_cub = 2. * R2 * rzD2p * rzD2p * idiscr15;
    double d2ldR2 = 1. + hess_off - hess_cub, d2ndR2 = 1. - hess_off + hess_cub;
    return amp * (d2ldR2 * dVdl + d2ndR2 * dVdn + dldR * dldR * d2Vdl2 +
                  dndR * dndR * d2Vdn2 + 2. * dldR * dndR * d2Vdln);
  }
  if (which == 1) {
    double rzmD2_isd = rzmD2 * isdiscr;
    double dldz = z * (1. + rzmD2_isd), dndz = z * (1. - rzmD2_isd);
    double hess_off = (R2 + 3. * z2 - D2) * isdiscr;
    double hess_cub = 2. * z2 * rzmD2 * rzmD2 * idiscr15;
    double d2ldz2 = 1. + hess_off - hess_cub, d2ndz2 = 1. - hess_off + hess_cub;
    return amp * (d2ldz2 * dVdl + d2ndz2 * dVdn + dldz * dldz * d2Vdl2 +
                  dndz * dndz * d2Vdn2 + 2. * dldz * dndz * d2Vdln);
  }
  double rzD2p_isd = rzD2p * isdiscr, rzmD2_isd = rzmD2 * isdiscr;
  double dldR = R * (1. + rzD2p_isd), dndR = R * (1. - rzD2p_isd);
  double dldz = z * (1. + rzmD2_isd), dndz = z * (1. - rzmD2_isd);
  double mix = 2. * R * z * isdiscr * (1. - (rz2 * rz2 - D4) * idiscr);
  return amp * (mix * dVdl - mix * dVdn + dldR * dldz * d2Vdl2 + dndR * dndz * d2Vdn2 +
                (dldR * dndz + dldz * dndR) * d2Vdln);
}

/* Einasto's radial functions (EinastoPotential.c), args (amp, h, n); the
   reference's GSL calls restated with tgamma and the incomplete gamma of
   incgamma.c; SphericalPotential.c applies amp */
static double einasto_rforce(const ocomp *c, double r)
{
  double h = c->p[1], n = c->p[2], s = r / h;
  double gamma_3n = tgamma(3 * n);
  double gamma_upper_3n = oracle_gamma_inc_Q(3 * n, pow(s, 1.0 / n));
  double s_2 = pow(s, -2.0);
  return (4.0 * M_PI * h * n * gamma_3n) * s_2 * (gamma_upper_3n - 1.0);
}
static double einasto_r2deriv(const ocomp *c, double r)
{
  double h = c->p[1], n = c->p[2], s = r / h, s_1n = pow(s, 1.0 / n);
  double gamma_3n = tgamma(3 * n);
  double gamma_upper_3n = oracle_gamma_inc_Q(3 * n, s_1n);
  return -(4.0 * M_PI * n * gamma_3n) *
         ((-2 * pow(s, -3)) * (gamma_upper_3n - 1) - ((1 / n) * exp(-s_1n) / gamma_3n));
}
static double einasto_revaluate(const ocomp *c, double r)
{
  double h = c->p[1], n = c->p[2], s = r / h, s_1n = pow(s, 1.0 / n);
  return (-(4.0 * M_PI * pow(h, 2) * n * tgamma(3 * n)) * pow(s, -1) *
          (1 - oracle_gamma_inc_Q(3 * n, s_1n) +
           s * (tgamma(2 * n) * oracle_gamma_inc_Q(2 * n, s_1n)) / tgamma(3 * n)));
}

/* 3D R or z force of the spherical potentials: X is R (Rforce) or Z
   (zforce), in the position where each reference formula has it
   (<name>Rforce / <name>zforce in potential_c_ext/) */
static double sph_force3(const ocomp *c, double R, double Z, double X)
{
  double amp = c->p[0];
  switch (c->type) {
  case PT_PLUMMER: { /* PlummerPotential.c:15-43 */
    double b2 = c->p[1] * c->p[1];
    return -amp * X * pow(R * R + Z * Z + b2, -1.5);
  }
  case PT_JAFFE: { /* JaffePotential.c */
    double a = c->p[1], sqrtRz = pow(R * R + Z * Z, 0.5);
    return -amp * X * pow(sqrtRz, -3.) / (1. + a / sqrtRz);
  }
  case PT_ISOCHRONE: { /* IsochronePotential.c */
    double b = c->p[1], r2 = R * R + Z * Z, rb = sqrt(r2 + b * b);
    return -amp * X / rb * pow(b + rb, -2.);
  }
  case PT_POWER: /* PowerSphericalPotential.c */
    return -amp * X * pow(R * R + Z * Z, -0.5 * c->p[1]);
  case PT_BURKERT: { /* BurkertPotential.c */
    double a = c->p[1], r = sqrt(R * R + Z * Z), x = r / a;
    return amp * a * M_PI / x / x *
           (M_PI - 2. * atan(1. / x) - 2. * log(1. + x) - log(1. + x * x)) * X / r;
  }
  case PT_PSEUDOISO: { /* PseudoIsothermalPotential.c */
    double a = c->p[1], r2 = R * R + Z * Z, r = sqrt(r2);
    return -amp * (1. / r - a / r2 * atan(r / a)) / a * X / r;
  }
  case PT_DEHNENCORE: { /* DehnenCorePotential.c */
    double a = c->p[1], sqrtRz = pow(R * R + Z * Z, 0.5);
    return -amp * (X / pow(a + sqrtRz, 3.) / 3.);
  }
  case PT_DEHNEN: { /* DehnenPotential.c */
    double a = c->p[1], alpha = c->p[2], sqrtRz = pow(R * R + Z * Z, 0.5);
    return -amp * (X * pow(1. + a / sqrtRz, alpha) / pow(a + sqrtRz, 3.) / (3. - alpha));
  }
  case PT_HOMSPHERE: { /* HomogeneousSpherePotential.c */
    double R2 = c->p[1], R3 = c->p[2], r2 = R * R + Z * Z;
    if (r2 < R2) return -2. * amp * X;
    return -2. * amp * R3 * X / pow(r2, 1.5);
  }
  case PT_EINASTO: { /* SphericalPotentialRforce / zforce */
    double r = sqrt(R * R + Z * Z);
    return amp * einasto_rforce(c, r) * X / r;
  }
  case PT_EXPTRUNCNFW: {
    double r = sqrt(R * R + Z * Z);
    return amp * etnfw_rforce(c, r) * X / r;
  }
  }
  return 0.;
}

/* planar R force (<name>PlanarRforce) */
static double sph_planarRforce(const ocomp *c, double R)
{
  double amp = c->p[0];
  switch (c->type) {
  case PT_PLUMMER: {
    double b2 = c->p[1] * c->p[1];
    return -amp * R * pow(R * R + b2, -1.5);
  }
  case PT_JAFFE: {
    double a = c->p[1];
    return -amp * pow(R, -2.) / (1. + a / R);
  }
  case PT_ISOCHRONE: {
    double b = c->p[1], r2 = R * R, rb = sqrt(r2 + b * b);
    return -amp * R / rb * pow(b + rb, -2.);
  }
  case PT_POWER:
    return -amp * pow(R, -c->p[1] + 1.);
  case PT_BURKERT: {
    double a = c->p[1], x = R / a;
    return amp * a * M_PI / x / x * (M_PI - 2. * atan(1. / x) - 2. * log(1. + x) - log(1. + x * x));
  }
  case PT_PSEUDOISO: {
    double a = c->p[1];
    return -amp * (1. / R - a / R / R * atan(R / a)) / a;
  }
  case PT_DEHNENCORE: {
    double a = c->p[1];
    return -amp * (R / pow(a + R, 3.) / 3.);
  }
  case PT_DEHNEN: {
    double a = c->p[1], alpha = c->p[2];
    return -amp * (R * pow(1. + a / R, alpha) / pow(a + R, 3.) / (3. - alpha));
  }
  case PT_HOMSPHERE: {
    double R2 = c->p[1], R3 = c->p[2], r2 = R * R;
    if (r2 < R2) return -2. * amp * R;
    return -2. * amp * R3 / r2;
  }
  case PT_EINASTO:
    return amp * einasto_rforce(c, R);
  case PT_EXPTRUNCNFW:
    return amp * etnfw_rforce(c, R);
  }
  return 0.;
}

/* planar d2Phi/dR2 (<name>PlanarR2deriv) */
static double sph_planarR2deriv(const ocomp *c, double R)
{
  double amp = c->p[0];
  switch (c->type) {
  case PT_PLUMMER: {
    double b2 = c->p[1] * c->p[1];
    return amp * (b2 - 2. * R * R) * pow(R * R + b2, -2.5);
  }
  case PT_JAFFE: {
    double a = c->p[1];
    return -amp * (a + 2. * R) * pow(R, -4.) * pow(1. + a / R, -2.);
  }
  case PT_ISOCHRONE: {
    double b = c->p[1], r2 = R * R, rb = sqrt(r2 + b * b);
    return -amp * (-pow(b, 3.) - b * b * rb + 2. * r2 * rb) * pow(rb * (b + rb), -3.);
  }
  case PT_POWER: {
    double alpha = c->p[1];
    return amp * (1. - alpha) * pow(R, -alpha);
  }
  case PT_BURKERT: {
    double a = c->p[1], x = R / a, R5 = pow(R, 5);
    return -amp * M_PI * pow(a, 3) / R5 *
           (-4. * R5 / (a * a + R * R) / (a + R) -
            2. * R * R * (M_PI - 2. * atan(1. / x) - 2. * log(1. + x) - log(1. + x * x)));
  }
  case PT_PSEUDOISO: {
    double a = c->p[1], a2 = a * a, R2 = R * R;
    return amp / R2 * (2. * a / R * atan(R / a) - (2. * a2 + R2) / (a2 + R2)) / a;
  }
  case PT_DEHNENCORE: {
    double a = c->p[1];
    return -amp * (pow(a + R, -4.) * (2. * R - a)) / 3.;
  }
  case PT_DEHNEN: {
    double a = c->p[1], alpha = c->p[2];
    return -amp * (pow(1. + a / R, alpha) * pow(a + R, -4.) * (2. * R + a * (alpha - 1.))) /
           (3. - alpha);
  }
  case PT_HOMSPHERE: {
    double R2 = c->p[1], R3 = c->p[2], r2 = R * R;
    if (r2 < R2) return 2. * amp;
    return -4. * amp * R3 / pow(r2, 1.5);
  }
  case PT_EINASTO:
    return amp * einasto_r2deriv(c, R);
  case PT_EXPTRUNCNFW:
    return amp * etnfw_r2deriv(c, R);
  }
  return 0.;
}

/* 3D Hessian terms (which = 0 R2, 1 z2, 2 Rz): Plummer and Jaffe have their
   own closed forms in the reference; the others assemble Phi'' and Phi'/r
   from the planar functions at r (e.g. IsochronePotential.c R2deriv) */
static double sph_hess3(const ocomp *c, int which, double R, double Z)
{
  double amp = c->p[0];
  if (c->type == PT_NULL || which > 2) return 0.;
  if (c->type == PT_PLUMMER) {
    double b2 = c->p[1] * c->p[1];
    if (which == 0) return amp * (b2 - 2. * R * R + Z * Z) * pow(R * R + Z * Z + b2, -2.5);
    if (which == 1) return amp * (b2 + R * R - 2. * Z * Z) * pow(R * R + Z * Z + b2, -2.5);
    return amp * (-3. * R * Z * pow(R * R + Z * Z + b2, -2.5));
  }
  if (c->type == PT_JAFFE) {
    double a = c->p[1], r = sqrt(R * R + Z * Z);
    double dphi = pow(r, -2.) / (1. + a / r);
    double d2phi = -(a + 2. * r) * pow(r, -4.) * pow(1. + a / r, -2.);
    if (which == 0) return amp * (d2phi * R * R / r / r + dphi * Z * Z / r / r / r);
    if (which == 1) return amp * (d2phi * Z * Z / r / r + dphi * R * R / r / r / r);
    return amp * R * Z * (d2phi / r / r - dphi / r / r / r);
  }
  double r2 = R * R + Z * Z, r = sqrt(r2);
  double Phipp = sph_planarR2deriv(c, r), Phip = -sph_planarRforce(c, r);
  double ir2 = 1. / r2, ir3 = ir2 / r;
  if (which == 0) return Phipp * R * R * ir2 + Phip * Z * Z * ir3;
  if (which == 1) return Phipp * Z * Z * ir2 + Phip * R * R * ir3;
  return R * Z * (Phipp * ir2 - Phip * ir3);
}

/* potential value (<name>Eval) */
static double sph_eval(const ocomp *c, double R, double Z)
{
  double amp = c->p[0];
  switch (c->type) {
  case PT_PLUMMER: {
    double b2 = c->p[1] * c->p[1];
    return -amp / sqrt(R * R + Z * Z + b2);
  }
  case PT_JAFFE: {
    double a = c->p[1], sqrtRz = pow(R * R + Z * Z, 0.5);
    return -amp * log(1. + a / sqrtRz) / a;
  }
  case PT_ISOCHRONE: {
    double b = c->p[1], r2 = R * R + Z * Z;
    return -amp / (b + sqrt(r2 + b * b));
  }
  case PT_POWER: {
    double alpha = c->p[1];
    if (alpha == 2.) return 0.5 * amp * log(R * R + Z * Z);
    return -amp * pow(R * R + Z * Z, 1. - 0.5 * alpha) / (alpha - 2.);
  }
  case PT_BURKERT: {
    double a = c->p[1], x = sqrt(R * R + Z * Z) / a;
    return -amp * a * a * M_PI / x *
           (-M_PI + 2. * (1. + x) * atan(1 / x) + 2. * (1. + x) * log(1. + x) +
            (1. - x) * log(1. + x * x));
  }
  case PT_PSEUDOISO: {
    double a = c->p[1], a2 = a * a, r2 = R * R + Z * Z, r = sqrt(r2);
    return amp * (0.5 * log(1 + r2 / a2) + a / r * atan(r / a)) / a;
  }
  case PT_DEHNENCORE: {
    double a = c->p[1], sqrtRz = pow(R * R + Z * Z, 0.5);
    return -amp * (1. - pow(sqrtRz / (sqrtRz + a), 2.)) / (6. * a);
  }
  case PT_DEHNEN: {
    double a = c->p[1], alpha = c->p[2], sqrtRz = pow(R * R + Z * Z, 0.5);
    return -amp * (1. - pow(sqrtRz / (sqrtRz + a), 2. - alpha)) /
           (a * (2. - alpha) * (3. - alpha));
  }
  case PT_HOMSPHERE: {
    double R2 = c->p[1], R3 = c->p[2], r2 = R * R + Z * Z;
    if (r2 < R2) return amp * (r2 - 3. * R2);
    return -2. * amp * R3 / sqrt(r2);
  }
  case PT_EINASTO:
    return amp * einasto_revaluate(c, sqrt(R * R + Z * Z));
  case PT_EXPTRUNCNFW:
    return amp * etnfw_revaluate(c, sqrt(R * R + Z * Z));
  }
  return 0.;
}

/* Decode galpy's (pot_type, pot_args) stream (integrateFullOrbit.c:69-1040,
   integratePlanarOrbit.c:55-742 restricted to types 0/5/7/8/9/10/12/14/15/
   16/17/18/20/29 (planar)/33/34/35/40/41/46).
   Returns 0, or -1 for an unsupported type. */
static int is_wrapper(int type)
{
  return type == PT_WRAP_SMOOTH || type == PT_WRAP_ROTATE || type == PT_WRAP_GAUSS ||
         type == PT_WRAP_KUZMIN || type == PT_WRAP_COROT;
}

/* n entries of the (type, args) streams into P->c from *idx on; a wrapper
   (parse_leapFuncArgs_Full's nwrapped recursion, integrateFullOrbit.c:
   1010-1018) is followed by its wrapped entries and records their count */
static int decode_entries(opot *P, int *idx, int n, const int **type, const double **args,
                          int planar)
{
  for (int e = 0; e < n; e++) {
    if (*idx >= OMAXPOT) return -1;
    const int t = *(*type)++;
    ocomp *c = &P->c[(*idx)++];
    c->type = t;
    c->t = 0.;
    c->nsub = 0;
    for (int k = 0; k < 9; k++) c->p[k] = 0.;
    if (is_wrapper(t)) {
      const int nw = (int)*(*args)++;
      const int first = *idx;
      if (nw < 1 || decode_entries(P, idx, nw, type, args, planar)) return -1;
      c->nsub = *idx - first;
      const int na = t == PT_WRAP_SMOOTH ? 4 : t == PT_WRAP_COROT ? 5 : 3;
      for (int k = 0; k < na; k++) c->p[k] = (*args)[k];
      c->ea = *args;
      *args += na;
      continue;
    }
    const double *a = *args;
    int na = is_ellipsoidal(t)    ? ell_nargs(a)
             : t == PT_SCF         ? scf_nargs(a)
             : t == PT_SPIRALARMS  ? 10 + (int)a[0]
                                   : nargs_of(t, planar);
    if (na < 0) return -1;
    c->ea = a;
    for (int k = 0; k < na && k < 9; k++) c->p[k] = a[k];
    *args += na;
  }
  return 0;
}

static int opot_decode(opot *P, int npot, const int *type, const double *args, int planar)
{
  if (npot > OMAXPOT || npot < 1) return -1;
  P->planar = planar;
  P->nforce = 0;
  P->t = 0.;
  int idx = 0;
  if (decode_entries(P, &idx, npot, &type, &args, planar)) return -1;
  P->n = idx;
  return 0;
}

/* PowerSphericalPotentialwCutoff enclosed mass (PSwC.c:9-11) */
static double pswc_mass(double r2, double alpha, double rc)
{
  return 2. * M_PI * pow(rc, 3. - alpha) *
         (tgamma(1.5 - 0.5 * alpha) * oracle_gamma_inc_P(1.5 - 0.5 * alpha, r2 / rc / rc));
}

/* spherical force factor with the (r^2, force) cache of PSwC.c:25-46 */
static double pswc_force_factor(ocomp *c, double r2)
{
  if (r2 == c->p[3]) return c->p[4];
  double f = -c->p[0] * pswc_mass(r2, c->p[1], c->p[2]) / pow(r2, 1.5);
  c->p[3] = r2;
  c->p[4] = f;
  return f;
}

static double pswc_planarRforce(const ocomp *c, double R)
{
  double r2 = R * R;
  return -c->p[0] * pswc_mass(r2, c->p[1], c->p[2]) / r2;
}

static double pswc_planarR2deriv(const ocomp *c, double R)
{
  double amp = c->p[0], alpha = c->p[1], rc = c->p[2], r2 = R * R;
  return amp * (4. * M_PI * pow(r2, -0.5 * alpha) * exp(-r2 / rc / rc) -
                2. * pswc_mass(r2, alpha, rc) / pow(r2, 1.5));
}

/* LogHalo helper: R_t^2 of the triaxial form */
static double lh_Rt2(const ocomp *c, double R, double phi)
{
  return R * R * (1. - c->p[3] * pow(sin(phi), 2));
}

/* ---- the ellipsoidal family ---- */
/* the density function m -> rho(m) (mdens), its derivative (mdensDeriv) and
   psi of each member, from its psi args */
static double ell_dens(int type, double m, const double *a)
{
  double mpa, m2;
  switch (type) {
  case PT_TRIHERNQUIST: mpa = m + a[0]; return a[1] * pow(mpa, -3) / m;
  case PT_TRIJAFFE: mpa = m + a[0]; return a[1] * a[1] * pow(m * mpa, -2);
  case PT_TRINFW: mpa = m + a[0]; return a[1] / m / mpa / mpa;
  case PT_TWOPOWERTRI: mpa = m / a[0] + 1.0; return pow(a[0] / m, a[1]) / pow(mpa, a[3]);
  case PT_PERFECTELL: m2 = m * m; return 1. / (a[0] + m2) / (a[0] + m2);
  case PT_TRIGAUSS: return exp(m * m / a[0]);
  default: m2 = m * m; return pow(m2, -a[0] / 2.); /* PowerTriaxial */
  }
}

static double ell_densderiv(int type, double m, const double *a)
{
  double mpa, m2, md;
  switch (type) {
  case PT_TRIHERNQUIST:
    mpa = m + a[0];
    return -a[1] * (a[0] + 4. * m) / m / m * pow(mpa, -4);
  case PT_TRIJAFFE:
    mpa = m + a[0];
    return -2. * a[1] * a[1] * (a[0] + 2. * m) * pow(m * mpa, -3);
  case PT_TRINFW:
    mpa = m + a[0];
    return -a[1] * (a[0] + 3. * m) / m / m * pow(mpa, -3);
  case PT_TWOPOWERTRI:
    mpa = m + a[0];
    md = pow(a[0] / m, a[1]) / pow(mpa / a[0], a[3]);
    return -md * (a[0] * a[1] + a[2] * m) / m / mpa;
  case PT_PERFECTELL: m2 = m * m; return -4. * m * pow(a[0] + m2, -3);
  case PT_TRIGAUSS: return 2. * m / a[0] * exp(m * m / a[0]);
  default: m2 = m * m; return -a[0] * pow(m2, (-a[0] - 1.) / 2.);
  }
}

/* psi(m); TwoPowerTriaxial's needs the Gauss hypergeometric function 2F1,
   which this restatement does not carry: NaN */
static double ell_psi(int type, double m, const double *a)
{
  double mpa, m2;
  switch (type) {
  case PT_TRIHERNQUIST: mpa = m + a[0]; return -a[1] / mpa / mpa;
  case PT_TRIJAFFE: mpa = m + a[0]; return 2. * a[1] * (a[0] / mpa + log(m / mpa));
  case PT_TRINFW: mpa = m + a[0]; return -2. * a[1] / mpa;
  case PT_PERFECTELL: m2 = m * m; return -1. / (a[0] + m2);
  case PT_TRIGAUSS: return a[0] * exp(m * m / a[0]);
  case PT_POWERTRI: m2 = m * m; return 2. / (2. - a[0]) * pow(m2, 1. - a[0] / 2.);
  default: return NAN;
  }
}

typedef struct {
  const double *psi, *rot, *glx, *glw;
  double b2, c2;
  int aligned, glorder;
} oell;

static oell ell_args(const ocomp *c)
{
  oell e;
  const double *a = c->ea, *p = a + 17 + (int)a[16];
  e.psi = a + 17;
  e.b2 = p[0];
  e.c2 = p[1];
  e.aligned = p[2] != 0.;
  e.rot = p + 3;
  e.glorder = (int)p[12];
  e.glx = p + 13;
  e.glw = p + 13 + e.glorder;
  return e;
}

/* x' = rot x (galpy_potentials.c rotate) and F = rot^T F' (rotate_force) */
static void ell_rotate(const double *r, double *x, double *y, double *z)
{
  double xp = r[0] * *x + r[1] * *y + r[2] * *z;
  double yp = r[3] * *x + r[4] * *y + r[5] * *z;
  double zp = r[6] * *x + r[7] * *y + r[8] * *z;
  *x = xp;
  *y = yp;
  *z = zp;
}

static void ell_rotate_back(const double *r, double *x, double *y, double *z)
{
  double xp = r[0] * *x + r[3] * *y + r[6] * *z;
  double yp = r[1] * *x + r[4] * *y + r[7] * *z;
  double zp = r[2] * *x + r[5] * *y + r[8] * *z;
  *x = xp;
  *y = yp;
  *z = zp;
}

/* Cartesian force per unit amp (EllipsoidalPotentialxyzforces_xyz) */
static void ell_forces(const ocomp *c, double x, double y, double z, double F[3])
{
  oell e = ell_args(c);
  if (!e.aligned) ell_rotate(e.rot, &x, &y, &z);
  F[0] = F[1] = F[2] = 0.;
  for (int i = 0; i < e.glorder; i++) {
    double t = 1. / e.glx[i] / e.glx[i] - 1.;
    double td = e.glw[i] * ell_dens(c->type, sqrt(x * x / (1. + t) + y * y / (e.b2 + t) +
                                                  z * z / (e.c2 + t)), e.psi);
    F[0] += td * x / (1. + t);
    F[1] += td * y / (e.b2 + t);
    F[2] += td * z / (e.c2 + t);
  }
  if (!e.aligned) ell_rotate_back(e.rot, &F[0], &F[1], &F[2]);
}

/* Cartesian second derivatives per unit amp (xx, xy, xz, yy, yz, zz) at the
   unrotated point, as EllipsoidalPotential_2ndderiv_xyz_all is called */
static void ell_hess_xyz(const ocomp *c, double x, double y, double z, double h[6])
{
  oell e = ell_args(c);
  double x2 = x * x, y2 = y * y, z2 = z * z;
  for (int k = 0; k < 6; k++) h[k] = 0.;
  for (int i = 0; i < e.glorder; i++) {
    double s = e.glx[i], t = 1. / s / s - 1.;
    double t1 = 1. + t, t2 = e.b2 + t, t3 = e.c2 + t;
    double m = sqrt(x2 / t1 + y2 / t2 + z2 / t3);
    double dv = e.glw[i] * ell_dens(c->type, m, e.psi);
    double dd = e.glw[i] * ell_densderiv(c->type, m, e.psi) / m;
    double xt = x / t1, yt = y / t2, zt = z / t3;
    h[0] -= dd * xt * xt + dv / t1;
    h[1] -= dd * xt * yt;
    h[2] -= dd * xt * zt;
    h[3] -= dd * yt * yt + dv / t2;
    h[4] -= dd * yt * zt;
    h[5] -= dd * zt * zt + dv / t3;
  }
}

/* which: 0 Rforce, 1 zforce, 2 phitorque (EllipsoidalPotentialRforce ...) */
static double ell_cyl_force(const ocomp *c, int which, double R, double Z, double phi)
{
  double F[3];
  ell_forces(c, R * cos(phi), R * sin(phi), Z, F);
  if (which == 0) return c->p[0] * (cos(phi) * F[0] + sin(phi) * F[1]);
  if (which == 1) return c->p[0] * F[2];
  return c->p[0] * R * (-sin(phi) * F[0] + cos(phi) * F[1]);
}

/* 3D Hessian terms, which = 0 R2, 1 z2, 2 Rz, 3 phi2, 4 Rphi, 5 zphi
   (EllipsoidalPotentialR2deriv ... zphideriv) */
static double ell_cyl_hess(const ocomp *c, int which, double R, double Z, double phi)
{
  double amp = c->p[0], x = R * cos(phi), y = R * sin(phi), h[6], F[3];
  double cp, sp;
  ell_hess_xyz(c, x, y, Z, h);
  cp = cos(phi);
  sp = sin(phi);
  switch (which) {
  case 0: return amp * (cp * cp * h[0] + sp * sp * h[3] + 2. * cp * sp * h[1]);
  case 1: return amp * h[5];
  case 2: return amp * (cp * h[2] + sp * h[4]);
  case 5: return amp * R * (cp * h[4] - sp * h[2]);
  }
  ell_forces(c, x, y, Z, F);
  if (which == 3)
    return amp * (R * R * (sp * sp * h[0] + cp * cp * h[3] - 2. * cp * sp * h[1]) +
                  R * (cp * F[0] + sp * F[1]));
  return amp * (R * (cp * sp * (h[3] - h[0]) + cos(2. * phi) * h[1]) + sp * F[0] - cp * F[1]);
}

/* EllipsoidalPotentialEval */
static double ell_eval(const ocomp *c, double R, double Z, double phi)
{
  oell e = ell_args(c);
  double x = R * cos(phi), y = R * sin(phi), z = Z, out = 0.;
  if (!e.aligned) ell_rotate(e.rot, &x, &y, &z);
  for (int i = 0; i < e.glorder; i++) {
    double s = 1. / e.glx[i] / e.glx[i] - 1.;
    out += e.glw[i] * ell_psi(c->type, sqrt(x * x / (1. + s) + y * y / (e.b2 + s) +
                                            z * z / (e.c2 + s)), e.psi);
  }
  return -0.5 * c->p[0] * out;
}

/* ---- DehnenBarPotential (DehnenBarPotential.c:5-314) ---- */
/* bar growth factor (dehnenBarSmooth): 0 before tform, the quintic
   3/16 xi^5 - 5/8 xi^3 + 15/16 xi + 1/2 of xi = 2 (t - tform) / (tsteady -
   tform) - 1 until tsteady, 1 after */
static double dbar_smooth(double t, double tform, double tsteady)
{
  if (t < tform) return 0.;
  if (t < tsteady) {
    double xi = 2. * (t - tform) / (tsteady - tform) - 1.;
    return 3. / 16. * pow(xi, 5.) - 5. / 8. * pow(xi, 3.) + 15. / 16. * xi + .5;
  }
  return 1.;
}

/* args: p0 amp, p1 tform, p2 tsteady, p3 rb, p4 omegab, p5 barphi;
   which: 0 Rforce, 1 zforce, 2 phitorque (3D) */
static double dbar_force3(const ocomp *c, int which, double R, double z, double phi)
{
  double amp = c->p[0], rb = c->p[3], t = c->t;
  double sm = dbar_smooth(t, c->p[1], c->p[2]);
  double ang = 2. * (phi - c->p[4] * t - c->p[5]);
  double r2 = R * R + z * z, r = sqrt(r2);
  if (which == 0) {
    if (r <= rb)
      return -amp * sm * cos(ang) * (pow(r / rb, 3.) * R * (3. * R * R + 2. * z * z) - 4. * R * z * z) /
             pow(r, 4.);
    return -amp * sm * cos(ang) * pow(rb / r, 3.) * R / pow(r, 4) * (3. * R * R - 2. * z * z);
  }
  if (which == 1) {
    if (r <= rb) return -amp * sm * cos(ang) * (pow(r / rb, 3.) + 4.) * R * R * z / pow(r, 4.);
    return -5. * amp * sm * cos(ang) * pow(rb / r, 3.) * R * R * z / pow(r, 4);
  }
  if (r <= rb) return 2. * amp * sm * sin(ang) * (pow(r / rb, 3.) - 2.) * R * R / r2;
  return -2. * amp * sm * sin(ang) * pow(rb / r, 3.) * R * R / r2;
}

/* planar: which 0 Rforce, 2 phitorque */
static double dbar_force2(const ocomp *c, int which, double R, double phi)
{
  double amp = c->p[0], rb = c->p[3], t = c->t;
  double sm = dbar_smooth(t, c->p[1], c->p[2]);
  double ang = 2. * (phi - c->p[4] * t - c->p[5]);
  if (which == 0) {
    if (R <= rb) return -3. * amp * sm * cos(ang) * pow(R / rb, 3.) / R;
    return -3. * amp * sm * cos(ang) * pow(rb / R, 3.) / R;
  }
  if (R <= rb) return 2. * amp * sm * sin(ang) * (pow(R / rb, 3.) - 2.);
  return -2. * amp * sm * sin(ang) * pow(rb / R, 3.);
}

/* planar second derivatives of the potential: which 0 R2, 1 phi2, 2 Rphi */
static double dbar_hess2(const ocomp *c, int which, double R, double phi)
{
  double amp = c->p[0], rb = c->p[3], t = c->t;
  double sm = dbar_smooth(t, c->p[1], c->p[2]);
  double ang = 2. * (phi - c->p[4] * t - c->p[5]);
  int in = R <= rb;
  if (which == 0)
    return in ? 6. * amp * sm * cos(ang) * pow(R / rb, 3.) / R / R
              : -12. * amp * sm * cos(ang) * pow(rb / R, 3.) / R / R;
  if (which == 1)
    return in ? -4. * amp * sm * cos(ang) * (pow(R / rb, 3.) - 2.)
              : 4. * amp * sm * cos(ang) * pow(rb / R, 3.);
  return in ? -6. * amp * sm * sin(ang) * pow(R / rb, 3.) / R
            : -6. * amp * sm * sin(ang) * pow(rb / R, 3.) / R;
}

/* 3D second derivatives: which 0 R2, 1 z2, 2 Rz, 3 phi2, 4 Rphi, 5 zphi */
static double dbar_hess3(const ocomp *c, int which, double R, double z, double phi)
{
  double amp = c->p[0], rb = c->p[3], t = c->t;
  double sm = dbar_smooth(t, c->p[1], c->p[2]);
  double ang = 2. * (phi - c->p[4] * t - c->p[5]);
  double R2 = R * R, z2 = z * z, r2 = R2 + z2, r4 = r2 * r2, r6 = r4 * r2;
  int in = r2 <= rb * rb;
  double pre;
  switch (which) {
  case 0:
    pre = amp * sm * cos(ang);
    if (in)
      return pre * (pow(r2, 1.5) / (rb * rb * rb) * ((9. * R2 + 2. * z2) / r4 - R2 / r6 * (3. * R2 + 2. * z2)) +
                    4. * z2 / r6 * (4. * R2 - r2));
    return pre * pow(rb, 3.) * pow(r2, -1.5) / r6 * ((r2 - 7. * R2) * (3. * R2 - 2. * z2) + 6. * R2 * r2);
  case 1:
    pre = amp * sm * cos(ang);
    if (in) return pre * R2 / r6 * (pow(r2, 1.5) / (rb * rb * rb) * (r2 - z2) + 4. * (r2 - 4. * z2));
    return pre * 5. * pow(rb, 3.) * pow(r2, -1.5) * R2 / r6 * (r2 - 7. * z2);
  case 2:
    pre = amp * sm * cos(ang);
    if (in) return pre * R * z / r6 * (pow(r2, 1.5) / (rb * rb * rb) * (2. * r2 - R2) + 8. * (r2 - 2. * R2));
    return pre * 5. * pow(rb, 3.) * pow(r2, -1.5) * R * z / r6 * (2. * r2 - 7. * R2);
  case 3:
    pre = 4. * amp * sm * cos(ang);
    if (in) return -pre * (pow(r2, 1.5) / (rb * rb * rb) - 2.) * R2 / r2;
    return pre * pow(rb, 3.) * pow(r2, -1.5) * R2 / r2;
  case 4:
    pre = -2. * amp * sm * sin(ang);
    if (in) return pre * (pow(r2, 1.5) / (rb * rb * rb) * R * (3. * R2 + 2. * z2) - 4. * R * z2) / r4;
    return pre * pow(rb, 3.) * pow(r2, -1.5) * R / r4 * (3. * R2 - 2. * z2);
  default:
    pre = -2. * amp * sm * sin(ang);
    if (in) return pre * (pow(r2, 1.5) / (rb * rb * rb) + 4.) * R2 * z / r4;
    return pre * 5. * pow(rb, 3.) * pow(r2, -1.5) * R2 * z / r4;
  }
}

/* ---- SCFPotential (SCFPotential.c:181-1025), static coefficients ---- */
/* Hernquist-Ostriker expansion Phi = sqrt(4 pi) sum_{nlm} (Acos cos m phi +
   Asin sin m phi) phiTilde_nl(r) P_l^m(cos theta) with phiTilde_nl =
   -(a r)^l / (a + r)^(2l+1) C_n^(2l+3/2)(xi), xi = (r - a)/(r + a).  The
   Gegenbauer and associated Legendre functions (GSL's in the reference) are
   this file's own three-term recurrences (DLMF 18.9.1, 14.10.3), checked
   against scipy in the tests. */
/* C_n^lam(x), n = 0..nmax: (n+1) C_{n+1} = 2 (n + lam) x C_n - (n + 2 lam - 1) C_{n-1} */
static void scf_gegen(int nmax, double lam, double x, double *C)
{
  C[0] = 1.;
  if (nmax >= 1) C[1] = 2. * lam * x;
  for (int n = 1; n < nmax; n++)
    C[n + 1] = (2. * (n + lam) * x * C[n] - (n + 2. * lam - 1.) * C[n - 1]) / (n + 1.);
}

/* P_l^m(x) with the Condon-Shortley phase for 0 <= m <= l < L (m < M) in
   the triangle layout l (l + 1) / 2 + m, and dP/dx, by the upward
   recurrences (l - m) P_l^m = (2l - 1) x P_{l-1}^m - (l + m - 1) P_{l-2}^m
   from P_m^m = (-1)^m (2m - 1)!! (1 - x^2)^(m/2), and (x^2 - 1) dP_l^m/dx =
   l x P_l^m - (l + m) P_{l-1}^m */
static void scf_legendre(double x, int L, int M, double *P, double *dP)
{
  double s = sqrt((1. - x) * (1. + x)), pmm = 1.;
  for (int m = 0; m < M && m < L; m++) {
    if (m > 0) pmm *= -(2. * m - 1.) * s;
    double pm2 = 0., pm1 = pmm;
    for (int l = m; l < L; l++) {
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
      if (dP) dP[i] = (l * x * p - (l + m) * prev) / (x * x - 1.);
      if (l > m) {
        pm2 = pm1;
        pm1 = p;
      }
    }
  }
}

typedef struct {
  double a;
  int nonaxi, N, L, M;
  const double *Acos, *Asin;
} oscf;

static oscf scf_args(const ocomp *c)
{
  oscf d;
  const double *a = c->ea;
  d.a = a[0];
  d.nonaxi = (int)a[1];
  d.N = (int)a[2];
  d.L = (int)a[3];
  d.M = (int)a[4];
  d.Acos = a + 6;
  d.Asin = d.nonaxi ? a + 6 + d.N * d.L * d.M : NULL;
  return d;
}

/* Spherical quantities at (r, theta, phi), summed as the reference sums
   them (sum_spher_forces, sum_expansion, sum_spher_full): F[0..2] the forces
   -dPhi/dr, -dPhi/dtheta, -dPhi/dphi, F[3] Phi and, if hess, H[0..7] =
   dPhi/dr, dPhi/dtheta, d2/dr2, d2/dtheta2, d2/drdtheta, d2/dphi2,
   d2/drdphi, d2/dthetadphi */
static void scf_spher(const ocomp *c, double r, double theta, double phi, int hess, double *F,
                      double *H)
{
  oscf d = scf_args(c);
  int N = d.N, L = d.L, M = d.M, Me = d.nonaxi ? M : 1;
  double a = d.a, xi = (r - a) / (r + a), ar = a + r;
  double C[SCF_MAXL][SCF_MAXN], dC[SCF_MAXL][SCF_MAXN], d2C[SCF_MAXL][SCF_MAXN];
  double phiT[SCF_MAXL][SCF_MAXN], dphiT[SCF_MAXL][SCF_MAXN], d2phiT[SCF_MAXL][SCF_MAXN];
  for (int l = 0; l < L; l++) {
    double tmp[SCF_MAXN];
    scf_gegen(N - 1, 1.5 + 2 * l, xi, C[l]);
    dC[l][0] = 0.;
    if (N > 1) {
      scf_gegen(N - 2, 2.5 + 2 * l, xi, tmp);
      for (int n = 1; n < N; n++) dC[l][n] = tmp[n - 1];
    }
    for (int n = 0; n < N; n++) dC[l][n] *= 2.0 * (2 * l + 1.5);
    d2C[l][0] = 0.;
    if (N > 1) d2C[l][1] = 0.;
    if (N > 2) {
      scf_gegen(N - 3, 3.5 + 2 * l, xi, tmp);
      for (int n = 2; n < N; n++) d2C[l][n] = tmp[n - 2];
    }
    for (int n = 0; n < N; n++) d2C[l][n] *= 4.0 * (2 * l + 1.5) * (2 * l + 2.5);
  }
  /* radial functions (compute_phiTilde, compute_dphiTilde, compute_d2phiTilde) */
  double rt = -1.0 / (r + a), rt1 = 1.0 / (r * ar * ar * ar);
  double rt2 = 1.0 / (r * r * ar * ar * ar * ar * ar);
  for (int l = 0; l < L; l++) {
    if (l > 0) {
      rt *= r * a / ((a + r) * (a + r));
      rt1 *= a * r / (ar * ar);
      rt2 *= a * r / (ar * ar);
    }
    for (int n = 0; n < N; n++) {
      double ar2 = ar * ar, ar3 = ar2 * ar, ar4 = ar3 * ar;
      phiT[l][n] = rt * C[l][n];
      dphiT[l][n] = rt1 * (((2 * l + 1) * r * ar - l * ar * ar) * C[l][n] - 2.0 * a * r * dC[l][n]);
      d2phiT[l][n] = rt2 * (C[l][n] * (l * (1 - l) * ar4 - (4.0 * l * l + 6.0 * l + 2.0) * r * r * ar2 +
                                       l * (4 * l + 2) * r * ar3) +
                            a * r *
                                ((4.0 * r * r + 4.0 * a * r + (8 * l + 4) * r * ar - 4 * l * ar2) * dC[l][n] -
                                 4.0 * a * r * d2C[l][n]));
    }
  }
  /* angular functions; theta derivatives as legendre_theta_from_x */
  double P[SCF_MAXL * (SCF_MAXL + 1) / 2], dPx[SCF_MAXL * (SCF_MAXL + 1) / 2];
  double x = cos(theta), st = sin(theta), is2 = 1.0 / (st * st);
  scf_legendre(x, L, Me, P, dPx);
  double f0 = 0., f1 = 0., f2 = 0., pot = 0.;
  if (hess)
    for (int k = 0; k < 8; k++) H[k] = 0.;
  for (int l = 0; l < L; l++) {
    for (int m = 0; m <= l && m < Me; m++) {
      double mc = cos(m * phi), ms = sin(m * phi);
      int pi = l * (l + 1) / 2 + m;
      double dPt = -st * dPx[pi];
      double d2Pt = x * dPx[pi] - l * (l + 1) * P[pi] + (m ? m * m * is2 * P[pi] : 0.0);
      for (int n = 0; n < N; n++) {
        int ci = n * L * M + l * M + m;
        double ac = d.Acos[ci], as = d.nonaxi ? d.Asin[ci] : 0.;
        double cs = ac * mc + as * ms, sd = ac * ms - as * mc;
        f0 -= cs * P[pi] * dphiT[l][n];
        f1 -= cs * dPx[pi] * phiT[l][n];
        f2 += m * sd * P[pi] * phiT[l][n];
        pot += cs * P[pi] * phiT[l][n];
        if (hess) {
          double dsum = m * (as * mc - ac * ms);
          H[0] += cs * P[pi] * dphiT[l][n];
          H[1] += cs * dPt * phiT[l][n];
          H[2] += cs * P[pi] * d2phiT[l][n];
          H[3] += cs * d2Pt * phiT[l][n];
          H[4] += cs * dPt * dphiT[l][n];
          H[5] -= m * m * cs * P[pi] * phiT[l][n];
          H[6] += dsum * P[pi] * dphiT[l][n];
          H[7] += dsum * dPt * phiT[l][n];
        }
      }
    }
  }
  double s4 = sqrt(4.0 * M_PI);
  F[0] = f0 * s4;
  F[1] = f1 * (s4 * (-st));
  F[2] = f2 * s4;
  F[3] = pot * s4;
  if (hess)
    for (int k = 0; k < 8; k++) H[k] *= s4;
}

/* which: 0 Rforce, 1 zforce, 2 phitorque (SCFPotentialRforce / zforce / phitorque) */
static double scf_force3(const ocomp *c, int which, double R, double Z, double phi)
{
  double r = sqrt(R * R + Z * Z), theta = atan2(R, Z), F[4];
  scf_spher(c, r, theta, phi, 0, F, NULL);
  if (which == 0) return F[0] * (R / r) + F[1] * (Z / (r * r));
  if (which == 1) return F[0] * (Z / r) + F[1] * (-R / (r * r));
  return F[2];
}

/* 3D second derivatives (compute_scf_hessian_cyl): 0 R2, 1 z2, 2 Rz, 3 phi2, 4 Rphi, 5 zphi */
static double scf_hess3(const ocomp *c, int which, double R, double Z, double phi)
{
  double r = sqrt(R * R + Z * Z), theta = atan2(R, Z), F[4], S[8];
  scf_spher(c, r, theta, phi, 1, F, S);
  double Pr = S[0], Pth = S[1], Prr = S[2], Pthth = S[3], Prth = S[4];
  double Ppp = S[5], Prp = S[6], Pthp = S[7];
  double ir = 1.0 / r, ir2 = ir * ir, ir3 = ir2 * ir, ir4 = ir2 * ir2;
  double rR = R * ir, rz = Z * ir, thR = Z * ir2, thz = -R * ir2;
  double rRR = Z * Z * ir3, rzz = R * R * ir3, rRz = -R * Z * ir3;
  double thRR = -2.0 * R * Z * ir4, thzz = 2.0 * R * Z * ir4, thRz = (R * R - Z * Z) * ir4;
  switch (which) {
  case 0: return Prr * rR * rR + 2.0 * Prth * rR * thR + Pthth * thR * thR + Pr * rRR + Pth * thRR;
  case 1: return Prr * rz * rz + 2.0 * Prth * rz * thz + Pthth * thz * thz + Pr * rzz + Pth * thzz;
  case 2:
    return Prr * rR * rz + Prth * (rR * thz + rz * thR) + Pthth * thR * thz + Pr * rRz + Pth * thRz;
  case 3: return Ppp;
  case 4: return Prp * rR + Pthp * thR;
  default: return Prp * rz + Pthp * thz;
  }
}

/* planar second derivatives (compute_spher_2nd_derivs at Z = 0): 0 R2, 1 phi2, 2 Rphi */
static double scf_hess2(const ocomp *c, int which, double R, double phi)
{
  double F[4], S[8];
  scf_spher(c, R, atan2(R, 0.0), phi, 1, F, S);
  if (which == 0) return S[2];
  if (which == 1) return S[5];
  return S[6];
}

static double scf_eval(const ocomp *c, double R, double Z, double phi)
{
  double F[4];
  scf_spher(c, sqrt(R * R + Z * Z), atan2(R, Z), phi, 0, F, NULL);
  return F[3];
}

/* ---- planar disk perturbations (TransientLogSpiralPotential.c,
   SteadyLogSpiralPotential.c, EllipticalDiskPotential.c,
   LopsidedDiskPotential.c, CosmphiDiskPotential.c) ---- */
static int is_disk_pert(int type)
{
  return type == PT_TRANSPIRAL || type == PT_STEADYSPIRAL || type == PT_ELLDISK ||
         type == PT_LOPSIDED || type == PT_COSMPHI;
}

/* growth of the steady spiral and the elliptical disk (dehnenSpiralSmooth,
   EllipticalDiskSmooth): 1 when tform is NaN */
static double pert_smooth(double t, double tform, double tsteady)
{
  if (isnan(tform)) return 1.;
  return dbar_smooth(t, tform, tsteady);
}

/* which: 0 Rforce, 1 phitorque, 2 R2deriv, 3 phi2deriv, 4 Rphideriv */
static double disk_pert(const ocomp *c, int which, double R, double phi)
{
  const double *a = c->p, t = c->t, amp = a[0];
  switch (c->type) {
  case PT_TRANSPIRAL: {
    double A = a[1], to = a[2], sigma2 = a[3], alpha = a[4], m = a[5], om = a[6], gam = a[7];
    double g = exp(-pow(t - to, 2.) / 2. / sigma2);
    double chi = alpha * log(R) - m * (phi - om * t - gam);
    switch (which) {
    case 0: return amp * A * g / R * sin(chi);
    case 1: return -amp * A * g / alpha * m * sin(chi);
    case 2: return amp * A * g / R / R * (sin(chi) - alpha * cos(chi));
    case 3: return -amp * A * g / alpha * m * m * cos(chi);
    default: return amp * A * g * m / R * cos(chi);
    }
  }
  case PT_STEADYSPIRAL: {
    double A = a[3], alpha = a[4], m = a[5], om = a[6], gam = a[7];
    double sm = pert_smooth(t, a[1], a[2]);
    double chi = alpha * log(R) - m * (phi - om * t - gam);
    switch (which) {
    case 0: return amp * sm * A / R * sin(chi);
    case 1: return -amp * sm * A / alpha * m * sin(chi);
    case 2: return amp * sm * A / R / R * (sin(chi) - alpha * cos(chi));
    case 3: return -amp * sm * A / alpha * m * m * cos(chi);
    default: return amp * sm * A * m / R * cos(chi);
    }
  }
  case PT_ELLDISK: {
    double twophio = a[3], p = a[4], phib = a[5], sm = pert_smooth(t, a[1], a[2]);
    switch (which) {
    case 0: return -amp * sm * p * twophio / 2. * pow(R, p - 1.) * cos(2. * (phi - phib));
    case 1: return amp * sm * twophio * pow(R, p) * sin(2. * (phi - phib));
    case 2: return amp * sm * p * (p - 1) * twophio / 2. * pow(R, p - 2.) * cos(2. * (phi - phib));
    case 3: return -2. * amp * sm * twophio * pow(R, p) * cos(2. * (phi - phib));
    default: return -amp * sm * p * twophio * pow(R, p - 1.) * sin(2. * (phi - phib));
    }
  }
  case PT_LOPSIDED: {
    double phio = a[1], p = a[2], phib = a[3];
    switch (which) {
    case 0: return -amp * p * phio * pow(R, p - 1.) * cos(phi - phib);
    case 1: return amp * phio * pow(R, p) * sin(phi - phib);
    case 2: return amp * p * (p - 1) * phio * pow(R, p - 2.) * cos(phi - phib);
    case 3: return -amp * phio * pow(R, p) * cos(phi - phib);
    default: return -amp * p * phio * pow(R, p - 1.) * sin(phi - phib);
    }
  }
  default: { /* PT_COSMPHI */
    double mphio = a[1], p = a[2], mphib = a[3], rb = a[5], rbp = a[6], rb2p = a[7], r1p = a[8];
    int m = (int)a[4];
    int in = R <= rb;
    switch (which) {
    case 0:
      return in ? -amp * p * mphio / m * rb2p / pow(R, p + 1.) * cos(m * phi - mphib)
                : -amp * p * mphio / m * pow(R, p - 1.) * cos(m * phi - mphib);
    case 1:
      return in ? amp * mphio * rbp * (2. * r1p - rbp / pow(R, p)) * sin(m * phi - mphib)
                : amp * mphio * pow(R, p) * sin(m * phi - mphib);
    case 2:
      return in ? -amp * p * (p + 1) * mphio / m * rb2p / pow(R, p + 2.) * cos(m * phi - mphib)
                : amp * p * (p - 1) * mphio / m * pow(R, p - 2.) * cos(m * phi - mphib);
    case 3:
      return in ? -amp * m * mphio * rbp * (2. * r1p - rbp / pow(R, p)) * cos(m * phi - mphib)
                : -amp * m * mphio * pow(R, p) * cos(m * phi - mphib);
    default:
      return in ? -amp * p * mphio / m * rb2p / pow(R, p + 1) * sin(m * phi - mphib)
                : -amp * p * mphio * pow(R, p - 1.) * sin(m * phi - mphib);
    }
  }
  }
}

/* ---- SpiralArmsPotential: the potential (SpiralArmsPotentialEval) with
   its derivatives by second-order forward differentiation over (R, z, phi)
   (this file's own dual arithmetic); the reference differentiates by hand,
   so the two agree to rounding, not bit for bit ---- */
typedef struct {
  double v, g[3], h[3][3];
} odual;

static odual od_var(double v, int i)
{
  odual r;
  memset(&r, 0, sizeof(r));
  r.v = v;
  r.g[i] = 1.;
  return r;
}

static odual od_apply(odual u, double f, double f1, double f2)
{
  odual r;
  r.v = f;
  for (int a = 0; a < 3; a++) r.g[a] = f1 * u.g[a];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) r.h[a][b] = f1 * u.h[a][b] + f2 * u.g[a] * u.g[b];
  return r;
}

static odual od_mul(odual x, odual y)
{
  odual r;
  r.v = x.v * y.v;
  for (int a = 0; a < 3; a++) r.g[a] = x.g[a] * y.v + x.v * y.g[a];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      r.h[a][b] = x.h[a][b] * y.v + x.g[a] * y.g[b] + x.g[b] * y.g[a] + x.v * y.h[a][b];
  return r;
}

static odual od_lin(double ca, odual x, double c0)
{
  odual r = x;
  r.v = ca * x.v + c0;
  for (int a = 0; a < 3; a++) {
    r.g[a] = ca * x.g[a];
    for (int b = 0; b < 3; b++) r.h[a][b] = ca * x.h[a][b];
  }
  return r;
}

static odual od_rcp(odual u) { double i = 1. / u.v; return od_apply(u, i, -i * i, 2. * i * i * i); }
static odual od_exp(odual u) { double e = exp(u.v); return od_apply(u, e, e, e); }
static odual od_log(odual u) { double i = 1. / u.v; return od_apply(u, log(u.v), i, -i * i); }
static odual od_cos(odual u) { return od_apply(u, cos(u.v), -sin(u.v), -cos(u.v)); }
static odual od_cosh(odual u) { return od_apply(u, cosh(u.v), sinh(u.v), cosh(u.v)); }

/* Phi = -amp H exp(-(R - r_ref)/Rs) sum_n Cn / (Kn Dn) cos(n gamma) /
   cosh(Kn z / Bn)^Bn with the reference's gam, K, B, D */
static odual spiral_pot(const ocomp *c, double R, double z, double phi)
{
  const double *a = c->ea;
  int nC = (int)a[0];
  double amp = a[1], N = a[2], sa = a[3], ta = a[4], rref = a[5], phiref = a[6], Rs = a[7];
  double H = a[8], om = a[9], t = c->t;
  odual vR = od_var(R, 0), vz = od_var(z, 1), iR = od_rcp(vR);
  odual gam = od_lin(-N / ta, od_log(od_lin(1. / rref, vR, 0.)), 0.);
  gam.g[2] += N;
  gam.v += N * (phi - om * t - phiref);
  odual sum = od_lin(0., vR, 0.);
  for (int n = 1; n <= nC; n++) {
    double Cn = a[9 + n];
    odual Kn = od_lin(n * N / sa, iR, 0.), KH = od_lin(H, Kn, 0.);
    odual Bn = od_mul(KH, od_lin(0.4, KH, 1.));
    odual Dn = od_mul(od_lin(1., od_mul(KH, od_lin(0.3, KH, 1.)), 1.), od_rcp(od_lin(0.3, KH, 1.)));
    odual cs = od_cos(od_lin((double)n, gam, 0.));
    odual arg = od_mul(od_mul(Kn, vz), od_rcp(Bn));
    odual sech = od_exp(od_mul(od_lin(-1., Bn, 0.), od_log(od_cosh(arg))));
    odual term = od_mul(od_mul(cs, sech), od_rcp(od_mul(Kn, Dn)));
    sum.v += Cn * term.v;
    for (int i = 0; i < 3; i++) {
      sum.g[i] += Cn * term.g[i];
      for (int j = 0; j < 3; j++) sum.h[i][j] += Cn * term.h[i][j];
    }
  }
  return od_lin(-amp * H, od_mul(od_exp(od_lin(-1. / Rs, vR, rref / Rs)), sum), 0.);
}

/* ---- SoftenedNeedleBar: Phi = amp ln[(x - a + T-) / (x + a + T+)] / (2a)
   in the frame turning with the bar (angle pa + omegab t), T+- = sqrt((a +-
   x)^2 + y^2 + (b + sqrt(z^2 + c^2))^2).  Restated in the reference's
   arithmetic order (SoftenedNeedleBarPotential.c:5-72, 143-205) so results
   are bit-identical; its force cache only repeats the same values ---- */
typedef struct {
  double x, y, z, zc, Tp, Tm, cd, sd;
} oneedle;

static oneedle needle_frame(const ocomp *c, double R, double z, double phi)
{
  const double a = c->p[1], b = c->p[2], c2 = c->p[3], pa = c->p[4], om = c->p[5];
  oneedle f;
  double phid = phi - pa - om * c->t;
  f.cd = cos(phid);
  f.sd = sin(phid);
  f.x = R * f.cd;
  f.y = R * f.sd;
  f.z = z;
  double rest = f.y * f.y + pow(b + sqrt(z * z + c2), 2);
  f.Tp = sqrt(pow(a + f.x, 2) + rest);
  f.Tm = sqrt(pow(a - f.x, 2) + rest);
  f.zc = sqrt(z * z + c2);
  return f;
}

/* the force per unit amplitude in the inertial frame: out[0] x, [1] y, [2] z */
static void needle_xyz(const ocomp *c, double R, double z, double phi, double *out)
{
  const double b = c->p[2], pa = c->p[4], om = c->p[5];
  oneedle f = needle_frame(c, R, z, phi);
  double S = f.Tp + f.Tm;
  double fx = -2. * f.x / f.Tp / f.Tm / S;
  double fy = -f.y / 2. / f.Tp / f.Tm * (S - 4. * f.x * f.x / S) / (f.y * f.y + pow(b + f.zc, 2));
  double fz = -f.z / 2. / f.Tp / f.Tm * (S - 4. * f.x * f.x / S) /
              (f.y * f.y + pow(b + f.zc, 2)) * (b + f.zc) / f.zc;
  double ca = cos(pa + om * c->t), sa = sin(pa + om * c->t);
  out[0] = ca * fx - sa * fy;
  out[1] = sa * fx + ca * fy;
  out[2] = fz;
}

/* which: 0 Rforce, 1 zforce, 2 phitorque */
static double needle_force(const ocomp *c, int which, double R, double z, double phi)
{
  double F[3];
  needle_xyz(c, R, z, phi, F);
  if (which == 0) return c->p[0] * (cos(phi) * F[0] + sin(phi) * F[1]);
  if (which == 1) return c->p[0] * F[2];
  return c->p[0] * R * (-sin(phi) * F[0] + cos(phi) * F[1]);
}

/* cylindrical second derivatives (amp times): 0 R2, 1 z2, 2 phi2, 3 Rz,
   4 Rphi, 5 zphi, from the bar-frame Cartesian Hessian */
static double needle_hess(const ocomp *c, int which, double R, double z, double phi)
{
  const double amp = c->p[0], a = c->p[1], b = c->p[2], c2 = c->p[3];
  oneedle f = needle_frame(c, R, z, phi);
  double cd = f.cd, sd = f.sd, x = R * cd, y = R * sd;
  double zc = sqrt(z * z + c2), u = b + zc, s2 = y * y + u * u;
  double Tp3 = f.Tp * f.Tp * f.Tp, Tm3 = f.Tm * f.Tm * f.Tm;
  double G = (a - x) / f.Tm + (a + x) / f.Tp;
  double H = (a - x) / Tm3 + (a + x) / Tp3;
  double K = 1. / Tm3 - 1. / Tp3;
  double w = z * u / zc;
  double px = (1. / f.Tm - 1. / f.Tp) / 2. / a, py = y * G / 2. / a / s2;
  double pxx = H / 2. / a, pxy = -y * K / 2. / a, pxz = -w * K / 2. / a;
  double pyy = (G * (s2 - 2. * y * y) / s2 / s2 - y * y * H / s2) / 2. / a;
  double pyz = -y * w * (2. * G / s2 / s2 + H / s2) / 2. / a;
  double pzz = ((1. + b * c2 / zc / zc / zc) * G / s2 - w * w * (H / s2 + 2. * G / s2 / s2)) / 2. / a;
  double h;
  switch (which) {
  case 0: h = cd * cd * pxx + 2. * cd * sd * pxy + sd * sd * pyy; break;
  case 1: h = pzz; break;
  case 2:
    h = R * R * (sd * sd * pxx - 2. * sd * cd * pxy + cd * cd * pyy) - R * (cd * px + sd * py);
    break;
  case 3: h = cd * pxz + sd * pyz; break;
  case 4:
    h = R * (-sd * cd * pxx + (cd * cd - sd * sd) * pxy + sd * cd * pyy) - sd * px + cd * py;
    break;
  default: h = R * (-sd * pxz + cd * pyz); break;
  }
  return amp * h;
}

static double needle_eval(const ocomp *c, double R, double z, double phi)
{
  const double a = c->p[1];
  oneedle f = needle_frame(c, R, z, phi);
  return 0.5 * c->p[0] * log((f.x - a + f.Tm) / (f.x + a + f.Tp)) / a;
}

/* ---- 3D component forces ---- */
static double comp_Rforce(ocomp *c, double R, double Z, double phi)
{
  if (c->type == PT_SPIRALARMS) return -spiral_pot(c, R, Z, phi).g[0];
  if (c->type == PT_DEHNENBAR) return dbar_force3(c, 0, R, Z, phi);
  if (c->type == PT_NEEDLEBAR) return needle_force(c, 0, R, Z, phi);
  if (c->type == PT_SCF) return scf_force3(c, 0, R, Z, phi);
  if (is_new_spherical(c->type)) return sph_force3(c, R, Z, R);
  if (is_ellipsoidal(c->type)) return ell_cyl_force(c, 0, R, Z, phi);
  double amp = c->p[0];
  switch (c->type) {
  case PT_KUZMINDISK: /* KuzminDiskPotentialRforce */
    return -amp * R * pow(R * R + pow(c->p[1] + fabs(Z), 2.), -1.5);
  case PT_KKS:
    return kks_Rz(c, R, Z, 0);
  case PT_FLATPOWER: {
    double alpha = c->p[1], q2 = c->p[2], core2 = c->p[3], m2;
    if (alpha == 0.) return -amp * R / (R * R + Z * Z / q2 + core2);
    m2 = core2 + R * R + Z * Z / q2;
    return -amp * pow(m2, -0.5 * alpha - 1.) * R;
  }
  case PT_LOGHALO: {
    double q = c->p[1], cc = c->p[2], om = c->p[3], zq = Z / q;
    if (om < 1) {
      double Rt2 = lh_Rt2(c, R, phi);
      return -amp * Rt2 / R / (Rt2 + zq * zq + cc);
    }
    return -amp * R / (R * R + zq * zq + cc);
  }
  case PT_MN: {
    double a = c->p[1], b = c->p[2];
    return -amp * R * pow(R * R + pow(a + pow(Z * Z + b * b, 0.5), 2.), -1.5);
  }
  case PT_HERNQUIST: {
    double a = c->p[1], sq = pow(R * R + Z * Z, 0.5);
    return -amp * R / a / sq * pow(1. + sq / a, -2.) / 2. / a;
  }
  case PT_NFW: {
    double a = c->p[1], Rz = R * R + Z * Z, sq = pow(Rz, 0.5);
    return amp * R * (1. / Rz / (a + sq) - log(1. + sq / a) / sq / Rz);
  }
  case PT_PSWC:
    return pswc_force_factor(c, R * R + Z * Z) * R;
  }
  return 0.;
}

static double comp_zforce(ocomp *c, double R, double Z, double phi)
{
  if (c->type == PT_SPIRALARMS) return -spiral_pot(c, R, Z, phi).g[1];
  if (c->type == PT_DEHNENBAR) return dbar_force3(c, 1, R, Z, phi);
  if (c->type == PT_NEEDLEBAR) return needle_force(c, 1, R, Z, phi);
  if (c->type == PT_SCF) return scf_force3(c, 1, R, Z, phi);
  if (is_new_spherical(c->type)) return sph_force3(c, R, Z, Z);
  if (is_ellipsoidal(c->type)) return ell_cyl_force(c, 1, R, Z, phi);
  double amp = c->p[0];
  switch (c->type) {
  case PT_KUZMINDISK: { /* KuzminDiskPotentialzforce */
    double zsign = (Z > 0) - (Z < 0), a = c->p[1];
    return -zsign * amp * pow(R * R + pow(a + fabs(Z), 2.), -1.5) * (a + fabs(Z));
  }
  case PT_KKS:
    return kks_Rz(c, R, Z, 1);
  case PT_FLATPOWER: {
    double alpha = c->p[1], q2 = c->p[2], core2 = c->p[3], m2;
    if (alpha == 0.) return -amp * Z / q2 / (R * R + Z * Z / q2 + core2);
    m2 = core2 + R * R + Z * Z / q2;
    return -amp * pow(m2, -0.5 * alpha - 1.) * Z / q2;
  }
  case PT_LOGHALO: {
    double q = c->p[1], cc = c->p[2], om = c->p[3], zq = Z / q;
    if (om < 1) {
      double Rt2 = lh_Rt2(c, R, phi);
      return -amp * zq / q / (Rt2 + zq * zq + cc);
    }
    return -amp * zq / q / (R * R + zq * zq + cc);
  }
  case PT_MN: {
    double a = c->p[1], b = c->p[2];
    double sqrtbz = pow(b * b + Z * Z, .5), asqrtbz = a + sqrtbz;
    if (a == 0.) return amp * (-Z * pow(R * R + asqrtbz * asqrtbz, -1.5));
    return amp * (-Z * asqrtbz / sqrtbz * pow(R * R + asqrtbz * asqrtbz, -1.5));
  }
  case PT_HERNQUIST: {
    double a = c->p[1], sq = pow(R * R + Z * Z, 0.5);
    return -amp * Z / a / sq * pow(1. + sq / a, -2.) / 2. / a;
  }
  case PT_NFW: {
    double a = c->p[1], Rz = R * R + Z * Z, sq = pow(Rz, 0.5);
    return amp * Z * (1. / Rz / (a + sq) - log(1. + sq / a) / sq / Rz);
  }
  case PT_PSWC:
    return pswc_force_factor(c, R * R + Z * Z) * Z;
  }
  return 0.;
}

static double comp_phitorque(const ocomp *c, double R, double Z, double phi)
{
  if (c->type == PT_SPIRALARMS) return -spiral_pot(c, R, Z, phi).g[2];
  if (c->type == PT_DEHNENBAR) return dbar_force3(c, 2, R, Z, phi);
  if (c->type == PT_NEEDLEBAR) return needle_force(c, 2, R, Z, phi);
  if (c->type == PT_SCF) return scf_force3(c, 2, R, Z, phi);
  if (is_ellipsoidal(c->type)) return ell_cyl_force(c, 2, R, Z, phi);
  if (c->type == PT_LOGHALO && c->p[3] < 1) {
    double amp = c->p[0], q = c->p[1], cc = c->p[2], om = c->p[3];
    double zq = Z / q, Rt2 = lh_Rt2(c, R, phi);
    return amp * R * R / (Rt2 + zq * zq + cc) * sin(2 * phi) * om / 2.;
  }
  return 0.;
}

/* spherical potentials: Phi'(r)/amp and Phi''(r)/amp as in the reference */
static void sph_derivs(const ocomp *c, double r, double *dphi, double *d2phi)
{
  double a = c->p[1];
  if (c->type == PT_HERNQUIST) {
    *dphi = 1. / 2. / a / a * pow(1. + r / a, -2.);
    *d2phi = -1. / a / a / a * pow(1. + r / a, -3.);
  } else { /* NFW */
    *dphi = log(1. + r / a) / r / r - 1. / r / (a + r);
    double ar = a + r;
    *d2phi = (r * (2. * a + 3. * r) - 2. * ar * ar * log(1. + r / a)) / r / r / r / ar / ar;
  }
}

/* 3D Hessian terms: which = 0 R2, 1 z2, 2 Rz, 3 phi2, 4 Rphi, 5 zphi */
static double comp_hess(const ocomp *c, int which, double R, double Z, double phi)
{
  if (c->type == PT_SPIRALARMS) { /* R2, z2, Rz, phi2, Rphi, zphi */
    odual P = spiral_pot(c, R, Z, phi);
    static const int ia[6] = {0, 1, 0, 2, 0, 1}, ib[6] = {0, 1, 1, 2, 2, 2};
    return P.h[ia[which]][ib[which]];
  }
  if (c->type == PT_DEHNENBAR) return dbar_hess3(c, which, R, Z, phi);
  if (c->type == PT_NEEDLEBAR) { /* R2, z2, Rz, phi2, Rphi, zphi -> its order */
    static const int map[6] = {0, 1, 3, 2, 4, 5};
    return needle_hess(c, map[which], R, Z, phi);
  }
  if (c->type == PT_SCF) return scf_hess3(c, which, R, Z, phi);
  if (is_new_spherical(c->type)) return sph_hess3(c, which, R, Z);
  if (is_ellipsoidal(c->type)) return ell_cyl_hess(c, which, R, Z, phi);
  double amp = c->p[0];
  switch (c->type) {
  case PT_KUZMINDISK: { /* KuzminDiskPotentialR2deriv / z2deriv / Rzderiv */
    double zsign = (Z > 0) - (Z < 0), az = c->p[1] + fabs(Z), denom = R * R + az * az;
    double d15 = 1. / (denom * sqrt(denom)), d25 = 1. / (denom * denom * sqrt(denom));
    if (which == 0) return amp * (d15 - 3. * R * R * d15 / denom);
    if (which == 1) return amp * (d15 - 3. * az * az * d15 / denom);
    if (which == 2) return amp * (-3. * zsign * R * az * d25);
    return 0.;
  }
  case PT_KKS:
    return which > 2 ? 0. : kks_hess(c, R, Z, which);
  case PT_FLATPOWER: {
    double alpha = c->p[1], q2 = c->p[2], core2 = c->p[3], denom, m2;
    if (which > 2) return 0.;
    if (alpha == 0.) {
      denom = 1. / (R * R + Z * Z / q2 + core2);
      if (which == 0) return amp * (denom - 2. * R * R * denom * denom);
      if (which == 1) return amp / q2 * (denom - 2. * Z * Z * denom * denom / q2);
      return -2. * amp * R * Z / q2 * denom * denom;
    }
    m2 = core2 + R * R + Z * Z / q2;
    if (which == 0) return -amp * pow(m2, -0.5 * alpha - 1.) * ((alpha + 2.) * R * R / m2 - 1.);
    if (which == 1)
      return -amp / q2 * pow(m2, -0.5 * alpha - 1.) * ((alpha + 2.) * Z * Z / m2 / q2 - 1.);
    return -amp * (alpha + 2.) * R * Z / q2 * pow(m2, -0.5 * alpha - 2.);
  }
  case PT_LOGHALO: {
    double q = c->p[1], cc = c->p[2], om = c->p[3], zq = Z / q, q2 = q * q;
    double Rt2, denom;
    int tri = om < 1;
    switch (which) {
    case 0:
      if (tri) {
        Rt2 = lh_Rt2(c, R, phi);
        denom = 1. / (Rt2 + zq * zq + cc);
        return amp * (denom - 2. * Rt2 * denom * denom) * Rt2 / (R * R);
      }
      denom = 1. / (R * R + zq * zq + cc);
      return amp * (denom - 2. * R * R * denom * denom);
    case 1:
      Rt2 = tri ? lh_Rt2(c, R, phi) : R * R;
      denom = 1. / (Rt2 + zq * zq + cc);
      return amp * (denom / q2 - 2. * Z * Z * denom * denom / (q2 * q2));
    case 2:
      if (tri) {
        Rt2 = lh_Rt2(c, R, phi);
        denom = 1. / (Rt2 + zq * zq + cc);
        return -amp * 2. * Rt2 / R * Z / q2 * denom * denom;
      }
      denom = 1. / (R * R + zq * zq + cc);
      return -amp * 2. * R * Z / q2 * denom * denom;
    case 3:
      if (tri) {
        double R2 = R * R, s2phi;
        Rt2 = R2 * (1. - om * pow(sin(phi), 2));
        denom = 1. / (Rt2 + zq * zq + cc);
        s2phi = sin(2. * phi);
        return -amp * om * (0.5 * R2 * R2 * s2phi * s2phi * om * denom * denom +
                            R2 * denom * cos(2. * phi));
      }
      return 0.;
    case 4:
      if (tri) {
        Rt2 = lh_Rt2(c, R, phi);
        denom = 1. / (Rt2 + zq * zq + cc);
        return -amp * (denom - Rt2 * denom * denom) * R * sin(2. * phi) * om;
      }
      return 0.;
    case 5:
      if (tri) {
        Rt2 = lh_Rt2(c, R, phi);
        denom = 1. / (Rt2 + zq * zq + cc);
        return amp * 2. * R * R * Z * sin(phi) * cos(phi) * om * denom * denom / q2;
      }
      return 0.;
    }
    return 0.;
  }
  case PT_MN: {
    double a = c->p[1], b = c->p[2];
    switch (which) {
    case 0: {
      double sqrtbz = pow(b * b + Z * Z, 0.5), asqrtbz = a + sqrtbz;
      double denom = R * R + asqrtbz * asqrtbz;
      return amp * (pow(denom, -1.5) - 3. * R * R * pow(denom, -2.5));
    }
    case 1: {
      double b2 = b * b, sqrtbz = pow(b2 + Z * Z, 0.5), asqrtbz = a + sqrtbz;
      if (a == 0.) return amp * (b2 + R * R - 2. * Z * Z) * pow(b2 + R * R + Z * Z, -2.5);
      return amp *
             (a * a * a * b2 + a * a * (3. * b2 - 2. * Z * Z) * sqrtbz +
              (b2 + R * R - 2. * Z * Z) * pow(b2 + Z * Z, 1.5) +
              a * (3. * b2 * b2 - 4. * Z * Z * Z * Z + b2 * (R * R - Z * Z))) /
             (pow(b2 + Z * Z, 1.5) * pow(R * R + asqrtbz * asqrtbz, 2.5));
    }
    case 2: {
      double sqrtbz = pow(b * b + Z * Z, 0.5), asqrtbz = a + sqrtbz;
      if (a == 0.) return amp * (-3. * R * Z * pow(R * R + asqrtbz * asqrtbz, -2.5));
      return amp * (-3. * R * Z * asqrtbz / sqrtbz * pow(R * R + asqrtbz * asqrtbz, -2.5));
    }
    }
    return 0.;
  }
  case PT_HERNQUIST:
  case PT_NFW: {
    if (which > 2) return 0.;
    double r = sqrt(R * R + Z * Z), dphi, d2phi;
    sph_derivs(c, r, &dphi, &d2phi);
    if (which == 0) return amp * (d2phi * R * R / r / r + dphi * Z * Z / r / r / r);
    if (which == 1) return amp * (d2phi * Z * Z / r / r + dphi * R * R / r / r / r);
    return amp * R * Z * (d2phi / r / r - dphi / r / r / r);
  }
  case PT_PSWC: {
    if (which > 2) return 0.;
    double r2 = R * R + Z * Z, r = sqrt(r2);
    double Phipp = pswc_planarR2deriv(c, r);
    double Phip = -pswc_planarRforce(c, r);
    double ir2 = 1. / r2, ir3 = ir2 / r;
    if (which == 0) return Phipp * R * R * ir2 + Phip * Z * Z * ir3;
    if (which == 1) return Phipp * Z * Z * ir2 + Phip * R * R * ir3;
    return R * Z * (Phipp * ir2 - Phip * ir3);
  }
  }
  return 0.;
}

/* ---- planar component forces ---- */
static double comp_planarRforce(const ocomp *c, double R, double phi)
{
  if (c->type == PT_SPIRALARMS) return -spiral_pot(c, R, 0., phi).g[0];
  if (is_disk_pert(c->type)) return disk_pert(c, 0, R, phi);
  if (c->type == PT_DEHNENBAR) return dbar_force2(c, 0, R, phi);
  if (c->type == PT_NEEDLEBAR) return needle_force(c, 0, R, 0., phi);
  if (c->type == PT_SCF) return scf_force3(c, 0, R, 0.0, phi); /* SCFPotentialPlanarRforce */
  if (is_new_spherical(c->type)) return sph_planarRforce(c, R);
  if (is_ellipsoidal(c->type)) return ell_cyl_force(c, 0, R, 0., phi);
  double amp = c->p[0];
  switch (c->type) {
  case PT_KUZMINDISK: /* KuzminDiskPotentialPlanarRforce */
    return -amp * R * pow(R * R + c->p[1] * c->p[1], -1.5);
  case PT_HENONHEILES: /* HenonHeilesPotentialRforce */
    return -amp * R * (1. + R * sin(3. * phi));
  case PT_KKS: { /* KuzminKutuzovStaeckelPotentialPlanarRforce */
    double ac = c->p[1], Delta = c->p[2];
    double gamma = Delta * Delta / (1. - ac * ac), alpha = gamma - Delta * Delta;
    double l = R * R - alpha, n = -gamma, dldR = 2. * R;
    double dVdl = 0.5 / sqrt(l) / pow(sqrt(l) + sqrt(n), 2.);
    return -amp * dldR * dVdl;
  }
  case PT_FLATPOWER: {
    double alpha = c->p[1], core2 = c->p[2], m2;
    if (alpha == 0.) return -amp * R / (R * R + core2);
    m2 = core2 + R * R;
    return -amp * pow(m2, -0.5 * alpha - 1.) * R;
  }
  case PT_LOGHALO: {
    double cc = c->p[2], om = c->p[3];
    if (om < 1) {
      double Rt2 = lh_Rt2(c, R, phi);
      return -amp * Rt2 / R / (Rt2 + cc);
    }
    return -amp * R / (R * R + cc);
  }
  case PT_MN: {
    double a = c->p[1], b = c->p[2];
    return -amp * R * pow(R * R + pow(a + b, 2.), -1.5);
  }
  case PT_HERNQUIST: {
    double a = c->p[1];
    return -amp / a * pow(1. + R / a, -2.) / 2. / a;
  }
  case PT_NFW: {
    double a = c->p[1];
    return amp / R * (1. / (a + R) - log(1. + R / a) / R);
  }
  case PT_PSWC:
    return pswc_planarRforce(c, R);
  }
  return 0.;
}

static double comp_planarphitorque(const ocomp *c, double R, double phi)
{
  if (c->type == PT_SPIRALARMS) return -spiral_pot(c, R, 0., phi).g[2];
  if (is_disk_pert(c->type)) return disk_pert(c, 1, R, phi);
  if (c->type == PT_DEHNENBAR) return dbar_force2(c, 2, R, phi);
  if (c->type == PT_NEEDLEBAR) return needle_force(c, 2, R, 0., phi);
  if (c->type == PT_SCF) return scf_force3(c, 2, R, 0.0, phi);
  if (is_ellipsoidal(c->type)) return ell_cyl_force(c, 2, R, 0., phi);
  if (c->type == PT_HENONHEILES) /* HenonHeilesPotentialphitorque */
    return -c->p[0] * pow(R, 3.) * cos(3. * phi);
  if (c->type == PT_LOGHALO && c->p[3] < 1) {
    double amp = c->p[0], cc = c->p[2], om = c->p[3], Rt2 = lh_Rt2(c, R, phi);
    return amp * R * R / (Rt2 + cc) * sin(2 * phi) * om / 2.;
  }
  return 0.;
}

/* planar Hessian: which = 0 R2, 1 phi2, 2 Rphi */
static double comp_planarhess(const ocomp *c, int which, double R, double phi)
{
  if (c->type == PT_SPIRALARMS) { /* R2, phi2, Rphi */
    odual P = spiral_pot(c, R, 0., phi);
    return which == 0 ? P.h[0][0] : which == 1 ? P.h[2][2] : P.h[0][2];
  }
  if (is_disk_pert(c->type)) return disk_pert(c, 2 + which, R, phi);
  if (c->type == PT_DEHNENBAR) return dbar_hess2(c, which, R, phi);
  if (c->type == PT_NEEDLEBAR) return needle_hess(c, which == 0 ? 0 : which == 1 ? 2 : 4, R, 0., phi);
  if (c->type == PT_SCF) return scf_hess2(c, which, R, phi);
  if (is_new_spherical(c->type)) return which ? 0. : sph_planarR2deriv(c, R);
  if (is_ellipsoidal(c->type)) /* EllipsoidalPotentialPlanarR2deriv / phi2 / Rphi */
    return ell_cyl_hess(c, which == 0 ? 0 : which + 2, R, 0., phi);
  double amp = c->p[0];
  switch (c->type) {
  case PT_KUZMINDISK: { /* KuzminDiskPotentialPlanarR2deriv */
    double denom = R * R + c->p[1] * c->p[1];
    return which ? 0. : amp * (-pow(denom, -1.5) + 3 * R * R * pow(denom, -2.5));
  }
  case PT_HENONHEILES: /* HenonHeilesPotential R2deriv / phi2deriv / Rphideriv */
    if (which == 0) return amp * (1. + 2. * R * sin(3. * phi));
    if (which == 1) return -3. * amp * pow(R, 3.) * sin(3. * phi);
    return 3. * amp * R * R * cos(3. * phi);
  case PT_KKS: { /* KuzminKutuzovStaeckelPotentialPlanarR2deriv */
    if (which) return 0.;
    double ac = c->p[1], Delta = c->p[2];
    double gamma = Delta * Delta / (1. - ac * ac), alpha = gamma - Delta * Delta;
    double l = R * R - alpha, n = -gamma, dldR = 2. * R, d2ldR2 = 2.;
    double dVdl = 0.5 / sqrt(l) / pow(sqrt(l) + sqrt(n), 2.);
    double d2Vdl2 = (-3. * sqrt(l) - sqrt(n)) / (4. * pow(l, 1.5) * pow(sqrt(l) + sqrt(n), 3.));
    return amp * (d2ldR2 * dVdl + dldR * dldR * d2Vdl2);
  }
  case PT_FLATPOWER: {
    double alpha = c->p[1], core2 = c->p[2], m2;
    if (which) return 0.;
    if (alpha == 0.) return amp * (1. - 2. * R * R / (R * R + core2)) / (R * R + core2);
    m2 = core2 + R * R;
    return -amp * pow(m2, -0.5 * alpha - 1.) * ((alpha + 2.) * R * R / m2 - 1.);
  }
  case PT_LOGHALO: {
    double cc = c->p[2], om = c->p[3];
    int tri = om < 1;
    if (which == 0) {
      if (tri) {
        double Rt2 = lh_Rt2(c, R, phi);
        return amp * (1. - 2. * Rt2 / (Rt2 + cc)) / (Rt2 + cc) * Rt2 / R / R;
      }
      return amp * (1. - 2. * R * R / (R * R + cc)) / (R * R + cc);
    }
    if (!tri) return 0.;
    double Rt2 = lh_Rt2(c, R, phi);
    if (which == 1)
      return -amp * om *
             (0.5 * pow(R * R * sin(2. * phi), 2.) * om / (Rt2 + cc) / (Rt2 + cc) +
              R * R / (Rt2 + cc) * cos(2. * phi));
    return -amp * cc / (Rt2 + cc) / (Rt2 + cc) * R * sin(2. * phi) * om;
  }
  case PT_MN: {
    if (which) return 0.;
    double a = c->p[1], b = c->p[2], denom = R * R + pow(a + b, 2.);
    return amp * (pow(denom, -1.5) - 3. * R * R * pow(denom, -2.5));
  }
  case PT_HERNQUIST: {
    if (which) return 0.;
    double a = c->p[1];
    return -amp / a / a / a * pow(1. + R / a, -3.);
  }
  case PT_NFW: {
    if (which) return 0.;
    double a = c->p[1], aR = a + R, aR2 = aR * aR;
    return amp * (((R * (2. * a + 3. * R)) - 2. * aR2 * log(1. + R / a)) / R / R / R / aR2);
  }
  case PT_PSWC:
    return which ? 0. : pswc_planarR2deriv(c, R);
  }
  return 0.;
}

/* ---- potential values (for energies) ---- */
static double comp_eval(const ocomp *c, double R, double Z, double phi)
{
  if (c->type == PT_SPIRALARMS) return spiral_pot(c, R, Z, phi).v;
  if (c->type == PT_SCF) return scf_eval(c, R, Z, phi);
  if (c->type == PT_DEHNENBAR) return NAN; /* no C evaluation in the reference */
  if (c->type == PT_NEEDLEBAR) return needle_eval(c, R, Z, phi);
  if (is_new_spherical(c->type)) return sph_eval(c, R, Z);
  if (is_ellipsoidal(c->type)) return ell_eval(c, R, Z, phi);
  double amp = c->p[0];
  switch (c->type) {
  case PT_KUZMINDISK: /* KuzminDiskPotentialEval */
    return -amp * pow(R * R + pow(c->p[1] + fabs(Z), 2.), -0.5);
  case PT_HENONHEILES: /* galpy's HenonHeilesPotential._evaluate (no C Eval) */
    return amp * (0.5 * R * R + pow(R, 3.) * sin(3. * phi) / 3.);
  case PT_KKS: { /* KuzminKutuzovStaeckelPotentialEval */
    double ac = c->p[1], Delta = c->p[2];
    double gamma = Delta * Delta / (1. - ac * ac), alpha = gamma - Delta * Delta;
    double term = R * R + Z * Z - alpha - gamma;
    double discr = pow(R * R + Z * Z - Delta * Delta, 2.) + (4. * Delta * Delta * R * R);
    double l = 0.5 * (term + sqrt(discr)), n = 0.5 * (term - sqrt(discr));
    n = ((n > 0.) ? n : 0.);
    return -amp / (sqrt(l) + sqrt(n));
  }
  case PT_FLATPOWER: {
    double alpha = c->p[1], q2 = c->p[2], core2 = c->p[3];
    if (alpha == 0.) return 0.5 * amp * log(R * R + Z * Z / q2 + core2);
    return -amp * pow(core2 + R * R + Z * Z / q2, -0.5 * alpha) / alpha;
  }
  case PT_LOGHALO: {
    double q = c->p[1], cc = c->p[2], om = c->p[3], zq = Z / q;
    if (om < 1) return 0.5 * amp * log(R * R * (1. - om * pow(sin(phi), 2)) + zq * zq + cc);
    return 0.5 * amp * log(R * R + zq * zq + cc);
  }
  case PT_MN: {
    double a = c->p[1], b = c->p[2];
    return -amp * pow(R * R + pow(a + pow(Z * Z + b * b, 0.5), 2.), -0.5);
  }
  case PT_HERNQUIST: {
    double a = c->p[1], sq = pow(R * R + Z * Z, 0.5);
    return -amp / (1. + sq / a) / 2. / a;
  }
  case PT_NFW: {
    double a = c->p[1], sq = pow(R * R + Z * Z, 0.5);
    return -amp * log(1. + sq / a) / sq;
  }
  case PT_PSWC: {
    double alpha = c->p[1], rc = c->p[2], r2 = R * R + Z * Z, r = sqrt(r2);
    double a1 = 1. - 0.5 * alpha, a2 = 1.5 - 0.5 * alpha, x = r2 / rc / rc;
    double g1 = tgamma(a1), g2 = tgamma(a2);
    return amp * 2. * M_PI * pow(rc, 3. - alpha) / r *
           (r / rc * (g1 - g1 * oracle_gamma_inc_Q(a1, x)) - (g2 - g2 * oracle_gamma_inc_Q(a2, x)));
  }
  }
  return 0.;
}

/* ---- sums over components, through wrappers ---- */
/* Quantities summed over a range of entries: 3D forces and second
   derivatives, planar forces and second derivatives, potential values. */
enum { Q_RF, Q_ZF, Q_PT, Q_H0, Q_H1, Q_H2, Q_H3, Q_H4, Q_H5, Q_PRF, Q_PPT, Q_PH0, Q_PH1,
       Q_PH2, Q_EVAL };

static double comp_quantity(ocomp *c, int q, double R, double z, double phi)
{
  switch (q) {
  case Q_RF: return comp_Rforce(c, R, z, phi);
  case Q_ZF: return comp_zforce(c, R, z, phi);
  case Q_PT: return comp_phitorque(c, R, z, phi);
  case Q_PRF: return comp_planarRforce(c, R, phi);
  case Q_PPT: return comp_planarphitorque(c, R, phi);
  case Q_PH0: case Q_PH1: case Q_PH2: return comp_planarhess(c, q - Q_PH0, R, phi);
  case Q_EVAL: return comp_eval(c, R, z, phi);
  default: return comp_hess(c, q - Q_H0, R, z, phi);
  }
}

/* xi and its derivatives, in the reference's forms
   (KuzminLikeWrapperPotential.c:5-40): d[0] xi, d[1] dxi/dR, d[2] dxi/dz,
   d[3] d2xi/dR2, d[4] d2xi/dz2, d[5] d2xi/dRdz */
static void kuzmin_xi(double R, double z, double a, double b2, double *d)
{
  double sbz = sqrt(z * z + b2), asbz = a + sbz;
  d[0] = sqrt(R * R + asbz * asbz);
  d[1] = R / sqrt(R * R + asbz * asbz);
  d[2] = asbz * z / sqrt(R * R + asbz * asbz) / sbz;
  d[3] = asbz * asbz / pow(R * R + asbz * asbz, 1.5);
  d[4] = (a * a * a * b2 + 3. * a * a * b2 * sbz + a * b2 * (3. * b2 + R * R + 3. * z * z) +
          (b2 + R * R) * pow(sbz, 3.0)) / pow(sbz, 3.0) / pow(d[0], 3.0);
  d[5] = -R * z * asbz / sbz / pow(R * R + asbz * asbz, 1.5);
}

static double range_sum(opot *P, int i0, int i1, int q, double R, double z, double phi);

/* a KuzminLike wrapper's contribution to quantity q: the chain rule of the
   wrapped list's in-plane radial force and second derivative at (xi, 0, 0)
   (the wrapper is axisymmetric: its torque and phi derivatives are 0) */
static double kuzmin_quantity(opot *P, const ocomp *c, int i, int q, double R, double z)
{
  const double amp = c->p[0], a = c->p[1], b2 = c->p[2];
  const int j0 = i + 1, j1 = i + 1 + c->nsub;
  const int planar = q == Q_PRF || q == Q_PPT || q == Q_PH0 || q == Q_PH1 || q == Q_PH2;
  double d[6];
  kuzmin_xi(R, planar ? 0.0 : z, a, b2, d);
  const int qf = planar ? Q_PRF : Q_RF;
  switch (q) {
  case Q_RF: case Q_PRF: return amp * range_sum(P, j0, j1, qf, d[0], 0.0, 0.0) * d[1];
  case Q_ZF: return amp * range_sum(P, j0, j1, Q_RF, d[0], 0.0, 0.0) * d[2];
  case Q_H0: case Q_PH0:
    return amp * (range_sum(P, j0, j1, planar ? Q_PH0 : Q_H0, d[0], 0.0, 0.0) * d[1] * d[1] -
                  range_sum(P, j0, j1, qf, d[0], 0.0, 0.0) * d[3]);
  case Q_H1:
    return amp * (range_sum(P, j0, j1, Q_H0, d[0], 0.0, 0.0) * d[2] * d[2] -
                  range_sum(P, j0, j1, Q_RF, d[0], 0.0, 0.0) * d[4]);
  case Q_H2:
    return amp * (range_sum(P, j0, j1, Q_H0, d[0], 0.0, 0.0) * d[1] * d[2] -
                  range_sum(P, j0, j1, Q_RF, d[0], 0.0, 0.0) * d[5]);
  case Q_EVAL: return amp * range_sum(P, j0, j1, Q_EVAL, d[0], 0.0, 0.0);
  default: return 0.0;
  }
}

/* a CorotatingRotation wrapper's contribution to quantity q: the wrapped
   list at phi' = phi - s(R, t), radial derivatives through the chain rule
   d/dR -> d/dR - s_R d/dphi' (CorotatingRotationWrapperPotential.c: each
   quantity in the reference's own grouping) */
static double corot_quantity(opot *P, const ocomp *c, int i, int q, double R, double z,
                             double phi)
{
  const double amp = c->p[0], vpo = c->p[1], beta = c->p[2], pa = c->p[3], to = c->p[4];
  const double t = c->t;
  const int j0 = i + 1, j1 = i + 1 + c->nsub;
  const double ph = phi - vpo * pow(R, beta - 1) * (t - to) - pa;
  const double dR = -vpo * (beta - 1) * pow(R, beta - 2) * (t - to);
#define CQ(Q) range_sum(P, j0, j1, (Q), R, z, ph)
  switch (q) {
  case Q_RF:
    return amp * (CQ(Q_RF) - CQ(Q_PT) * vpo * (beta - 1) * pow(R, beta - 2) * (t - to));
  case Q_PRF:
    return amp * (CQ(Q_PRF) - CQ(Q_PPT) * vpo * (beta - 1) * pow(R, beta - 2) * (t - to));
  case Q_ZF: case Q_PT: case Q_PPT: case Q_H1: case Q_H3: case Q_H5: case Q_PH1:
    return amp * CQ(q);
  case Q_H0:
    return amp * (CQ(Q_H0) + 2. * dR * CQ(Q_H4) + dR * dR * CQ(Q_H3) +
                  CQ(Q_PT) * vpo * (beta - 1) * (beta - 2) * pow(R, beta - 3) * (t - to));
  case Q_PH0:
    return amp * (CQ(Q_PH0) + 2. * dR * CQ(Q_PH2) + dR * dR * CQ(Q_PH1) +
                  CQ(Q_PPT) * vpo * (beta - 1) * (beta - 2) * pow(R, beta - 3) * (t - to));
  case Q_H2: return amp * (CQ(Q_H2) + dR * CQ(Q_H5));
  case Q_H4: return amp * (CQ(Q_H4) + dR * CQ(Q_H3));
  case Q_PH2:
    return amp * (CQ(Q_PH2) - CQ(Q_PH1) * vpo * (beta - 1) * pow(R, beta - 2) * (t - to));
  default: return NAN; /* no potential evaluation in the reference's C */
  }
#undef CQ
}

/* sum of quantity q over entries [i0, i1), in order; a wrapper contributes
   its factor times the sum over its entries (at phi - omega t - pa for the
   rotation wrapper): DehnenSmooth amp s(t) (1 - s(t) if not growing),
   GaussianAmplitude amp exp(-(t - to)^2 / (2 sigma^2)), SolidBodyRotation
   amp (galpy_potentials.c calc* over the wrapped list) */
static double range_sum(opot *P, int i0, int i1, int q, double R, double z, double phi)
{
  double sum = 0.;
  for (int i = i0; i < i1; i++) {
    ocomp *c = &P->c[i];
    if (!is_wrapper(c->type)) {
      sum += comp_quantity(c, q, R, z, phi);
      continue;
    }
    if (c->type == PT_WRAP_KUZMIN || c->type == PT_WRAP_COROT) {
      sum += c->type == PT_WRAP_KUZMIN ? kuzmin_quantity(P, c, i, q, R, z)
                                        : corot_quantity(P, c, i, q, R, z, phi);
      i += c->nsub;
      continue;
    }
    const double *a = c->p, t = c->t;
    double fac, ph = phi;
    if (c->type == PT_WRAP_SMOOTH) {
      double sm = dbar_smooth(t, a[1], a[2]); /* dehnenSmooth: the same quintic */
      fac = a[0] * ((int)a[3] ? sm : 1. - sm);
    } else if (c->type == PT_WRAP_GAUSS) {
      fac = a[0] * exp(-0.5 * (t - a[1]) * (t - a[1]) / a[2]);
    } else {
      fac = a[0];
      ph = phi - a[1] * t - a[2];
      if (q == Q_EVAL) fac = NAN; /* no C evaluation in the reference */
    }
    sum += fac * range_sum(P, i + 1, i + 1 + c->nsub, q, R, z, ph);
    i += c->nsub;
  }
  return sum;
}

/* ------------------------------------------------------------------ */
/* right-hand sides                                                    */
/* ------------------------------------------------------------------ */
typedef struct {
  opot *P;
} octx;

/* How the angle of the Cartesian force routes is formed: 0 (default) as the
 * reference, acos(x/R) mapped to [0, 2 pi) (integrateFullOrbit.c:1313,
 * integratePlanarOrbit.c:1022); 1 atan2(y, x).  acos is ill-conditioned
 * where x/R is near +-1: a step that lands within ~1e-8 rad of the x axis
 * gets its angle wrong by up to sqrt(2 eps) ~ 2e-8, which in a
 * non-axisymmetric potential moves that force by as much.  The tests use
 * mode 1 to tell that reference-side error from the engine's (the engine
 * evaluates the force in Cartesian form, with no angle at all).  Test
 * infrastructure; not thread-safe against concurrent integrations. */
static int g_phi_mode = 0;
void oracle_set_phi_mode(int mode) { g_phi_mode = mode; }

/* cylindrical angle of (x,y) as the reference computes it */
static void cyl_of(double x, double y, double *R, double *phi, double *sp, double *cp)
{
  *R = sqrt(x * x + y * y);
  if (g_phi_mode == 1) {
    *phi = atan2(y, x);
    if (*phi < 0.) *phi += 2. * M_PI;
  } else {
    *phi = acos(x / *R);
  }
  *sp = y / *R;
  *cp = x / *R;
  if (g_phi_mode == 0 && y < 0.) *phi = 2. * M_PI - *phi;
}

/* the stepper's evaluation time, handed to the time-dependent components */
static void stamp_time(opot *P)
{
  for (int i = 0; i < P->n; i++) P->c[i].t = P->t;
}

static void sum3(opot *P, double R, double z, double phi, double *Rf, double *zf, double *pt)
{
  double a = 0., b = 0., c = 0.;
  stamp_time(P);
  a = range_sum(P, 0, P->n, Q_RF, R, z, phi);
  c = range_sum(P, 0, P->n, Q_PT, R, z, phi);
  b = range_sum(P, 0, P->n, Q_ZF, R, z, phi);
  *Rf = a;
  *zf = b;
  *pt = c;
  P->nforce++;
}

static void sum2(opot *P, double R, double phi, double *Rf, double *pt)
{
  double a = 0., c = 0.;
  stamp_time(P);
  a = range_sum(P, 0, P->n, Q_PRF, R, 0., phi);
  c = range_sum(P, 0, P->n, Q_PPT, R, 0., phi);
  *Rf = a;
  *pt = c;
  P->nforce++;
}

typedef void (*rhs_fn)(opot *P, const double *q, double *a);

/* evalRectForce (integrateFullOrbit.c:1307) */
static void rect_force3(opot *P, const double *q, double *a)
{
  double R, phi, sp, cp, Rf, zf, pt;
  cyl_of(q[0], q[1], &R, &phi, &sp, &cp);
  sum3(P, R, q[2], phi, &Rf, &zf, &pt);
  a[0] = cp * Rf - 1. / R * sp * pt;
  a[1] = sp * Rf + 1. / R * cp * pt;
  a[2] = zf;
}

/* evalRectDeriv (integrateFullOrbit.c:1326) */
static void rect_deriv3(opot *P, const double *q, double *a)
{
  a[0] = q[3];
  a[1] = q[4];
  a[2] = q[5];
  rect_force3(P, q, a + 3);
}

/* evalPlanarRectForce (integratePlanarOrbit.c:1015) */
static void rect_force2(opot *P, const double *q, double *a)
{
  double R, phi, sp, cp, Rf, pt;
  cyl_of(q[0], q[1], &R, &phi, &sp, &cp);
  sum2(P, R, phi, &Rf, &pt);
  a[0] = cp * Rf - 1. / R * sp * pt;
  a[1] = sp * Rf + 1. / R * cp * pt;
}

static void rect_deriv2(opot *P, const double *q, double *a)
{
  a[0] = q[2];
  a[1] = q[3];
  rect_force2(P, q, a + 2);
}

/* Cartesian tidal tensor K = -grad grad Phi in the plane, from cylindrical
   derivatives (integratePlanarOrbit.c:1150-1174 / integrateFullOrbit.c:1570-1590) */
static void planar_K(double R, double sp, double cp, double Rf, double pt, double R2d,
                     double p2d, double Rpd, double *Kxx, double *Kxy, double *Kyx, double *Kyy)
{
  *Kxx = -cp * cp * R2d + 2. * cp * sp / R / R * pt + sp * sp / R * Rf + 2. * sp * cp / R * Rpd -
         sp * sp / R / R * p2d;
  *Kxy = -sp * cp * R2d + (sp * sp - cp * cp) / R / R * pt - cp * sp / R * Rf -
         (cp * cp - sp * sp) / R * Rpd + cp * sp / R / R * p2d;
  *Kyx = -cp * sp * R2d + (sp * sp - cp * cp) / R / R * pt + (sp * sp - cp * cp) / R * Rpd -
         sp * cp / R * Rf + sp * cp / R / R * p2d;
  *Kyy = -sp * sp * R2d - 2. * sp * cp / R / R * pt - 2. * sp * cp / R * Rpd + cp * cp / R * Rf -
         cp * cp / R / R * p2d;
}

static void hess3(opot *P, double R, double z, double phi, double h[6])
{
  stamp_time(P);
  for (int w = 0; w < 6; w++) {
    double s = 0.;
    s = range_sum(P, 0, P->n, Q_H0 + w, R, z, phi);
    h[w] = s;
  }
}

/* full 3D K (symmetric) into k[6] = xx, xy, yy, xz, yz, zz */
static void full_K(opot *P, double R, double z, double phi, double sp, double cp, double Rf,
                   double pt, double k[6])
{
  double h[6], Kyx;
  hess3(P, R, z, phi, h); /* R2, z2, Rz, phi2, Rphi, zphi */
  planar_K(R, sp, cp, Rf, pt, h[0], h[3], h[4], &k[0], &k[1], &Kyx, &k[2]);
  k[3] = -cp * h[2] + sp / R * h[5];
  k[4] = -sp * h[2] - cp / R * h[5];
  k[5] = -h[1];
}

/* evalRectDeriv_dxdv (integrateFullOrbit.c:1496): 12-D state */
static void rect_deriv3_dxdv(opot *P, const double *q, double *a)
{
  double R, phi, sp, cp, Rf, zf, pt, k[6];
  a[0] = q[3];
  a[1] = q[4];
  a[2] = q[5];
  cyl_of(q[0], q[1], &R, &phi, &sp, &cp);
  sum3(P, R, q[2], phi, &Rf, &zf, &pt);
  a[3] = cp * Rf - 1. / R * sp * pt;
  a[4] = sp * Rf + 1. / R * cp * pt;
  a[5] = zf;
  a[6] = q[9];
  a[7] = q[10];
  a[8] = q[11];
  full_K(P, R, q[2], phi, sp, cp, Rf, pt, k);
  double dx = q[6], dy = q[7], dz = q[8];
  a[9] = k[0] * dx + k[1] * dy + k[3] * dz;
  a[10] = k[1] * dx + k[2] * dy + k[4] * dz;
  a[11] = k[3] * dx + k[4] * dy + k[5] * dz;
}

/* evalRectForce_dxdv with nde = 1 (integrateFullOrbit.c:1627): q[6] = (x,y,z,dx,dy,dz) */
static void rect_force3_dxdv(opot *P, const double *q, double *a)
{
  double R, phi, sp, cp, Rf, zf, pt, k[6];
  cyl_of(q[0], q[1], &R, &phi, &sp, &cp);
  sum3(P, R, q[2], phi, &Rf, &zf, &pt);
  a[0] = cp * Rf - 1. / R * sp * pt;
  a[1] = sp * Rf + 1. / R * cp * pt;
  a[2] = zf;
  full_K(P, R, q[2], phi, sp, cp, Rf, pt, k);
  double dx = q[3], dy = q[4], dz = q[5];
  a[3] = k[0] * dx + k[1] * dy + k[3] * dz;
  a[4] = k[1] * dx + k[2] * dy + k[4] * dz;
  a[5] = k[3] * dx + k[4] * dy + k[5] * dz;
}

static void planar_hess_sum(opot *P, double R, double phi, double *R2d, double *p2d, double *Rpd)
{
  double a = 0., b = 0., c = 0.;
  stamp_time(P);
  a = range_sum(P, 0, P->n, Q_PH0, R, 0., phi);
  b = range_sum(P, 0, P->n, Q_PH1, R, 0., phi);
  c = range_sum(P, 0, P->n, Q_PH2, R, 0., phi);
  *R2d = a;
  *p2d = b;
  *Rpd = c;
}

/* evalPlanarRectDeriv_dxdv (integratePlanarOrbit.c:1124): 8-D state */
static void rect_deriv2_dxdv(opot *P, const double *q, double *a)
{
  double R, phi, sp, cp, Rf, pt, R2d, p2d, Rpd, Kxx, Kxy, Kyx, Kyy;
  a[0] = q[2];
  a[1] = q[3];
  cyl_of(q[0], q[1], &R, &phi, &sp, &cp);
  sum2(P, R, phi, &Rf, &pt);
  a[2] = cp * Rf - 1. / R * sp * pt;
  a[3] = sp * Rf + 1. / R * cp * pt;
  a[4] = q[6];
  a[5] = q[7];
  planar_hess_sum(P, R, phi, &R2d, &p2d, &Rpd);
  planar_K(R, sp, cp, Rf, pt, R2d, p2d, Rpd, &Kxx, &Kxy, &Kyx, &Kyy);
  a[6] = Kxx * q[4] + Kxy * q[5];
  a[7] = Kyx * q[4] + Kyy * q[5];
}

/* evalPlanarRectForce_dxdv, nde = 1 (integratePlanarOrbit.c:1228): q = (x,y,dx,dy) */
static void rect_force2_dxdv(opot *P, const double *q, double *a)
{
  double R, phi, sp, cp, Rf, pt, R2d, p2d, Rpd, Kxx, Kxy, Kyx, Kyy;
  cyl_of(q[0], q[1], &R, &phi, &sp, &cp);
  sum2(P, R, phi, &Rf, &pt);
  a[0] = cp * Rf - 1. / R * sp * pt;
  a[1] = sp * Rf + 1. / R * cp * pt;
  planar_hess_sum(P, R, phi, &R2d, &p2d, &Rpd);
  planar_K(R, sp, cp, Rf, pt, R2d, p2d, Rpd, &Kxx, &Kxy, &Kyx, &Kyy);
  a[2] = Kxx * q[2] + Kxy * q[3];
  a[3] = Kxy * q[2] + Kyy * q[3];
}

/* ------------------------------------------------------------------ */
/* steppers                                                            */
/* ------------------------------------------------------------------ */
#define DT_SENTINEL -9999.99
#define MAX_DT_REDUCE 10000.
#define MAXD 12

static const double S4C[4] = {0.6756035959798289, -0.1756035959798288, -0.1756035959798288,
                              0.6756035959798289};
static const double S4D[3] = {1.3512071919596578, -1.7024143839193153, 1.3512071919596578};

static inline void drift(int n, const double *q, const double *p, double h, double *qn)
{
  for (int i = 0; i < n; i++) qn[i] = q[i] + h * p[i];
}
static inline void kick(int n, const double *p, double h, const double *a, double *pn)
{
  for (int i = 0; i < n; i++) pn[i] = p[i] + h * a[i];
}

/* log-sum-exp error scale of the symplectic / rk estimators
   (bovy_symplecticode.c:609-624) */
static double est_scale(int n, const double *v, double rtol, double atol)
{
  double m = log(fabs(v[0]));
  for (int i = 1; i < n; i++)
    if (log(fabs(v[i])) > m) m = log(fabs(v[i]));
  double c = fmax(atol, rtol + m);
  return log(exp(atol - c) + exp(rtol + m - c)) + c;
}

/* Output ordering of a symplectic state: plain runs store [q(dim),p(dim)];
   variational runs store [q_base,p_base,q_dev,p_dev] (save_qp_dxdv). */
static void save_qp(int ndim, int dim_base, const double *q, const double *p, double *out)
{
  if (ndim == dim_base) {
    for (int i = 0; i < ndim; i++) out[i] = q[i];
    for (int i = 0; i < ndim; i++) out[ndim + i] = p[i];
  } else {
    int nb = ndim / dim_base;
    for (int b = 0; b < nb; b++) {
      for (int k = 0; k < dim_base; k++) *out++ = q[dim_base * b + k];
      for (int k = 0; k < dim_base; k++) *out++ = p[dim_base * b + k];
    }
  }
}

typedef struct {
  long long nsteps;
  long long max_attempts;
  int err;
} ostat;

/* Drift-kick composition schemes: nk kicks d[0..nk-1] between nk+1 drifts
   c[0..nk] (coefficients of bovy_symplecticode.c:96-104; leapfrog is the
   scheme c = (1/2, 1/2), d = (1), whose products with dt are the reference's
   dt/2 and dt exactly). */
typedef struct {
  int nk;
  const double *c, *d;
} oscheme;
static const double LFC[2] = {0.5, 0.5}, LFD[1] = {1.0};
static const double S6C[8] = {0.392256805238780,   0.510043411918458,  -0.471053385409758,
                              0.687531682525198e-1, 0.687531682525198e-1, -0.471053385409758,
                              0.510043411918458,   0.392256805238780};
static const double S6D[7] = {0.784513610477560,   0.235573213359357, -0.117767998417887e1,
                              0.131518632068391e1, -0.117767998417887e1, 0.235573213359357,
                              0.784513610477560};
static const oscheme SCH_LF = {1, LFC, LFD}, SCH_S4 = {3, S4C, S4D}, SCH_S6 = {7, S6C, S6D};

/* nstep steps of size h from (q0, p0) to (q, p): first drift c0 h, kicks and
   drifts in turn, the last drift of a step merged with the first of the next
   ((c_nk + c_0) h), the final drift c_nk h.  This is the step sequence of
   leapfrog / symplec4 / symplec6 (bovy_symplecticode.c:132-587) and of the
   one- and two-step trials of their estimators (:588-1052). */
/* Force times, as the reference keeps its time `to`: TM_DRIFTS (symplec4,
   symplec6 and their estimators) adds each drift's length to *to and kicks
   at *to; TM_LEAP (leapfrog) kicks at *to + h/2 and adds h after each step;
   TM_LEAP_EST (leapfrog_estimate_step) kicks at to + dt/2 (one step of dt)
   or to + dt/4 and to + 3 dt/4 (two of dt/2), *to unchanged. */
enum { TM_DRIFTS = 0, TM_LEAP = 1, TM_LEAP_EST = 2 };

static void comp_advance(const oscheme *S, rhs_fn f, opot *P, int n, const double *q0,
                         const double *p0, double h, long nstep, double *q, double *p,
                         double *to, int tmode)
{
  double a[MAXD];
  drift(n, q0, p0, S->c[0] * h, q);
  if (tmode == TM_DRIFTS) *to += S->c[0] * h;
  for (int k = 0; k < n; k++) p[k] = p0[k];
  for (long s = 0; s < nstep; s++) {
    for (int j = 0; j < S->nk; j++) {
      if (tmode == TM_DRIFTS)
        P->t = *to;
      else if (tmode == TM_LEAP || nstep == 1)
        P->t = *to + h / 2.;
      else /* the estimator's two half steps, dt = 2 h */
        P->t = s == 0 ? *to + (2. * h) / 4. : *to + 3. * (2. * h) / 4.;
      f(P, q, a);
      kick(n, p, S->d[j] * h, a, p);
      double c;
      if (j < S->nk - 1)
        c = S->c[j + 1] * h;
      else
        c = (s < nstep - 1) ? (S->c[S->nk] + S->c[0]) * h : S->c[S->nk] * h;
      drift(n, q, p, c, q);
      if (tmode == TM_DRIFTS) *to += c;
    }
    if (tmode == TM_LEAP) *to = *to + h;
  }
}

/* leapfrog_estimate_step / symplec4_estimate_step / symplec6_estimate_step
   (bovy_symplecticode.c:588-664, 665-809, 810-1052): halve dt until one step
   and two half steps agree to the tolerance */
static double comp_est(const oscheme *S, rhs_fn f, opot *P, int dim, const double *qo,
                       const double *po, double dt, double t0, double rtol, double atol)
{
  double err = 2., init_dt = dt, to = t0;
  int tmode = S == &SCH_LF ? TM_LEAP_EST : TM_DRIFTS;
  double q11[MAXD], q12[MAXD], p11[MAXD], p12[MAXD];
  double sq = est_scale(dim, qo, rtol, atol), sp = est_scale(dim, po, rtol, atol);
  dt *= 2.;
  while (err > 1. && init_dt / dt < MAX_DT_REDUCE) {
    dt /= 2.;
    comp_advance(S, f, P, dim, qo, po, dt, 1, q11, p11, &to, tmode);
    if (tmode == TM_DRIFTS) to -= dt;
    comp_advance(S, f, P, dim, qo, po, dt / 2., 2, q12, p12, &to, tmode);
    if (tmode == TM_DRIFTS) to -= dt;
    err = 0.;
    for (int i = 0; i < dim; i++) {
      err += exp(2. * log(fabs(q11[i] - q12[i])) - 2. * sq);
      err += exp(2. * log(fabs(p11[i] - p12[i])) - 2. * sp);
    }
    err = sqrt(err / 2. / dim);
  }
  return dt;
}

/* leapfrog / symplec4 / symplec6 (bovy_symplecticode.c:132-587 and the
   *_dxdv steppers :1053-1400).  f steps the ndim-vector, fb is the base
   force for the estimator over dim_base components; yo is in save_qp
   layout. */
static void symplectic(const oscheme *S, rhs_fn f, rhs_fn fb, opot *P, int ndim, int dim_base,
                       const double *yo, int nt, double dt, const double *t, double rtol,
                       double atol, double *result, ostat *st)
{
  double qo[MAXD], po[MAXD];
  int nb = ndim / dim_base;
  for (int b = 0; b < nb; b++)
    for (int k = 0; k < dim_base; k++) {
      qo[dim_base * b + k] = yo[2 * dim_base * b + k];
      po[dim_base * b + k] = yo[2 * dim_base * b + dim_base + k];
    }
  save_qp(ndim, dim_base, qo, po, result);
  result += 2 * ndim;
  st->err = 0;
  double init_dt = t[1] - t[0];
  if (dt == DT_SENTINEL) dt = comp_est(S, fb, P, dim_base, qo, po, init_dt, t[0], rtol, atol);
  long ndt = (long)(init_dt / dt);
  if (ndt < 1) ndt = 1; /* the reference's loop always makes the output step */
  double to = t[0];
  for (int ii = 0; ii < nt - 1; ii++) {
    comp_advance(S, f, P, ndim, qo, po, dt, ndt, qo, po, &to, S == &SCH_LF ? TM_LEAP : TM_DRIFTS);
    save_qp(ndim, dim_base, qo, po, result);
    result += 2 * ndim;
  }
  st->nsteps = (long long)ndt * (nt - 1);
}

/* bovy_rk4_onestep (bovy_rk.c:142-170) */
static void rk4_onestep(rhs_fn f, opot *P, int dim, const double *yn, double *yn1, double tn,
                        double dt, double *ynk, double *a)
{
  P->t = tn;
  f(P, yn, a);
  for (int i = 0; i < dim; i++) yn1[i] += dt * a[i] / 6.;
  for (int i = 0; i < dim; i++) ynk[i] = yn[i] + dt * a[i] / 2.;
  P->t = tn + dt / 2.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) yn1[i] += dt * a[i] / 3.;
  for (int i = 0; i < dim; i++) ynk[i] = yn[i] + dt * a[i] / 2.;
  P->t = tn + dt / 2.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) yn1[i] += dt * a[i] / 3.;
  for (int i = 0; i < dim; i++) ynk[i] = yn[i] + dt * a[i];
  P->t = tn + dt;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) yn1[i] += dt * a[i] / 6.;
}

/* bovy_rk6_onestep (bovy_rk.c:256-327): seven stages, weights
   (11, 0, 81, 81, -32, -32, 11)/120 accumulated into yn1 stage by stage */
static void rk6_onestep(rhs_fn f, opot *P, int dim, const double *yn, double *yn1, double tn,
                        double dt, double *ynk, double *a)
{
  double k1[MAXD], k2[MAXD], k3[MAXD], k4[MAXD], k5[MAXD];
  P->t = tn;
  f(P, yn, a);
  for (int i = 0; i < dim; i++) {
    yn1[i] += 11. * dt * a[i] / 120.;
    k1[i] = dt * a[i];
    ynk[i] = yn[i] + k1[i] / 3.;
  }
  P->t = tn + dt / 3.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) {
    k2[i] = dt * a[i];
    ynk[i] = yn[i] + 2. * k2[i] / 3.;
  }
  P->t = tn + 2. * dt / 3.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) {
    yn1[i] += 81. * dt * a[i] / 120.;
    k3[i] = dt * a[i];
    ynk[i] = yn[i] + (k1[i] + 4. * k2[i] - k3[i]) / 12.;
  }
  P->t = tn + dt / 3.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) {
    yn1[i] += 81. * dt * a[i] / 120.;
    k4[i] = dt * a[i];
    ynk[i] = yn[i] + (-k1[i] + 18. * k2[i] - 3. * k3[i] - 6. * k4[i]) / 16.;
  }
  P->t = tn + dt / 2.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) {
    yn1[i] -= 32. * dt * a[i] / 120.;
    k5[i] = dt * a[i];
    ynk[i] = yn[i] + (9. * k2[i] - 3. * k3[i] - 6. * k4[i] + 4. * k5[i]) / 8.;
  }
  P->t = tn + dt / 2.;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) {
    yn1[i] -= 32. * dt * a[i] / 120.;
    const double k6 = dt * a[i];
    ynk[i] = yn[i] + (9. * k1[i] - 36. * k2[i] + 63. * k3[i] + 72. * k4[i] - 64. * k6) / 44.;
  }
  P->t = tn + dt;
  f(P, ynk, a);
  for (int i = 0; i < dim; i++) yn1[i] += 11. * dt * a[i] / 120.;
}

typedef void (*rk_step_fn)(rhs_fn f, opot *P, int dim, const double *yn, double *yn1, double tn,
                           double dt, double *ynk, double *a);

/* rk4_estimate_step / rk6_estimate_step (bovy_rk.c:328-395, 396-480): divide
   dt by ceil(err^(1/(order+1))) until one step and two half steps agree */
static double rk_est(rk_step_fn onestep, double expo, rhs_fn f, opot *P, int dim,
                     const double *yo, double dt, double to, double rtol, double atol)
{
  double err = 2., init_dt = dt;
  double yn[MAXD], y1[MAXD], y21[MAXD], y2[MAXD], ynk[MAXD], a[MAXD];
  double s = est_scale(dim, yo, rtol, atol);
  while (err > 1.) {
    for (int i = 0; i < dim; i++) yn[i] = y1[i] = y21[i] = yo[i];
    onestep(f, P, dim, yn, y1, to, dt, ynk, a);
    onestep(f, P, dim, yn, y21, to, dt / 2., ynk, a);
    for (int i = 0; i < dim; i++) y2[i] = y21[i];
    onestep(f, P, dim, y21, y2, to + dt / 2., dt / 2., ynk, a);
    err = 0.;
    for (int i = 0; i < dim; i++) err += exp(2. * log(fabs(y1[i] - y2[i])) - 2. * s);
    err = sqrt(err / dim);
    if (ceil(pow(err, expo)) > 1. && init_dt / dt * ceil(pow(err, expo)) < MAX_DT_REDUCE)
      dt /= ceil(pow(err, expo));
    else
      break;
  }
  return dt;
}

/* bovy_rk4 / bovy_rk6 (bovy_rk.c:66-141, 171-255) */
static void rk_fixed(int order, rhs_fn f, opot *P, int dim, const double *yo, int nt, double dt,
                     const double *t, double rtol, double atol, double *result, ostat *st)
{
  rk_step_fn onestep = order == 6 ? rk6_onestep : rk4_onestep;
  double yn[MAXD], yn1[MAXD], ynk[MAXD], a[MAXD];
  for (int i = 0; i < dim; i++) result[i] = yo[i];
  result += dim;
  st->err = 0;
  for (int i = 0; i < dim; i++) yn[i] = yn1[i] = yo[i];
  double init_dt = t[1] - t[0];
  if (dt == DT_SENTINEL)
    dt = rk_est(onestep, order == 6 ? 1. / 7. : 1. / 5., f, P, dim, yo, init_dt, t[0], rtol,
                atol);
  long ndt = (long)(init_dt / dt);
  double to = t[0];
  for (int ii = 0; ii < nt - 1; ii++) {
    for (long jj = 0; jj < ndt - 1; jj++) {
      onestep(f, P, dim, yn, yn1, to, dt, ynk, a);
      to += dt;
      for (int k = 0; k < dim; k++) yn[k] = yn1[k];
    }
    onestep(f, P, dim, yn, yn1, to, dt, ynk, a);
    to += dt;
    for (int k = 0; k < dim; k++) result[k] = yn1[k];
    result += dim;
    for (int k = 0; k < dim; k++) yn[k] = yn1[k];
  }
  st->nsteps = (long long)ndt * (nt - 1);
}

/* Dormand-Prince 5(4) tableau (bovy_rk.c:630-665) */
#define DP5_A21 0.2
#define DP5_A31 (3. / 40.)
#define DP5_A32 (9. / 40.)
#define DP5_A41 (44. / 45.)
#define DP5_A42 (-56. / 15.)
#define DP5_A43 (32. / 9.)
#define DP5_A51 (19372. / 6561.)
#define DP5_A52 (-25360. / 2187.)
#define DP5_A53 (64448. / 6561.)
#define DP5_A54 (-212. / 729.)
#define DP5_A61 (9017. / 3168.)
#define DP5_A62 (-355. / 33.)
#define DP5_A63 (46732. / 5247.)
#define DP5_A64 (49. / 176.)
#define DP5_A65 (-5103. / 18656.)
#define DP5_B1 (35. / 384.)
#define DP5_B3 (500. / 1113.)
#define DP5_B4 (125. / 192.)
#define DP5_B5 (-2187. / 6784.)
#define DP5_B6 (11. / 84.)
#define DP5_E1 (DP5_B1 - 5179. / 57600.)
#define DP5_E3 (DP5_B3 - 7571. / 16695.)
#define DP5_E4 (DP5_B4 - 393. / 640.)
#define DP5_E5 (DP5_B5 + 92097. / 339200.)
#define DP5_E6 (DP5_B6 - 187. / 2100.)
#define DP5_E7 (-1. / 40.)

/* bovy_dopr54_actualstep (bovy_rk.c:617-760): one attempt of size dt from
   (yo, a1 = f(yo)); on acceptance (the power-of-two step factor is >= 1, or
   the attempt is forced) yo, a1 and *to advance.  Returns the next step. */
static double dopr54_attempt(rhs_fn f, opot *P, int dim, double *yo, double *a1, double dt,
                             double *to, double rtol, double atol, int accept, ostat *st)
{
  double k1[MAXD], k2[MAXD], k3[MAXD], k4[MAXD], k5[MAXD], k6[MAXD];
  double yn1[MAXD], yerr[MAXD], ynk[MAXD], a[MAXD];
  int i;
  for (i = 0; i < dim; i++) {
    yn1[i] = yo[i];
    k1[i] = dt * a1[i];
    yn1[i] += DP5_B1 * k1[i];
    yerr[i] = DP5_E1 * k1[i];
    ynk[i] = yo[i] + DP5_A21 * k1[i];
  }
  P->t = *to + 0.2 * dt;
  f(P, ynk, a);
  for (i = 0; i < dim; i++) {
    k2[i] = dt * a[i];
    ynk[i] = yo[i] + DP5_A31 * k1[i] + DP5_A32 * k2[i];
  }
  P->t = *to + 0.3 * dt;
  f(P, ynk, a);
  for (i = 0; i < dim; i++) {
    k3[i] = dt * a[i];
    yn1[i] += DP5_B3 * k3[i];
    yerr[i] += DP5_E3 * k3[i];
    ynk[i] = yo[i] + DP5_A41 * k1[i] + DP5_A42 * k2[i] + DP5_A43 * k3[i];
  }
  P->t = *to + 0.8 * dt;
  f(P, ynk, a);
  for (i = 0; i < dim; i++) {
    k4[i] = dt * a[i];
    yn1[i] += DP5_B4 * k4[i];
    yerr[i] += DP5_E4 * k4[i];
    ynk[i] = yo[i] + DP5_A51 * k1[i] + DP5_A52 * k2[i] + DP5_A53 * k3[i] + DP5_A54 * k4[i];
  }
  P->t = *to + 8. / 9. * dt;
  f(P, ynk, a);
  for (i = 0; i < dim; i++) {
    k5[i] = dt * a[i];
    yn1[i] += DP5_B5 * k5[i];
    yerr[i] += DP5_E5 * k5[i];
    ynk[i] = yo[i] + DP5_A61 * k1[i] + DP5_A62 * k2[i] + DP5_A63 * k3[i] + DP5_A64 * k4[i] +
             DP5_A65 * k5[i];
  }
  P->t = *to + dt;
  f(P, ynk, a);
  for (i = 0; i < dim; i++) {
    k6[i] = dt * a[i];
    yn1[i] += DP5_B6 * k6[i];
    yerr[i] += DP5_E6 * k6[i];
    /* the seventh stage point uses the b weights as its a7j (a72 = 0) */
    ynk[i] = yo[i] + DP5_B1 * k1[i] + DP5_B3 * k3[i] + DP5_B4 * k4[i] + DP5_B5 * k5[i] +
             DP5_B6 * k6[i];
  }
  P->t = *to + dt;
  f(P, ynk, a);
  for (i = 0; i < dim; i++) yerr[i] += DP5_E7 * dt * a[i];
  double s = est_scale(dim, yo, rtol, atol);
  double err = 0.;
  for (i = 0; i < dim; i++) err += exp(2. * log(fabs(yerr[i])) - 2. * s);
  err = sqrt(err / dim);
  double corr = 0.85 * pow(err, -.2);
  double powertwo = round(log(corr) / log(2.));
  if (powertwo > 3.)
    powertwo = 3.;
  else if (powertwo < -3.)
    powertwo = -3.;
  if (powertwo >= 0. || accept) {
    for (i = 0; i < dim; i++) {
      a1[i] = a[i];
      yo[i] = yn1[i];
    }
    *to += dt;
    st->nsteps++;
  }
  return dt * pow(2., powertwo);
}

/* bovy_dopr54 (bovy_rk.c:501-616): adaptive steps, each output interval
   ended by a step clipped to its end; a step that would shrink below the
   interval's first step / 10000 (or is NaN) is forced at that size and
   flags err = 1.  The first step comes from rk4_estimate_step. */
static void dopr54(rhs_fn f, opot *P, int dim, const double *yin, int nt, double dt_one,
                   const double *t, double rtol, double atol, double *result, ostat *st)
{
  double yo[MAXD], a1[MAXD];
  for (int i = 0; i < dim; i++) yo[i] = result[i] = yin[i];
  result += dim;
  st->err = 0;
  st->nsteps = 0;
  double dt = t[1] - t[0];
  if (dt_one == DT_SENTINEL)
    dt_one = rk_est(rk4_onestep, 1. / 5., f, P, dim, yo, dt, t[0], rtol, atol);
  double to = t[0];
  P->t = to;
  f(P, yo, a1);
  long long attempts = 0;
  for (int ii = 0; ii < nt - 1; ii++) {
    double init_dt_one = dt_one, init_to = to;
    while ((dt >= 0. && to < (init_to + dt)) || (dt < 0. && to > (init_to + dt))) {
      if (st->max_attempts > 0 && attempts >= st->max_attempts) {
        st->err = 2;
        return;
      }
      attempts++;
      int accept = 0;
      if (init_dt_one / dt_one > MAX_DT_REDUCE || dt_one != dt_one) {
        dt_one = init_dt_one / MAX_DT_REDUCE;
        accept = 1;
        if (st->err % 2 == 0) st->err += 1;
      }
      if (dt >= 0. && dt_one > (init_to + dt - to)) dt_one = (init_to + dt - to);
      if (dt < 0. && dt_one < (init_to + dt - to)) dt_one = (init_to + dt - to);
      dt_one = dopr54_attempt(f, P, dim, yo, a1, dt_one, &to, rtol, atol, accept, st);
    }
    for (int i = 0; i < dim; i++) result[i] = yo[i];
    result += dim;
  }
}

#define DMAX(a, b) (((a) > (b)) ? (a) : (b))
#define DMIN(a, b) (((a) < (b)) ? (a) : (b))
static inline double csign(double x, double y) { return (y > 0.0) ? fabs(x) : -fabs(x); }

/* dop853 (leung_dop853.c:231-517); rtol/atol arrive as logs */
static void dop853(rhs_fn f, opot *P, int dim, const double *yin, int nt, const double *t,
                   double rtol, double atol, double *result, ostat *st)
{
  rtol = exp(rtol);
  atol = exp(atol);
  const double safe = 0.9, expo1 = 1.0 / 8.0, facc1 = 1.0 / 0.333, facc2 = 1.0 / 6.0;
  const double uround = 2.3e-16;
  double facold = 1.0e-4;
  double hmax = t[nt - 1] - t[0];
  double pos_neg = csign(1.0, hmax);
  double y0[MAXD], yy1[MAXD], k1[MAXD], k2[MAXD], k3[MAXD], k4[MAXD], k5[MAXD], k6[MAXD],
      k7[MAXD], k8[MAXD], k9[MAXD], k10[MAXD];
  double rc1[MAXD], rc2[MAXD], rc3[MAXD], rc4[MAXD], rc5[MAXD], rc6[MAXD], rc7[MAXD], rc8[MAXD];
  int i;
  for (i = 0; i < dim; i++) y0[i] = yin[i];
  for (i = 0; i < dim; i++) result[i] = y0[i];
  result += dim;
  st->err = 0;
  st->nsteps = 0;

  P->t = t[0];
  f(P, y0, k1);
  double dnf = 0.0, dny = 0.0, sk, sqr;
  for (i = 0; i < dim; i++) {
    sk = atol + rtol * fabs(y0[i]);
    sqr = k1[i] / sk;
    dnf += sqr * sqr;
    sqr = y0[i] / sk;
    dny += sqr * sqr;
  }
  double h = csign(DMIN(sqrt(dny / dnf) * 0.01, fabs(hmax)), pos_neg);
  for (i = 0; i < dim; i++) k3[i] = y0[i] + h * k1[i];
  P->t = t[0] + h;
  f(P, k3, k2);
  double der2 = 0.0;
  for (i = 0; i < dim; i++) {
    sk = atol + rtol * fabs(y0[i]);
    sqr = (k2[i] - k1[i]) / sk;
    der2 += sqr * sqr;
  }
  der2 = sqrt(der2) / h;
  double der12 = DMAX(fabs(der2), sqrt(dnf));
  double h1 = pow(0.01 / der12, 1.0 / 8.0);
  h = csign(DMIN(100.0 * fabs(h), DMIN(fabs(h1), fabs(hmax))), pos_neg);

  int reject = 0;
  double t_current = t[0], t_old = t[0], t_old_older = t_old;
  int done = 0;
  long long attempts = 0;
  while (done < nt - 1) {
    if (st->max_attempts > 0 && attempts >= st->max_attempts) {
      st->err = 2;
      break;
    }
    attempts++;
    h = pos_neg * DMAX(fabs(h), 1e3 * uround);
    for (i = 0; i < dim; i++) yy1[i] = y0[i] + h * DP_A21 * k1[i];
    P->t = t_current + DP_C2 * h;
    f(P, yy1, k2);
    for (i = 0; i < dim; i++) yy1[i] = y0[i] + h * (DP_A31 * k1[i] + DP_A32 * k2[i]);
    P->t = t_current + DP_C3 * h;
    f(P, yy1, k3);
    for (i = 0; i < dim; i++) yy1[i] = y0[i] + h * (DP_A41 * k1[i] + DP_A43 * k3[i]);
    P->t = t_current + DP_C4 * h;
    f(P, yy1, k4);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A51 * k1[i] + DP_A53 * k3[i] + DP_A54 * k4[i]);
    P->t = t_current + DP_C5 * h;
    f(P, yy1, k5);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A61 * k1[i] + DP_A64 * k4[i] + DP_A65 * k5[i]);
    P->t = t_current + DP_C6 * h;
    f(P, yy1, k6);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A71 * k1[i] + DP_A74 * k4[i] + DP_A75 * k5[i] + DP_A76 * k6[i]);
    P->t = t_current + DP_C7 * h;
    f(P, yy1, k7);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A81 * k1[i] + DP_A84 * k4[i] + DP_A85 * k5[i] + DP_A86 * k6[i] +
                            DP_A87 * k7[i]);
    P->t = t_current + DP_C8 * h;
    f(P, yy1, k8);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A91 * k1[i] + DP_A94 * k4[i] + DP_A95 * k5[i] + DP_A96 * k6[i] +
                            DP_A97 * k7[i] + DP_A98 * k8[i]);
    P->t = t_current + DP_C9 * h;
    f(P, yy1, k9);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A101 * k1[i] + DP_A104 * k4[i] + DP_A105 * k5[i] +
                            DP_A106 * k6[i] + DP_A107 * k7[i] + DP_A108 * k8[i] +
                            DP_A109 * k9[i]);
    P->t = t_current + DP_C10 * h;
    f(P, yy1, k10);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A111 * k1[i] + DP_A114 * k4[i] + DP_A115 * k5[i] +
                            DP_A116 * k6[i] + DP_A117 * k7[i] + DP_A118 * k8[i] +
                            DP_A119 * k9[i] + DP_A1110 * k10[i]);
    P->t = t_current + DP_C11 * h;
    f(P, yy1, k2);
    for (i = 0; i < dim; i++)
      yy1[i] = y0[i] + h * (DP_A121 * k1[i] + DP_A124 * k4[i] + DP_A125 * k5[i] +
                            DP_A126 * k6[i] + DP_A127 * k7[i] + DP_A128 * k8[i] +
                            DP_A129 * k9[i] + DP_A1210 * k10[i] + DP_A1211 * k2[i]);
    t_old_older = t_old;
    t_old = t_current;
    t_current = t_current + h;
    P->t = t_current;
    f(P, yy1, k3);
    for (i = 0; i < dim; i++) {
      k4[i] = DP_B1 * k1[i] + DP_B6 * k6[i] + DP_B7 * k7[i] + DP_B8 * k8[i] + DP_B9 * k9[i] +
              DP_B10 * k10[i] + DP_B11 * k2[i] + DP_B12 * k3[i];
      k5[i] = y0[i] + h * k4[i];
    }
    double err = 0.0, err2 = 0.0, erri;
    for (i = 0; i < dim; i++) {
      sk = atol + rtol * DMAX(fabs(y0[i]), fabs(k5[i]));
      erri = k4[i] - DP_BHH1 * k1[i] - DP_BHH2 * k9[i] - DP_BHH3 * k3[i];
      sqr = erri / sk;
      err2 += sqr * sqr;
      erri = DP_ER1 * k1[i] + DP_ER6 * k6[i] + DP_ER7 * k7[i] + DP_ER8 * k8[i] +
             DP_ER9 * k9[i] + DP_ER10 * k10[i] + DP_ER11 * k2[i] + DP_ER12 * k3[i];
      sqr = erri / sk;
      err += sqr * sqr;
    }
    double deno = err + 0.01 * err2;
    if (deno <= 0.0) deno = 1.0;
    err = fabs(h) * err * sqrt(1.0 / (deno * (double)dim));
    double fac11 = pow(err, expo1);
    double fac = fac11 / pow(facold, 0.0);
    fac = DMAX(facc2, DMIN(facc1, fac / safe));
    double hnew = h / fac;
    if (err <= 1.0) {
      facold = DMAX(err, 1.0e-4);
      st->nsteps++;
      P->t = t_current;
      f(P, k5, k4);
      for (i = 0; i < dim; i++) {
        rc1[i] = y0[i];
        double ydiff = k5[i] - y0[i];
        rc2[i] = ydiff;
        double bspl = h * k1[i] - ydiff;
        rc3[i] = bspl;
        rc4[i] = ydiff - h * k4[i] - bspl;
        rc5[i] = DP_D41 * k1[i] + DP_D46 * k6[i] + DP_D47 * k7[i] + DP_D48 * k8[i] +
                 DP_D49 * k9[i] + DP_D410 * k10[i] + DP_D411 * k2[i] + DP_D412 * k3[i];
        rc6[i] = DP_D51 * k1[i] + DP_D56 * k6[i] + DP_D57 * k7[i] + DP_D58 * k8[i] +
                 DP_D59 * k9[i] + DP_D510 * k10[i] + DP_D511 * k2[i] + DP_D512 * k3[i];
        rc7[i] = DP_D61 * k1[i] + DP_D66 * k6[i] + DP_D67 * k7[i] + DP_D68 * k8[i] +
                 DP_D69 * k9[i] + DP_D610 * k10[i] + DP_D611 * k2[i] + DP_D612 * k3[i];
        rc8[i] = DP_D71 * k1[i] + DP_D76 * k6[i] + DP_D77 * k7[i] + DP_D78 * k8[i] +
                 DP_D79 * k9[i] + DP_D710 * k10[i] + DP_D711 * k2[i] + DP_D712 * k3[i];
      }
      for (i = 0; i < dim; i++)
        yy1[i] = y0[i] + h * (DP_A141 * k1[i] + DP_A147 * k7[i] + DP_A148 * k8[i] +
                              DP_A149 * k9[i] + DP_A1410 * k10[i] + DP_A1411 * k2[i] +
                              DP_A1412 * k3[i] + DP_A1413 * k4[i]);
      P->t = t_old + DP_C14 * h;
      f(P, yy1, k10);
      for (i = 0; i < dim; i++)
        yy1[i] = y0[i] + h * (DP_A151 * k1[i] + DP_A156 * k6[i] + DP_A157 * k7[i] +
                              DP_A158 * k8[i] + DP_A1511 * k2[i] + DP_A1512 * k3[i] +
                              DP_A1513 * k4[i] + DP_A1514 * k10[i]);
      P->t = t_old + DP_C15 * h;
      f(P, yy1, k2);
      for (i = 0; i < dim; i++)
        yy1[i] = y0[i] + h * (DP_A161 * k1[i] + DP_A166 * k6[i] + DP_A167 * k7[i] +
                              DP_A168 * k8[i] + DP_A169 * k9[i] + DP_A1613 * k4[i] +
                              DP_A1614 * k10[i] + DP_A1615 * k2[i]);
      P->t = t_old + DP_C16 * h;
      f(P, yy1, k3);
      for (i = 0; i < dim; i++) {
        rc5[i] = h * (rc5[i] + DP_D413 * k4[i] + DP_D414 * k10[i] + DP_D415 * k2[i] +
                      DP_D416 * k3[i]);
        rc6[i] = h * (rc6[i] + DP_D513 * k4[i] + DP_D514 * k10[i] + DP_D515 * k2[i] +
                      DP_D516 * k3[i]);
        rc7[i] = h * (rc7[i] + DP_D613 * k4[i] + DP_D614 * k10[i] + DP_D615 * k2[i] +
                      DP_D616 * k3[i]);
        rc8[i] = h * (rc8[i] + DP_D713 * k4[i] + DP_D714 * k10[i] + DP_D715 * k2[i] +
                      DP_D716 * k3[i]);
        k1[i] = k4[i];
        y0[i] = k5[i];
      }
      while (done < nt - 1 && pos_neg * t[done + 1] < pos_neg * t_current) {
        double s = (t[done + 1] - t_old) / h, s1 = 1.0 - s;
        for (i = 0; i < dim; i++)
          result[i] =
              rc1[i] +
              s * (rc2[i] +
                   s1 * (rc3[i] +
                         s * (rc4[i] + s1 * (rc5[i] + s * (rc6[i] + s1 * (rc7[i] + s * rc8[i]))))));
        result += dim;
        done++;
      }
      hnew = (fabs(hnew) > fabs(hmax)) ? pos_neg * hmax : hnew;
      if (reject) hnew = pos_neg * DMIN(fabs(hnew), fabs(h));
      reject = 0;
    } else {
      /* extra over the reference: an attempt rejected at the smallest step
         repeats exactly, where the reference loops forever; stop (err 2) */
      if (fabs(h) <= 1e3 * uround) {
        st->err = 2;
        break;
      }
      hnew = h / DMIN(facc1, fac11 / safe);
      reject = 1;
      t_current = t_old;
      t_old = t_old_older;
    }
    h = hnew;
  }
}

/* ------------------------------------------------------------------ */
/* coordinates (bovy_coords.c:57-148)                                  */
/* ------------------------------------------------------------------ */
static void cyl_to_rect(double *v)
{
  double R = v[0], phi = v[5], cp = cos(phi), sp = sin(phi), vR = v[1], vT = v[2];
  v[0] = R * cp;
  v[1] = R * sp;
  v[2] = v[3];
  v[5] = v[4];
  v[3] = vR * cp - vT * sp;
  v[4] = vR * sp + vT * cp;
}
static void rect_to_cyl(double *v)
{
  double x = v[0], y = v[1], vx = v[3], vy = v[4];
  v[3] = v[2];
  v[4] = v[5];
  v[5] = atan2(y, x);
  double cp = cos(v[5]), sp = sin(v[5]);
  v[0] = sqrt(x * x + y * y);
  v[1] = vx * cp + vy * sp;
  v[2] = -vx * sp + vy * cp;
}
static void polar_to_rect(double *v)
{
  double R = v[0], phi = v[3], cp = cos(phi), sp = sin(phi), vR = v[1], vT = v[2];
  v[0] = R * cp;
  v[1] = R * sp;
  v[2] = vR * cp - vT * sp;
  v[3] = vR * sp + vT * cp;
}
static void rect_to_polar(double *v)
{
  double x = v[0], y = v[1], vx = v[2], vy = v[3];
  v[3] = atan2(y, x);
  double cp = cos(v[3]), sp = sin(v[3]);
  v[0] = sqrt(x * x + y * y);
  v[1] = vx * cp + vy * sp;
  v[2] = -vx * sp + vy * cp;
}

/* ------------------------------------------------------------------ */
/* surface of section (integrateFullOrbit.c:1151-1233, 1353-1390)       */
/* ------------------------------------------------------------------ */
/* evalSOSDeriv: q = (x, y, vx, vy, A, t, psi), derivative w.r.t. the psi
   increment; the force at (x, y, A sin psi) */
static void sos_deriv(opot *P, const double *q, double *a)
{
  double sinpsi = sin(q[6]), cospsi = cos(q[6]);
  double x = q[0], y = q[1], z = q[4] * sinpsi;
  double R = sqrt(x * x + y * y), phi = atan2(y, x);
  double sinphi = y / R, cosphi = x / R, Rf, zf, pt;
  P->t = q[5]; /* the state carries the time */
  sum3(P, R, z, phi, &Rf, &zf, &pt);
  a[3] = cosphi * Rf - 1. / R * sinphi * pt;
  a[4] = sinphi * Rf + 1. / R * cosphi * pt;
  a[5] = zf;
  double psidot = cospsi * cospsi - sinpsi * a[5] / q[4];
  a[0] = q[2] / psidot;
  a[1] = q[3] / psidot;
  a[2] = a[3] / psidot;
  a[3] = a[4] / psidot;
  a[4] = cospsi * (q[4] * sinpsi + a[5]) / psidot;
  a[5] = 1. / psidot;
  a[6] = 1.;
}

/* cyl_to_sos_galpy / sos_to_cyl_galpy (bovy_coords.c:149-189) */
static void cyl_to_sos(double *v)
{
  double R = v[0], cp = cos(v[5]), sp = sin(v[5]), vR = v[1], vT = v[2];
  v[5] = v[6];
  v[6] = atan2(v[3], v[4]);
  v[4] = sqrt(v[3] * v[3] + v[4] * v[4]);
  v[0] = R * cp;
  v[1] = R * sp;
  v[2] = vR * cp - vT * sp;
  v[3] = vR * sp + vT * cp;
}
static void sos_to_cyl(double *v)
{
  double x = v[0], y = v[1], vx = v[2], vy = v[3], phi = atan2(y, x), cp = cos(phi),
         sp = sin(phi);
  v[0] = sqrt(x * x + y * y);
  v[1] = vx * cp + vy * sp;
  v[2] = -vx * sp + vy * cp;
  v[3] = v[4] * sin(v[6]);
  v[4] = v[4] * cos(v[6]);
  v[6] = v[5];
  v[5] = phi;
}

/* planar surface of section (integratePlanarOrbit.c:848-939, 1056-1123):
   q = (u, vu, A, t, psi); surface x = 0: (u, vu) = (y, vy), x = A sin psi */
static void sos_planar_derivx(opot *P, const double *q, double *a)
{
  double sinpsi = sin(q[4]), cospsi = cos(q[4]);
  double x = q[2] * sinpsi, y = q[0];
  double R = sqrt(x * x + y * y), phi = atan2(y, x), sinphi = y / R, cosphi = x / R, Rf, pt;
  P->t = q[3];
  sum2(P, R, phi, &Rf, &pt);
  a[2] = cosphi * Rf - 1. / R * sinphi * pt;
  a[3] = sinphi * Rf + 1. / R * cosphi * pt;
  double psidot = cospsi * cospsi - sinpsi * a[2] / q[2];
  a[0] = q[1] / psidot;
  a[1] = a[3] / psidot;
  a[2] = cospsi * (q[2] * sinpsi + a[2]) / psidot;
  a[3] = 1. / psidot;
  a[4] = 1.;
}
/* surface y = 0: (u, vu) = (x, vx), y = A sin psi */
static void sos_planar_derivy(opot *P, const double *q, double *a)
{
  double sinpsi = sin(q[4]), cospsi = cos(q[4]);
  double x = q[0], y = q[2] * sinpsi;
  double R = sqrt(x * x + y * y), phi = atan2(y, x), sinphi = y / R, cosphi = x / R, Rf, pt;
  P->t = q[3];
  sum2(P, R, phi, &Rf, &pt);
  a[2] = cosphi * Rf - 1. / R * sinphi * pt;
  a[3] = sinphi * Rf + 1. / R * cosphi * pt;
  double psidot = cospsi * cospsi - sinpsi * a[3] / q[2];
  a[0] = q[1] / psidot;
  a[1] = a[2] / psidot;
  a[2] = cospsi * (q[2] * sinpsi + a[3]) / psidot;
  a[3] = 1. / psidot;
  a[4] = 1.;
}
/* polar_to_sos_galpy / sos_to_polar_galpy (bovy_coords.c:200-260) */
static void polar_to_sos(double *v, int surface)
{
  double R = v[0], cp = cos(v[3]), sp = sin(v[3]), vR = v[1], vT = v[2], x, y, vx, vy;
  if (surface == 1) {
    v[0] = R * cp;
    v[1] = vR * cp - vT * sp;
    y = R * sp;
    vy = vR * sp + vT * cp;
    v[2] = sqrt(y * y + vy * vy);
    v[3] = v[4];
    v[4] = atan2(y, vy);
  } else {
    v[0] = R * sp;
    v[1] = vR * sp + vT * cp;
    x = R * cp;
    vx = vR * cp - vT * sp;
    v[2] = sqrt(x * x + vx * vx);
    v[3] = v[4];
    v[4] = atan2(x, vx);
  }
}
static void sos_to_polar(double *v, int surface)
{
  double x, y, vx, vy;
  if (surface == 1) {
    x = v[0];
    vx = v[1];
    y = v[2] * sin(v[4]);
    vy = v[2] * cos(v[4]);
  } else {
    y = v[0];
    vy = v[1];
    x = v[2] * sin(v[4]);
    vx = v[2] * cos(v[4]);
  }
  double phi = atan2(y, x), cp = cos(phi), sp = sin(phi);
  v[0] = sqrt(x * x + y * y);
  v[1] = vx * cp + vy * sp;
  v[2] = -vx * sp + vy * cp;
  v[4] = v[3];
  v[3] = phi;
}

/* ------------------------------------------------------------------ */
/* exported drivers                                                    */
/* ------------------------------------------------------------------ */
#define EXPORT_SOS __attribute__((visibility("default")))

/* Planar surface-of-section integration (integratePlanarOrbit_sos): yo
   [nobj][5] = (R, vR, vT, phi, t0), overwritten with the SOS state;
   surface 0 (x = 0) or 1 (y = 0); result [nobj][npsi][5] = (R, vR, vT, phi,
   t). */
EXPORT_SOS int oracle_integrate_sos_planar(int nobj, double *yo, int npsi, const double *psi,
                                           int indiv_psi, int surface, int npot,
                                           const int *pot_type, const double *pot_args,
                                           double dpsi, double rtol, double atol,
                                           double *result, int *err, int method,
                                           long long *nsteps, int nthreads)
{
  opot P0;
  if (opot_decode(&P0, npot, pot_type, pot_args, 1)) return -3;
  if (method != 1 && method != 2 && method != 5 && method != 6) return -2;
  rhs_fn f = surface == 1 ? sos_planar_derivy : sos_planar_derivx;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int ii = 0; ii < nobj; ii++) {
    opot P = P0;
    ostat st = {0, 0, 0};
    double *w = yo + 5L * ii;
    const double *ps = psi + (long)npsi * ii * indiv_psi;
    double *out = result + 5L * npsi * ii;
    polar_to_sos(w, surface);
    switch (method) {
    case 1: rk_fixed(4, f, &P, 5, w, npsi, dpsi, ps, rtol, atol, out, &st); break;
    case 2: rk_fixed(6, f, &P, 5, w, npsi, dpsi, ps, rtol, atol, out, &st); break;
    case 5: dopr54(f, &P, 5, w, npsi, dpsi, ps, rtol, atol, out, &st); break;
    case 6: dop853(f, &P, 5, w, npsi, ps, rtol, atol, out, &st); break;
    }
    for (int jj = 0; jj < npsi; jj++) sos_to_polar(out + 5L * jj, surface);
    err[ii] = st.err;
    if (nsteps) nsteps[ii] = st.nsteps;
  }
  return 0;
}

/* Surface-of-section integration of nobj orbits (integrateFullOrbit_sos):
   yo [nobj][7] = (R, vR, vT, z, vz, phi, t0), overwritten with the SOS
   state; psi [npsi] or [nobj][npsi] increments; result [nobj][npsi][7] =
   (R, vR, vT, z, vz, phi, t).  method 1 rk4, 2 rk6, 5 dopr54, 6 dop853. */
EXPORT_SOS int oracle_integrate_sos(int nobj, double *yo, int npsi, const double *psi,
                                    int indiv_psi, int npot, const int *pot_type,
                                    const double *pot_args, double dpsi, double rtol, double atol,
                                    double *result, int *err, int method, long long *nsteps,
                                    int nthreads)
{
  opot P0;
  if (opot_decode(&P0, npot, pot_type, pot_args, 0)) return -3;
  if (method != 1 && method != 2 && method != 5 && method != 6) return -2;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int ii = 0; ii < nobj; ii++) {
    opot P = P0;
    ostat st = {0, 0, 0};
    double *w = yo + 7L * ii;
    const double *ps = psi + (long)npsi * ii * indiv_psi;
    double *out = result + 7L * npsi * ii;
    cyl_to_sos(w);
    switch (method) {
    case 1: rk_fixed(4, sos_deriv, &P, 7, w, npsi, dpsi, ps, rtol, atol, out, &st); break;
    case 2: rk_fixed(6, sos_deriv, &P, 7, w, npsi, dpsi, ps, rtol, atol, out, &st); break;
    case 5: dopr54(sos_deriv, &P, 7, w, npsi, dpsi, ps, rtol, atol, out, &st); break;
    case 6: dop853(sos_deriv, &P, 7, w, npsi, ps, rtol, atol, out, &st); break;
    }
    for (int jj = 0; jj < npsi; jj++) sos_to_cyl(out + 7L * jj);
    err[ii] = st.err;
    if (nsteps) nsteps[ii] = st.nsteps;
  }
  return 0;
}
#define EXPORT __attribute__((visibility("default")))

/* One orbit of the plain integration in rectangular coordinates.
   w: [2*dim] rectangular ICs; out: nt*2*dim rectangular rows. */
static int run_plain(opot *P, int planar, int method, const double *w, int nt, const double *t,
                     double dt, double rtol, double atol, double *out, ostat *st)
{
  int dim = planar ? 2 : 3;
  rhs_fn force = planar ? rect_force2 : rect_force3;
  rhs_fn deriv = planar ? rect_deriv2 : rect_deriv3;
  switch (method) {
  case 0: symplectic(&SCH_LF, force, force, P, dim, dim, w, nt, dt, t, rtol, atol, out, st); return 0;
  case 3: symplectic(&SCH_S4, force, force, P, dim, dim, w, nt, dt, t, rtol, atol, out, st); return 0;
  case 4: symplectic(&SCH_S6, force, force, P, dim, dim, w, nt, dt, t, rtol, atol, out, st); return 0;
  case 1: rk_fixed(4, deriv, P, 2 * dim, w, nt, dt, t, rtol, atol, out, st); return 0;
  case 2: rk_fixed(6, deriv, P, 2 * dim, w, nt, dt, t, rtol, atol, out, st); return 0;
  case 5: dopr54(deriv, P, 2 * dim, w, nt, dt, t, rtol, atol, out, st); return 0;
  case 6: dop853(deriv, P, 2 * dim, w, nt, t, rtol, atol, out, st); return 0;
  }
  return -1;
}

/* Batched integration with galpy's layout (integrateFullOrbit.c:1046 /
   integratePlanarOrbit.c:743): yo [nobj][6] (R,vR,vT,z,vz,phi) or [nobj][4]
   (R,vR,vT,phi), overwritten with rectangular ICs like the reference;
   result [nobj][nt][6|4] cylindrical.  method: 0 leapfrog, 1 rk4, 2 rk6,
   3 symplec4, 4 symplec6, 5 dopr54, 6 dop853.  nsteps/nforce (optional) receive per-orbit counts.
   Returns 0, -2 unsupported method, -3 unsupported potential. */
EXPORT int oracle_integrate(int planar, int nobj, double *yo, int nt, const double *t,
                            int indiv_t, int npot, const int *pot_type, const double *pot_args,
                            double dt, double rtol, double atol, double *result, int *err,
                            int method, long long *nsteps, long long *nforce,
                            long long max_attempts, int nthreads)
{
  opot P0;
  if (opot_decode(&P0, npot, pot_type, pot_args, planar)) return -3;
  if (method < 0 || method > 6) return -2;
  int nv = planar ? 4 : 6;
  int bad = 0;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int ii = 0; ii < nobj; ii++) {
    opot P = P0;
    ostat st = {0, max_attempts, 0};
    double *w = yo + (long)nv * ii;
    if (planar)
      polar_to_rect(w);
    else
      cyl_to_rect(w);
    double *out = result + (long)nv * nt * ii;
    if (run_plain(&P, planar, method, w, nt, t + (long)nt * ii * indiv_t, dt, rtol, atol, out,
                  &st))
      bad = 1;
    for (int jj = 0; jj < nt; jj++) {
      if (planar)
        rect_to_polar(out + nv * jj);
      else
        rect_to_cyl(out + nv * jj);
    }
    err[ii] = st.err;
    if (nsteps) nsteps[ii] = st.nsteps;
    if (nforce) nforce[ii] = P.nforce;
  }
  return bad ? -2 : 0;
}

/* Variational integration of nobj orbits, each with one deviation column,
   in rectangular coordinates (integrateFullOrbit.c:1234 /
   integratePlanarOrbit.c:940 per orbit).  yo: [nobj][4*dim] =
   (x..., v..., dx..., dv...); result [nobj][nt][4*dim]. */
EXPORT int oracle_integrate_dxdv(int planar, int nobj, const double *yo, int nt, const double *t,
                                 int indiv_t, int npot, const int *pot_type,
                                 const double *pot_args, double dt, double rtol, double atol,
                                 double *result, int *err, int method, long long *nsteps,
                                 int nthreads)
{
  opot P0;
  if (opot_decode(&P0, npot, pot_type, pot_args, planar)) return -3;
  if (method < 0 || method > 6) return -2;
  int dim = planar ? 2 : 3, nv = 4 * dim;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int ii = 0; ii < nobj; ii++) {
    opot P = P0;
    ostat st = {0, 0, 0};
    const double *w = yo + (long)nv * ii;
    const double *tt = t + (long)nt * ii * indiv_t;
    double *out = result + (long)nv * nt * ii;
    rhs_fn fa = planar ? rect_force2_dxdv : rect_force3_dxdv;
    rhs_fn fb = planar ? rect_force2 : rect_force3;
    rhs_fn fd = planar ? rect_deriv2_dxdv : rect_deriv3_dxdv;
    switch (method) {
    case 0: symplectic(&SCH_LF, fa, fb, &P, 2 * dim, dim, w, nt, dt, tt, rtol, atol, out, &st); break;
    case 3: symplectic(&SCH_S4, fa, fb, &P, 2 * dim, dim, w, nt, dt, tt, rtol, atol, out, &st); break;
    case 4: symplectic(&SCH_S6, fa, fb, &P, 2 * dim, dim, w, nt, dt, tt, rtol, atol, out, &st); break;
    case 1: rk_fixed(4, fd, &P, nv, w, nt, dt, tt, rtol, atol, out, &st); break;
    case 2: rk_fixed(6, fd, &P, nv, w, nt, dt, tt, rtol, atol, out, &st); break;
    case 5: dopr54(fd, &P, nv, w, nt, dt, tt, rtol, atol, out, &st); break;
    case 6: dop853(fd, &P, nv, w, nt, tt, rtol, atol, out, &st); break;
    }
    err[ii] = st.err;
    if (nsteps) nsteps[ii] = st.nsteps;
  }
  return 0;
}

/* Forces and Hessian terms at n points (R, z, phi), for unit tests.
   out[n][9] = Rforce, zforce, phitorque, R2deriv, z2deriv, Rzderiv,
   phi2deriv, Rphideriv, zphideriv; planar: out[n][5] = planarRforce,
   planarphitorque, planarR2deriv, planarphi2deriv, planarRphideriv; t the
   time (time-dependent components). */
EXPORT int oracle_forces(int planar, int n, const double *R, const double *z, const double *phi,
                         int npot, const int *pot_type, const double *pot_args, double *out,
                         double t)
{
  opot P;
  if (opot_decode(&P, npot, pot_type, pot_args, planar)) return -3;
  P.t = t;
  for (int i = 0; i < n; i++) {
    if (planar) {
      double Rf, pt, h0, h1, h2;
      sum2(&P, R[i], phi[i], &Rf, &pt);
      planar_hess_sum(&P, R[i], phi[i], &h0, &h1, &h2);
      double *o = out + 5L * i;
      o[0] = Rf;
      o[1] = pt;
      o[2] = h0;
      o[3] = h1;
      o[4] = h2;
    } else {
      double Rf, zf, pt, h[6];
      sum3(&P, R[i], z[i], phi[i], &Rf, &zf, &pt);
      hess3(&P, R[i], z[i], phi[i], h);
      double *o = out + 9L * i;
      o[0] = Rf;
      o[1] = zf;
      o[2] = pt;
      for (int w = 0; w < 6; w++) o[3 + w] = h[w];
    }
  }
  return 0;
}

/* Potential energy per unit mass, summed over components (evaluatePotentials,
   galpy_potentials.c:105-117). */
EXPORT int oracle_potential(int n, const double *R, const double *z, const double *phi, int npot,
                            const int *pot_type, const double *pot_args, double *out)
{
  opot P;
  if (opot_decode(&P, npot, pot_type, pot_args, 0)) return -3;
  for (int i = 0; i < n; i++) {
    double s = 0.;
    s = range_sum(&P, 0, P.n, Q_EVAL, R[i], z[i], phi[i]);
    out[i] = s;
  }
  return 0;
}

EXPORT double oracle_gammainc_P(double a, double x) { return oracle_gamma_inc_P(a, x); }
EXPORT double oracle_expint(double x) { return oracle_expint_E1(x); }
