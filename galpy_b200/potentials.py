"""Potentials supported by the engine, with galpy's parameter conventions.

The engine integrates in the potentials galpy hands to C as pot_type codes
0 (LogarithmicHaloPotential), 5 (MiyamotoNagaiPotential), 8
(HernquistPotential), 9 (NFWPotential), 15 (PowerSphericalPotentialwCutoff)
12 (FlattenedPower), 16 (KuzminKutuzovStaeckel) and the spherical 7 (PowerSpherical / Kepler), 10
(Jaffe), 14 (Isochrone),
17 (Plummer), 18 (PseudoIsothermal), 20 (Burkert), 33
(DehnenCoreSpherical), 34 (DehnenSpherical), 35 (HomogeneousSphere), 40
(Null), 41 (Einasto) and 46 (ExpTruncNFW), the time-dependent 1
(DehnenBar) and 24 (SCF, static coefficients), and the wrappers -1
(DehnenSmooth), -2 (SolidBodyRotation) and -5 (GaussianAmplitude) around
them, and in the plane 2, 3, 4, 6 and 28 (the log spirals and the
elliptical, lopsided and cos(m phi) disks) -- the parsing is
galpy/orbit/integrateFullOrbit.py:43-614 (3D) and
galpy/orbit/integratePlanarOrbit.py:33-663 (planar).

``parse_pot`` accepts
  * galpy potential instances (or lists of them) -- galpy's own ``_parse_pot``
    is used, so the arguments are exactly galpy's;
  * the light-weight classes below, which reproduce galpy's constructors for
    the five potentials of types 0, 5, 8, 9 and 15 (amp, scale parameters
    and ``normalize``) for use without galpy;
  * an already-parsed ``(pot_type, pot_args)`` pair.
"""
import math

import numpy as np

T_LOGHALO, T_MN, T_HERNQUIST, T_NFW, T_PSWC = 0, 5, 8, 9, 15
# spherical: PowerSpherical (and Kepler), Jaffe, Isochrone, Plummer,
# PseudoIsothermal, Burkert, DehnenCoreSpherical, DehnenSpherical,
# HomogeneousSphere, Null, Einasto, ExpTruncNFW
SPHERICAL_TYPES = (7, 10, 14, 17, 18, 20, 33, 34, 35, 40, 41, 46)
T_FLATPOWER, T_KKS = 12, 16
T_HENONHEILES = 29  # planar only
T_KUZMINDISK = 19
# EllipsoidalPotential family: TriaxialHernquist, TriaxialNFW, TriaxialJaffe,
# PerfectEllipsoid, TriaxialGaussian, PowerTriaxial, TwoPowerTriaxial
ELLIPSOIDAL_TYPES = (21, 22, 23, 30, 37, 38, 43)
# DehnenBarPotential (its force depends on the time) and SCFPotential (the
# Hernquist-Ostriker expansion; static coefficients only)
T_DEHNENBAR, T_SCF = 1, 24
# wrappers around other components (one level deep): DehnenSmooth,
# SolidBodyRotation, CorotatingRotation, GaussianAmplitude, KuzminLike
WRAPPER_TYPES = (-1, -2, -4, -5, -10)
# planar disk perturbations: TransientLogSpiral, SteadyLogSpiral,
# EllipticalDisk, LopsidedDisk, CosmphiDisk (no potential evaluation in C)
DISK_PERTURBATION_TYPES = (2, 3, 4, 6, 28)
# SpiralArmsPotential (Cox & Gomez arms rotating at omega; up to six terms)
# and the rotating SoftenedNeedleBarPotential
T_SPIRALARMS, T_NEEDLEBAR = 27, 25
TIME_DEPENDENT_TYPES = (T_DEHNENBAR, T_SPIRALARMS, T_NEEDLEBAR) + WRAPPER_TYPES + \
    DISK_PERTURBATION_TYPES
SUPPORTED_TYPES = (T_LOGHALO, T_MN, T_HERNQUIST, T_NFW, T_PSWC, T_FLATPOWER,
                   T_KKS, T_HENONHEILES, T_KUZMINDISK, T_DEHNENBAR, T_SCF,
                   T_SPIRALARMS, T_NEEDLEBAR) + SPHERICAL_TYPES + \
    ELLIPSOIDAL_TYPES + WRAPPER_TYPES + DISK_PERTURBATION_TYPES


class _Potential:
    """Base: Rforce_amp1(R, z) is the radial force for amp = 1."""

    def _apply_normalize(self, normalize):
        if normalize is not False and normalize is not None:
            # galpy's Potential.normalize (galpy/potential/Potential.py:902-920):
            # scale amp so that -Rforce(1, 0) = normalize
            self._amp = self._amp * float(normalize) / abs(self.Rforce(1.0, 0.0))

    def Rforce(self, R, z):
        return self._amp * self._Rforce_amp1(R, z)

    def c_args(self, planar=False):
        raise NotImplementedError


class PowerSphericalPotentialwCutoff(_Potential):
    """rho ~ amp r^-alpha exp(-(r/rc)^2) (galpy/potential/PowerSphericalPotentialwCutoff.py)."""

    pot_type = T_PSWC

    def __init__(self, amp=1.0, alpha=1.0, rc=1.0, normalize=False):
        self._amp = float(amp)
        self.alpha = float(alpha)
        self.rc = float(rc)
        self._apply_normalize(normalize)

    def _mass(self, r2):
        from scipy.special import gamma, gammainc

        a = 1.5 - 0.5 * self.alpha
        return 2.0 * math.pi * self.rc ** (3.0 - self.alpha) * gamma(a) * gammainc(
            a, r2 / self.rc**2)

    def _Rforce_amp1(self, R, z):
        r2 = R * R + z * z
        return -self._mass(r2) / r2**1.5 * R

    def c_args(self, planar=False):
        args = [self._amp, self.alpha, self.rc]
        return args if planar else args + [0.0, 0.0]  # two cache slots in 3D


class MiyamotoNagaiPotential(_Potential):
    pot_type = T_MN

    def __init__(self, amp=1.0, a=1.0, b=0.1, normalize=False):
        self._amp = float(amp)
        self._a = float(a)
        self._b = float(b)
        self._apply_normalize(normalize)

    def _Rforce_amp1(self, R, z):
        return -R * (R * R + (self._a + math.sqrt(z * z + self._b**2)) ** 2) ** -1.5

    def c_args(self, planar=False):
        return [self._amp, self._a, self._b]


class NFWPotential(_Potential):
    pot_type = T_NFW

    def __init__(self, amp=1.0, a=1.0, normalize=False):
        self._amp = float(amp)
        self.a = float(a)
        self._apply_normalize(normalize)

    def _Rforce_amp1(self, R, z):
        r2 = R * R + z * z
        r = math.sqrt(r2)
        return R * (1.0 / r2 / (self.a + r) - math.log(1.0 + r / self.a) / r / r2)

    def c_args(self, planar=False):
        return [self._amp, self.a]


class HernquistPotential(_Potential):
    """Phi = -amp / (2 (r + a)) (galpy's amp is twice the mass)."""

    pot_type = T_HERNQUIST

    def __init__(self, amp=1.0, a=1.0, normalize=False):
        self._amp = float(amp)
        self.a = float(a)
        self._apply_normalize(normalize)

    def _Rforce_amp1(self, R, z):
        r = math.sqrt(R * R + z * z)
        return -R / (2.0 * r * (r + self.a) ** 2)

    def c_args(self, planar=False):
        return [self._amp, self.a]


class LogarithmicHaloPotential(_Potential):
    """Phi = amp/2 ln(R^2 (1 - (1-1/b^2) sin^2 phi) + (z/q)^2 + core^2)."""

    pot_type = T_LOGHALO

    def __init__(self, amp=1.0, core=1e-8, q=1.0, b=None, normalize=False):
        self._amp = float(amp)
        self._core2 = float(core) ** 2
        self._q = float(q)
        self.isNonAxi = b is not None and b != 1.0
        self._1m1overb2 = 1.0 - 1.0 / float(b) ** 2 if self.isNonAxi else 2.0
        self._apply_normalize(normalize)

    def _Rforce_amp1(self, R, z):
        return -R / (R * R + (z / self._q) ** 2 + self._core2)

    def c_args(self, planar=False):
        return [self._amp, self._q, self._core2, self._1m1overb2]


def MWPotential2014():
    """galpy's MWPotential2014 (galpy/potential/mwpotentials.py:25-29)."""
    return [
        PowerSphericalPotentialwCutoff(normalize=0.05, alpha=1.8, rc=1.9 / 8.0),
        MiyamotoNagaiPotential(a=3.0 / 8.0, b=0.28 / 8.0, normalize=0.6),
        NFWPotential(a=16 / 8.0, normalize=0.35),
    ]


def _is_galpy(p):
    mod = type(p).__module__ or ""
    return mod.startswith("galpy.")


def parse_pot(pot, planar=False):
    """(npot, pot_type int32[], pot_args float64[]) for the C ABI.  An
    already-parsed potential is (pot_type, pot_args), or (pot_type,
    pot_args, npot) when a wrapper's wrapped types make galpy's count of
    top-level entries npot differ from len(pot_type)."""
    if isinstance(pot, tuple) and len(pot) in (2, 3) and not isinstance(pot[0], _Potential):
        pt = np.ascontiguousarray(pot[0], dtype=np.int32)
        pa = np.ascontiguousarray(pot[1], dtype=np.float64)
        return (int(pot[2]) if len(pot) == 3 else len(pt)), pt, pa
    plist = pot if isinstance(pot, (list, tuple)) else [pot]
    if any(_is_galpy(p) for p in plist):
        if planar:
            from galpy.orbit.integratePlanarOrbit import _parse_pot as gparse
        else:
            from galpy.orbit.integrateFullOrbit import _parse_pot as gparse
        npot, pt, pa, tfuncs = gparse(pot)
        if len(tfuncs):
            raise NotImplementedError("time-dependent potentials are not supported on the GPU")
        return int(npot), np.ascontiguousarray(pt, np.int32), np.ascontiguousarray(pa, np.float64)
    types, args = [], []
    for p in plist:
        if not isinstance(p, _Potential):
            raise TypeError(f"unsupported potential {p!r}")
        types.append(p.pot_type)
        args.extend(p.c_args(planar=planar))
    return len(types), np.asarray(types, np.int32), np.asarray(args, np.float64)


def supported(pot_type):
    return all(int(t) in SUPPORTED_TYPES for t in np.atleast_1d(pot_type))
