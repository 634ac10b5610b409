"""galpy's (pot_type, pot_args) for the time-dependent DehnenBarPotential and
the SCFPotential, built without galpy (TEST ONLY): the layouts of
galpy/orbit/integrateFullOrbit.py (DehnenBar: type 1, (amp * af, tform,
tsteady, rb, omegab, barphi); SCF: type 24 through _parse_scf_pot in
integratePlanarOrbit.py, (a, isNonAxi, N, L, M, Nt = 0, amp * Acos,
amp * Asin if non-axisymmetric, 11 cache slots)).  tests/test_timedep.py
checks them against galpy's own _parse_pot where galpy is importable."""
import numpy as np


def mw14(planar=False):
    """MWPotential2014's (types, args) as galpy marshals them, from the
    package's galpy-free parser."""
    import galpy_b200 as gb

    _, pt, pa = gb.parse_pot(gb.MWPotential2014(), planar=planar)
    return [int(x) for x in pt], [float(x) for x in pa]


def dehnen_bar_args(amp_af=0.01, tform=-2.0, tsteady=3.0, rb=0.8, omegab=1.85, barphi=0.4):
    return [amp_af, tform, tsteady, rb, omegab, barphi]


def scf_coefficients(N=6, L=5, nonaxi=True, seed=3):
    """Coefficients (Acos, Asin) of a smooth Hernquist-like expansion: the
    (0, 0, 0) term 1, the others small; m <= l only, Asin[..., 0] = 0."""
    rng = np.random.default_rng(seed)
    M = L if nonaxi else 1
    Acos = rng.normal(size=(N, L, M)) * 0.05
    Acos[0, 0, 0] = 1.0
    Asin = rng.normal(size=(N, L, M)) * 0.05 if nonaxi else None
    for l in range(L):
        Acos[:, l, l + 1:] = 0.0
        if nonaxi:
            Asin[:, l, l + 1:] = 0.0
    if nonaxi:
        Asin[:, :, 0] = 0.0
    return Acos, Asin


def scf_args(Acos, Asin=None, a=1.1, amp=1.0):
    N, L, M = Acos.shape
    nonaxi = Asin is not None
    out = [a, float(nonaxi), float(N), float(L), float(M), 0.0]
    out.extend((amp * Acos).ravel().tolist())
    if nonaxi:
        out.extend((amp * Asin).ravel().tolist())
    out.extend([-1.0] + [0.0] * 10)
    return out


def potential(name, planar=False):
    """(pot_type int32, pot_args float64) of a named test potential."""
    mw_t, mw_a = mw14(planar)
    if name == "bar+mw14":
        t, a = mw_t + [1], mw_a + dehnen_bar_args()
    elif name == "bar_growing+mw14":  # the bar grows during the integration
        t, a = mw_t + [1], mw_a + dehnen_bar_args(amp_af=0.02, tform=1.0, tsteady=6.0)
    elif name == "scf_nonaxi":
        t, a = [24], scf_args(*scf_coefficients(nonaxi=True), a=1.1)
    elif name == "scf_axi+mn":
        nb = 3 if planar else 5  # the bulge's argument count
        t, a = [24, 5], scf_args(*scf_coefficients(nonaxi=False), a=0.9) + mw_a[nb:nb + 3]
    else:
        raise KeyError(name)
    return np.asarray(t, np.int32), np.asarray(a, np.float64)


NAMES = ["bar+mw14", "bar_growing+mw14", "scf_nonaxi", "scf_axi+mn"]


def loghalo_triaxial_args():
    """galpy's LogarithmicHaloPotential args (amp, q, core^2, 1 - 1/b^2), b = 0.8."""
    return [0.5, 0.9, 0.01, 1.0 - 1.0 / 0.64]


def wrapped(name, planar=False):
    """(pot_type, pot_args, npot) of a wrapper around one component, next to
    MWPotential2014: galpy's layout (type, wrapped types; nwrapped, wrapped
    args, wrapper args), npot counting top-level entries."""
    mw_t, mw_a = mw14(planar)
    if name == "smooth(bar)+mw14":  # a bar that grows, then a wrapper that grows it again
        t, a = [-1, 1], [1] + dehnen_bar_args(amp_af=0.02) + [1.0, 0.5, 4.0, 1.0]
    elif name == "decay(bar)+mw14":  # DehnenSmooth with grow = 0: decaying
        t, a = [-1, 1], [1] + dehnen_bar_args(amp_af=0.02) + [1.0, 0.5, 4.0, 0.0]
    elif name == "rotate(loghalo)+mw14":  # a triaxial halo in solid-body rotation
        t, a = [-2, 0], [1] + loghalo_triaxial_args() + [1.0, 0.6, 0.3]
    elif name == "gauss(loghalo)+mw14":  # a triaxial halo with a Gaussian amplitude in time
        t, a = [-5, 0], [1] + loghalo_triaxial_args() + [1.0, 3.0, 4.0]
    elif name == "corot(needle)+mw14":  # a needle bar winding up with the rotation curve
        t, a = [-4, 25], [1] + needle_bar_args(amp=0.08, b=0.05, omegab=0.0) + \
            [1.0, 1.0, 0.1, 0.3, -1.0]
    elif name == "corot(loghalo)+mw14":  # a triaxial halo in differential rotation
        t, a = [-4, 0], [1] + loghalo_triaxial_args() + [1.0, 0.7, 0.8, 0.2, 0.5]
    elif name == "kuzmin(plummer)+mw14":  # KuzminLike: a flattened Plummer (amp, a, b^2)
        t, a = [-10, 17], [1, 0.3, 0.4] + [0.8, 0.5, 0.05]
    elif name == "kuzmin(hernquist,plummer)":  # two wrapped spheres, no other component
        mw_t, mw_a = [], []
        t, a = [-10, 8, 17], [2, 0.6, 0.7, 0.3, 0.2] + [1.2, 0.4, 0.01]
    else:
        raise KeyError(name)
    return (np.asarray(mw_t + t, np.int32), np.asarray(mw_a + a, np.float64), len(mw_t) + 1)


WRAPPED = ["smooth(bar)+mw14", "decay(bar)+mw14", "rotate(loghalo)+mw14", "gauss(loghalo)+mw14",
           "kuzmin(plummer)+mw14", "kuzmin(hernquist,plummer)", "corot(needle)+mw14",
           "corot(loghalo)+mw14"]


def crosses_bar_radius(ref_cyl, rb=0.8):
    """Orbits (cylindrical rows [n][nt][6|4]) whose radius r crosses the bar
    radius, where the bar potential's second derivative jumps: there
    DOP853's error estimate sits near 1 more often, and accept / reject
    decisions flip on rounding-level differences of the force."""
    R = ref_cyl[..., 0]
    z = ref_cyl[..., 3] if ref_cyl.shape[-1] == 6 else 0.0 * R
    r = np.sqrt(R * R + z * z)
    return (r.min(axis=1) < rb) & (r.max(axis=1) > rb)


def ulp_response(oracle, ics, t, pt, pa, method, planar, ref, seed=3, **kw):
    """Per-orbit change of the oracle's orbit under a one-ulp change of its
    initial conditions: the orbit's own conditioning."""
    from helpers import cyl_diff

    ulp = 1 + np.finfo(float).eps * np.random.default_rng(seed).choice([-1, 1], ics.shape)
    pert, _, _, _ = oracle.integrate(ics * ulp, t, pt, pa, method, planar=planar, **kw)
    return cyl_diff(ref, pert).max(axis=(1, 2))


def planar_perturbation(name):
    """(pot_type, pot_args) of MWPotential2014 in the plane plus one of
    galpy's planar disk perturbations (the layouts of integratePlanarOrbit.py):
    TransientLogSpiral (2), SteadyLogSpiral (3, grown or always on),
    EllipticalDisk (4), LopsidedDisk (6), CosmphiDisk (28)."""
    mw_t, mw_a = mw14(True)
    gam = np.pi / 4
    if name == "transspiral+mw14":
        t, a = [2], [1.0, -0.035, 5.0, 4.0, -7.0, 2.0, 0.65, gam]
    elif name == "steadyspiral+mw14":
        t, a = [3], [1.0, 1.0, 5.0, -0.035, -7.0, 2.0, 0.65, gam]
    elif name == "steadyspiral_on+mw14":
        t, a = [3], [1.0, float("nan"), float("nan"), -0.035, -7.0, 2.0, 0.65, gam]
    elif name == "elldisk+mw14":
        t, a = [4], [1.0, 0.5, 3.0, 0.02, 1.0, 0.4]
    elif name == "lopsided+mw14":
        t, a = [6], [1.0, 0.02, 1.0, 0.4]
    elif name == "cosmphi+mw14":
        rb, p = 0.6, 1.0
        t, a = [28], [1.0, 0.02, p, 0.8, 3.0, rb, rb**p, rb**(2 * p), 1.0]
    else:
        raise KeyError(name)
    return np.asarray(mw_t + t, np.int32), np.asarray(mw_a + a, np.float64)


PLANAR_PERTURBATIONS = ["transspiral+mw14", "steadyspiral+mw14", "steadyspiral_on+mw14",
                        "elldisk+mw14", "lopsided+mw14", "cosmphi+mw14"]


def spiral_arms_args(Cs=(1.0,), amp=1.0, N=2, alpha=0.2, r_ref=1.0, phi_ref=0.0, Rs=0.3,
                     H=0.125, omega=0.0):
    """SpiralArmsPotential's argument list (integrateFullOrbit.py's layout:
    nCs, amp, N, sin alpha, tan alpha, r_ref, phi_ref, Rs, H, omega, Cs) for
    the constructor's N and alpha, which galpy stores negated (trailing
    arms)."""
    return [float(len(Cs)), amp, float(-N), np.sin(-alpha), np.tan(-alpha), r_ref, phi_ref, Rs,
            H, omega] + [float(c) for c in Cs]


def spiral_arms(name, planar=False):
    """(pot_type, pot_args) of MWPotential2014 plus one SpiralArmsPotential
    (type 27): galpy's defaults set rotating, or four arms with three
    Fourier terms (the Cox & Gomez sinusoidal-density coefficients)."""
    mw_t, mw_a = mw14(planar)
    if name == "spiral+mw14":
        a = spiral_arms_args(omega=0.65)
    elif name == "spiral3+mw14":
        a = spiral_arms_args(Cs=(8 / (3 * np.pi), 0.5, 8 / (15 * np.pi)), amp=0.8, N=4,
                             alpha=np.deg2rad(12), r_ref=1.1, phi_ref=0.3, Rs=0.4, H=0.1,
                             omega=0.55)
    else:
        raise KeyError(name)
    return np.asarray(mw_t + [27], np.int32), np.asarray(mw_a + a, np.float64)


SPIRAL_ARMS = ["spiral+mw14", "spiral3+mw14"]


def needle_bar_args(amp=0.05, a=0.5, b=0.0, c=0.125, pa=0.4, omegab=1.8):
    """SoftenedNeedleBarPotential's argument list (amp, a, b, c^2, pa,
    omegab, and seven cache slots galpy passes as zeros)."""
    return [amp, a, b, c * c, pa, omegab] + [0.0] * 7


def needle_bar(name, planar=False):
    """(pot_type, pot_args) of MWPotential2014 plus a rotating softened
    needle bar (type 25): galpy's default shape, or a thick bar (b > 0)."""
    mw_t, mw_a = mw14(planar)
    if name == "needle+mw14":
        a = needle_bar_args()
    elif name == "needle_thick+mw14":
        a = needle_bar_args(amp=0.08, a=0.4, b=0.1, c=0.2, pa=-0.3, omegab=1.5)
    else:
        raise KeyError(name)
    return np.asarray(mw_t + [25], np.int32), np.asarray(mw_a + a, np.float64)


NEEDLE_BARS = ["needle+mw14", "needle_thick+mw14"]
