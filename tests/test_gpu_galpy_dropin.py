"""galpy's own ``Orbit.integrate`` driving the engine on a B200.

The drop-in path end to end: ``galpy_b200.galpy_hooks.install()`` patches
galpy's dispatch (galpy/orbit/Orbits.py:1733-1826), then
``Orbit(vxvv).integrate(ts, pot, method='<name>_cuda')`` runs the real
kernels and stores the result in the Orbit exactly as galpy's ``*_c`` methods
do.  Each result is checked against

* the oracle (the CPU restatement of galpy's C integrators), and
* galpy's own C integrators -- the reference's orbit_c_ext sources built by
  oracle/Makefile into oracle/_ref -- when that build is present,

for the four methods the engine's plain form is specified for (leapfrog,
symplec4, rk4, dop853), 3D and planar, in MWPotential2014, a Hernquist
sphere and the logarithmic halo (axisymmetric and triaxial).  The potential
arguments come from galpy's own ``_parse_pot`` in both arms.

galpy comes from the reference tree or from the pure-Python copy installed
into baseline/_ref (tests/galpy_stub.py); without either the module skips.

Tolerances: the fixed-step methods take the reference's step size per orbit
and agree to the orbits' own conditioning (<= 1e-10 on [0, 10]); DOP853
takes the same accepted steps on all but rare accept/reject flips at
err ~ 1, where the two results still agree inside the integrator tolerance.
"""
import numpy as np
import pytest
from galpy_stub import import_galpy
from helpers import cyl_diff, cyl_to_rect, rect_to_cyl, seeded_ics

galpy = import_galpy()
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(galpy is None, reason="no galpy copy (reference tree or "
                                 "baseline/_ref) to drive the engine")]

METHODS = ["leapfrog", "symplec4", "rk4", "dop853"]
POTENTIALS = ["MWPotential2014", "Hernquist", "LogHalo", "LogHaloTriaxial"]


@pytest.fixture(scope="module", autouse=True)
def hooks():
    from galpy_b200 import _lib, build, galpy_hooks

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "GPU tests need a GPU"
    galpy_hooks.install()
    yield
    galpy_hooks.uninstall()


def make_pot(name):
    from galpy import potential as P

    if name == "MWPotential2014":
        return P.MWPotential2014
    if name == "Hernquist":
        return P.HernquistPotential(normalize=1.0, a=0.8)
    if name == "LogHalo":
        return P.LogarithmicHaloPotential(normalize=1.0, q=0.9, core=0.1)
    return P.LogarithmicHaloPotential(normalize=1.0, q=0.9, b=0.8, core=0.1)


def parsed(pot, planar):
    """pot_type / pot_args exactly as galpy hands them to its C code."""
    if planar:
        from galpy.orbit.integratePlanarOrbit import _parse_pot
        from galpy.potential import toPlanarPotential

        pot = toPlanarPotential(pot)
    else:
        from galpy.orbit.integrateFullOrbit import _parse_pot
    npot, pt, pa, tfuncs = _parse_pot(pot)
    assert len(tfuncs) == 0
    return np.asarray(pt, np.int32), np.asarray(pa, np.float64)


def galpy_orbits(ics, ts, pot, method):
    from galpy.orbit import Orbit

    o = Orbit(ics)
    o.integrate(ts, pot, method=method, progressbar=False)
    return o.getOrbit()


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("potname", POTENTIALS)
def test_orbit_integrate_cuda(oracle, potname, planar, method):
    pot = make_pot(potname)
    pt, pa = parsed(pot, planar)
    ics = seeded_ics(96, 40 + POTENTIALS.index(potname), planar=planar)
    ts = np.linspace(0.0, 10.0, 101)
    out = galpy_orbits(ics, ts, pot, method + "_cuda")
    assert out.shape == ics.shape[:1] + ts.shape + ics.shape[1:]
    assert np.isfinite(out).all()
    # the Orbit stores the initial conditions as its first row (phi as
    # atan2 in (-pi, pi], as galpy's C returns it)
    assert cyl_diff(ics, out[:, 0]).max() < 1e-14
    ref, err, _, _ = oracle.integrate(ics, ts, pt, pa, method, planar=planar)
    assert not err.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    if method == "dop853":
        assert (d < 1e-10).mean() >= 0.97, (d < 1e-10).mean()
        assert d.max() < 1e-7, d.max()
    else:
        assert d.max() < 1e-10, d.max()
    if oracle.ref_available():
        refc, errc, _, _ = oracle.integrate(ics, ts, pt, pa, method, planar=planar, impl="ref")
        assert not errc.any()
        # the oracle is bit-identical to the reference's C (tests/test_oracle.py)
        assert np.array_equal(refc, ref)


@pytest.mark.parametrize("method", METHODS)
def test_orbit_integrate_cuda_matches_engine_call(method):
    """The Orbit path and a direct call of the galpy-facing wrapper give the
    same numbers (the hooks add no conversion of their own)."""
    import galpy_b200 as gb
    from galpy.potential import MWPotential2014

    ics = seeded_ics(64, 47)
    ts = np.linspace(0.0, 5.0, 51)
    out = galpy_orbits(ics, ts, MWPotential2014, method + "_cuda")
    direct, err = gb.integrateFullOrbit_cuda(MWPotential2014, ics.copy(), ts, method + "_cuda",
                                             progressbar=False)
    assert not err.any()
    assert np.array_equal(out, direct)


def test_orbit_integrate_cuda_ragged_times(oracle):
    """Per-orbit time arrays (galpy's indiv_t) with dop853_cuda, unevenly
    spaced, through Orbit.integrate."""
    from galpy.potential import MWPotential2014

    pt, pa = parsed(MWPotential2014, False)
    ics = seeded_ics(48, 48)
    rng = np.random.default_rng(48)
    tend = rng.uniform(2.0, 20.0, len(ics))
    ts = np.sort(rng.uniform(0, 1, (len(ics), 31)), axis=1)
    ts[:, 0] = 0.0
    ts = ts * tend[:, None]
    out = galpy_orbits(ics, ts, MWPotential2014, "dop853_cuda")
    ref, err, _, _ = oracle.integrate(ics, ts, pt, pa, "dop853")
    assert not err.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    assert (d < 1e-10).mean() >= 0.97 and d.max() < 1e-7, d.max()


def test_unsupported_potential_keeps_galpy_path():
    """A potential the engine does not implement runs galpy's own
    integrator (the hooks fall back to galpy's method of the same name)."""
    from galpy.orbit import Orbit
    from galpy.potential import TwoPowerSphericalPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    o.integrate(np.linspace(0, 1, 11), TwoPowerSphericalPotential(alpha=1.5, beta=3.5),
                method="dop853_cuda", progressbar=False)
    assert np.isfinite(o.getOrbit()).all()


@pytest.mark.parametrize("planar", [False, True])
def test_orbit_integrate_dxdv_cuda(oracle, planar):
    """Orbit.integrate_dxdv(method='dop853_cuda'): every (orbit, deviation)
    pair in one GPU launch (galpy maps its single-orbit C integrator over
    the orbits in Python, Orbits.py:2445), against the reference's own
    variational C integrator run orbit by orbit (oracle/_ref) where present,
    else the oracle (bit-identical to it)."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    ics = seeded_ics(128, 49, planar=planar)
    n, nv = ics.shape
    dxdv = np.random.default_rng(49).normal(size=(n, nv)) * 1e-4
    ts = np.linspace(0, 10, 101)
    o = Orbit(ics)
    o.integrate_dxdv(dxdv, ts, MWPotential2014, method="dop853_cuda", rectIn=True,
                     rectOut=True, rtol=1e-11, atol=1e-11, progressbar=False)
    # orbit_dxdv: orbit (cylindrical) then deviation (rectangular, rectOut)
    # columns; getOrbit_dxdv() returns the deviation columns alone
    got = o.orbit_dxdv
    assert np.array_equal(o.getOrbit_dxdv(), got[..., nv:])
    pt, pa = parsed(MWPotential2014, planar)
    w = np.hstack([cyl_to_rect(ics), dxdv])
    impl = "ref" if oracle.ref_available() else "port"
    ref, err, _ = oracle.integrate_dxdv(w, ts, pt, pa, "dop853", planar=planar, rtol=1e-11,
                                        atol=1e-11, impl=impl)
    assert not err.any()
    d = np.abs(got[..., nv:] - ref[..., nv:]) / np.abs(ref[..., nv:]).max(axis=1, keepdims=True)
    assert np.quantile(d.max(axis=(1, 2)), 0.97) < 1e-9 and d.max() < 1e-6, d.max()
    assert cyl_diff(rect_to_cyl(ref[..., :nv]), got[..., :nv]).max() < 1e-6


def test_orbit_lyapunov_cuda():
    """Orbit.lyapunov(method='dop853_cuda') against galpy's own pure-Python
    dop853 estimate (same algorithm, renormalisation every 10 outputs)."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    ics = seeded_ics(8, 50)
    ts = np.linspace(0, 20, 41)
    lam = Orbit(ics).lyapunov(ts, MWPotential2014, method="dop853_cuda", rtol=1e-12,
                              atol=1e-12)
    ref = Orbit(ics).lyapunov(ts, MWPotential2014, method="dop853", rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(lam[:, 1:], ref[:, 1:], rtol=1e-6, atol=1e-9)


def test_orbit_energy_and_jacobi_on_device():
    """Orbit.E and Orbit.Jacobi after a dop853_cuda integration: the routed
    potential sums (GPU) against galpy's own (hooks removed)."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    from galpy_b200 import galpy_hooks

    ics = seeded_ics(256, 51)
    ts = np.linspace(0, 10, 51)
    o = Orbit(ics)
    o.integrate(ts, MWPotential2014, method="dop853_cuda", progressbar=False)
    E, J = o.E(ts), o.Jacobi(ts, OmegaP=0.4)
    galpy_hooks.uninstall()
    try:
        Eref, Jref = o.E(ts), o.Jacobi(ts, OmegaP=0.4)
    finally:
        galpy_hooks.install()
    np.testing.assert_allclose(E, Eref, rtol=1e-13)
    np.testing.assert_allclose(J, Jref, rtol=1e-13)
