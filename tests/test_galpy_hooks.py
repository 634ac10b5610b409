"""galpy's Orbit.integrate dispatching the *_cuda methods to this package.

Runs galpy from the reference tree (skipped where that tree is absent).  On
CPU machines the engine call is replaced by a recorder, so the test checks the
dispatch and argument passing; the GPU suite checks the engine itself."""
import numpy as np
import pytest
from galpy_stub import import_galpy

galpy = import_galpy()
pytestmark = pytest.mark.skipif(galpy is None, reason="galpy reference tree not available")


@pytest.fixture()
def hooks(monkeypatch):
    from galpy_b200 import galpy_hooks, integrate

    calls = []

    def recorder(planar, pot, yo, t, int_method, rtol, atol, progressbar, dt, precision,
                 max_attempts, return_nsteps, device, stream_rows=-1, devices=None):
        calls.append(dict(planar=planar, pot=pot, yo=np.array(yo), t=np.array(t),
                          method=int_method, rtol=rtol, atol=atol, dt=dt))
        yo2 = np.atleast_2d(yo)
        out = np.repeat(yo2[:, None, :], np.asarray(t).shape[-1], axis=1)
        err = np.zeros(len(yo2), np.int32)
        return (out[0], err[0]) if np.ndim(yo) == 1 else (out, err)

    monkeypatch.setattr(integrate, "_integrate_c", recorder)
    galpy_hooks.install()
    yield calls
    galpy_hooks.uninstall()


def test_orbit_integrate_routes_cuda_methods(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    vxvv = [[1.0, 0.1, 1.1, 0.05, 0.02, 0.3], [1.5, -0.1, 0.9, -0.02, 0.01, 2.0]]
    o = Orbit(vxvv)
    ts = np.linspace(0, 10, 101)
    for method in ("leapfrog_cuda", "rk4_cuda", "symplec4_cuda", "dop853_cuda"):
        o.integrate(ts, MWPotential2014, method=method)
        call = hooks[-1]
        assert call["method"] == method and not call["planar"]
        assert call["yo"].shape == (2, 6)
        np.testing.assert_allclose(call["yo"], np.array(vxvv))
        np.testing.assert_allclose(call["t"], ts)
        # the recorder returns the initial condition at every time
        np.testing.assert_allclose(o.R(ts[-1]), [1.0, 1.5])
    assert len(hooks) == 4


def test_planar_orbit_routes(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    o = Orbit([[1.0, 0.1, 1.1, 0.3]])
    o.integrate(np.linspace(0, 5, 11), MWPotential2014, method="dop853_cuda")
    assert hooks[-1]["planar"] and hooks[-1]["yo"].shape == (1, 4)


def test_unsupported_potential_falls_back(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import TwoPowerSphericalPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    o.integrate(np.linspace(0, 1, 11), TwoPowerSphericalPotential(alpha=1.5, beta=3.5),
                method="dop853_cuda")
    assert hooks == []  # galpy's own integrator ran


def test_bar_and_scf_route(hooks):
    """The time-dependent DehnenBarPotential and a static SCFPotential go to
    the engine; an SCF expansion with time-dependent coefficients stays with
    galpy."""
    from galpy.orbit import Orbit
    from galpy.potential import DehnenBarPotential, MWPotential2014, SCFPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    o.integrate(np.linspace(0, 1, 11), [*MWPotential2014, DehnenBarPotential()],
                method="dop853_cuda")
    assert len(hooks) == 1
    o.integrate(np.linspace(0, 1, 11), SCFPotential(normalize=1.0), method="rk4_cuda")
    assert len(hooks) == 2 and hooks[-1]["method"] == "rk4_cuda"
    Acos = np.zeros((2, 1, 1, 1))
    Acos[:, 0, 0, 0] = [1.0, 1.2]
    try:
        tdep = SCFPotential(Acos=Acos, tgrid=np.array([0.0, 2.0]))
    except TypeError:  # a galpy without time-dependent SCF coefficients
        return
    o.integrate(np.linspace(0, 1, 11), tdep, method="rk4_cuda")
    assert len(hooks) == 2


def test_spiral_arms_route(hooks):
    """SpiralArmsPotential goes to the engine with up to six Fourier terms;
    more stay with galpy."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014, SpiralArmsPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    arms = SpiralArmsPotential(N=4, omega=0.6, Cs=[1.0, 0.5, 0.2])
    o.integrate(np.linspace(0, 1, 11), [*MWPotential2014, arms], method="dop853_cuda")
    assert len(hooks) == 1
    o.integrate(np.linspace(0, 1, 11), SpiralArmsPotential(Cs=[1.0] * 7), method="dop853_cuda")
    assert len(hooks) == 1


def test_needle_bar_routes(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014, SoftenedNeedleBarPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    bar = SoftenedNeedleBarPotential(amp=0.05, a=0.5, c=0.125, omegab=1.8)
    o.integrate(np.linspace(0, 1, 11), [*MWPotential2014, bar], method="rk4_cuda")
    assert len(hooks) == 1 and hooks[-1]["method"] == "rk4_cuda"


def test_spherical_potential_routes(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import PlummerPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    o.integrate(np.linspace(0, 1, 11), PlummerPotential(normalize=1.0), method="dopr54_cuda")
    assert len(hooks) == 1 and hooks[-1]["method"] == "dopr54_cuda"
    assert type(hooks[-1]["pot"]).__name__ == "PlummerPotential"


def test_wrappers_route(hooks):
    """Wrapped potentials go to the engine; a wrapper inside a wrapper stays
    with galpy."""
    from galpy.orbit import Orbit
    from galpy.potential import (DehnenBarPotential, DehnenSmoothWrapperPotential,
                                 LogarithmicHaloPotential, MWPotential2014,
                                 SolidBodyRotationWrapperPotential)

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    ts = np.linspace(0, 1, 11)
    bar = DehnenSmoothWrapperPotential(pot=DehnenBarPotential(), tform=0.5, tsteady=2.0)
    o.integrate(ts, [*MWPotential2014, bar], method="dop853_cuda")
    assert len(hooks) == 1
    halo = SolidBodyRotationWrapperPotential(
        pot=LogarithmicHaloPotential(normalize=0.5, b=0.8, q=0.9), omega=0.6)
    o.integrate(ts, [*MWPotential2014, halo], method="rk4_cuda")
    assert len(hooks) == 2
    nested = DehnenSmoothWrapperPotential(pot=halo, tform=0.5, tsteady=2.0)
    o.integrate(ts, [*MWPotential2014, nested], method="rk4_cuda")
    assert len(hooks) == 2
    from galpy.potential import KuzminLikeWrapperPotential, PlummerPotential

    disk = KuzminLikeWrapperPotential(pot=PlummerPotential(amp=0.5, b=0.4), a=0.3, b=0.1)
    o.integrate(ts, [*MWPotential2014, disk], method="dopr54_cuda")
    assert len(hooks) == 3
    from galpy.potential import CorotatingRotationWrapperPotential

    wound = CorotatingRotationWrapperPotential(pot=DehnenBarPotential(), vpo=1.0, beta=0.1)
    o.integrate(ts, [*MWPotential2014, wound], method="dop853_cuda")
    assert len(hooks) == 4


def test_unknown_method_still_rejected(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    with pytest.raises(ValueError):
        o.integrate(np.linspace(0, 1, 11), MWPotential2014, method="euler_cuda")


def test_integrate_sos_routes(monkeypatch):
    """Orbit.integrate_SOS with a *_cuda method reaches
    integrateFullOrbit_sos_cuda (orbits without phi padded and unpadded as
    galpy's C branch does); symplectic *_cuda methods are refused as galpy
    refuses symplec4_c there."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    from galpy_b200 import galpy_hooks

    calls = []

    def fake(pot, yo, psi, t0, int_method, **kw):
        calls.append((np.array(yo).shape, int_method))
        yo = np.atleast_2d(yo)
        out = np.zeros((len(yo), len(psi), 7))
        out[..., :6] = yo[:, None, :6]
        out[..., 6] = psi  # time increasing with psi
        return out, np.zeros(len(yo), np.int32)

    monkeypatch.setattr(galpy_hooks, "integrateFullOrbit_sos_cuda", fake)
    galpy_hooks.install()
    try:
        psi = np.linspace(0, 10 * np.pi, 6)
        o = Orbit([[1.0, 0.1, 1.1, 0.05, 0.02, 0.3], [1.2, 0.0, 1.0, 0.1, 0.0, 1.0]])
        o.integrate_SOS(psi, MWPotential2014, method="dop853_cuda")
        assert calls[-1] == ((2, 6), "dop853_cuda") and o.orbit.shape == (2, 6, 6)
        o5 = Orbit([[1.0, 0.1, 1.1, 0.05, 0.02]])
        o5.integrate_SOS(psi, MWPotential2014, method="dopr54_cuda")
        assert calls[-1][0] == (1, 6) and o5.orbit.shape == (1, 6, 5)
        with pytest.raises(ValueError, match="symplec4_cuda"):
            o.integrate_SOS(psi, MWPotential2014, method="symplec4_cuda")
    finally:
        galpy_hooks.uninstall()


def test_planar_integrate_sos_routes(monkeypatch):
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    from galpy_b200 import galpy_hooks

    calls = []

    def fake(pot, yo, psi, t0, int_method, **kw):
        calls.append((np.array(yo).shape, int_method, kw.get("surface", "x")))
        yo = np.atleast_2d(yo)
        out = np.zeros((len(yo), len(psi), 5))
        out[..., :4] = yo[:, None, :4]
        out[..., 4] = psi
        return out, np.zeros(len(yo), np.int32)

    monkeypatch.setattr(galpy_hooks, "integratePlanarOrbit_sos_cuda", fake)
    galpy_hooks.install()
    try:
        psi = np.linspace(0, 10 * np.pi, 6)
        o = Orbit([[1.0, 0.1, 1.1, 0.3], [1.2, 0.0, 1.0, 1.0]])
        o.integrate_SOS(psi, MWPotential2014, method="rk4_cuda", surface="y")
        assert calls[-1] == ((2, 4), "rk4_cuda", "y") and o.orbit.shape == (2, 6, 4)
        o3 = Orbit([[1.0, 0.1, 1.1]])
        o3.integrate_SOS(psi, MWPotential2014, method="dop853_cuda")
        assert calls[-1][0] == (1, 4) and calls[-1][2] == "x" and o3.orbit.shape == (1, 6, 3)
    finally:
        galpy_hooks.uninstall()


@pytest.mark.parametrize("pot_name, kwargs, planar", [
    ("TriaxialNFWPotential", dict(amp=2.0, a=2.0, b=0.9, c=0.7, pa=0.3), False),
    ("PerfectEllipsoidPotential", dict(amp=1.1, a=1.2, b=0.9, c=0.8), False),
    ("KuzminDiskPotential", dict(amp=1.3, a=0.7), False),
    ("HenonHeilesPotential", dict(amp=1.0), True),
])
def test_added_potential_types_route(hooks, pot_name, kwargs, planar):
    """The ellipsoidal family, KuzminDisk and the planar HenonHeiles reach the
    engine (their parsed types are in the supported set)."""
    from galpy import potential
    from galpy.orbit import Orbit

    pot = getattr(potential, pot_name)(**kwargs)
    vxvv = [0.3, 0.05, 0.25, 0.5] if planar else [1.0, 0.1, 1.1, 0.05, 0.02, 0.3]
    o = Orbit(vxvv)
    o.integrate(np.linspace(0, 1, 11), pot, method="dop853_cuda")
    assert len(hooks) == 1 and hooks[-1]["planar"] == planar
    assert type(hooks[-1]["pot"]).__name__ == pot_name


@pytest.fixture()
def host_engine(monkeypatch, harness, oracle):
    """The hooks with the engine's variational integration run by the host
    build of the device code (tests/harness) and the potential sums by the
    oracle: galpy's own integrate_dxdv, lyapunov and E then run the routed
    paths on the CPU with real numbers."""
    from galpy_b200 import galpy_hooks, integrate, orbit_quantities
    from galpy_b200.potentials import parse_pot

    calls = []

    def batch(pot, w, t, int_method, planar=False, dt=None, rtol=None, atol=None, **kw):
        _, pt, pa = parse_pot(pot, planar=planar)
        calls.append(("dxdv", int_method, np.shape(w)))
        out, err, _ = harness.integrate(w, t, pt, pa, int_method[: -len("_cuda")],
                                        planar=planar, var=True, dt=dt, rtol=rtol, atol=atol)
        return out, err

    def potvals(pot, R, z=0.0, phi=0.0, planar=False):
        _, pt, pa = parse_pot(pot, planar=planar)
        calls.append(("phi", np.size(R)))
        R, z, phi = np.broadcast_arrays(R, z, phi)
        return oracle.potential(R.ravel(), z.ravel(), phi.ravel(), pt, pa).reshape(R.shape)

    def interp(rows, t, tq):
        from oracle import spline

        calls.append(("interp", np.shape(rows), np.size(tq)))
        t = np.asarray(t)
        if t.size > 1 and t[1] < t[0]:
            t, rows = t[::-1], np.asarray(rows)[:, ::-1]
        return spline.interpolate(rows, t, tq)

    monkeypatch.setattr(integrate, "integrate_dxdv_batch", batch)
    monkeypatch.setattr(orbit_quantities, "potential_values", potvals)
    monkeypatch.setattr(orbit_quantities, "interpolate", interp)
    galpy_hooks.install()
    yield calls
    galpy_hooks.uninstall()


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("rect", [False, True])
def test_integrate_dxdv_routes(host_engine, planar, rect):
    """Orbit.integrate_dxdv with dop853_cuda: one batched call for all
    orbits, galpy's coordinate conventions around it (cylindrical or
    rectangular deviations in and out), the same numbers as galpy's own
    pure-Python dop853 variational integration."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    vxvv = ([[1.0, 0.1, 1.1, 0.3], [1.3, -0.05, 0.9, 2.0], [0.8, 0.02, 1.2, -1.0]] if planar
            else [[1.0, 0.1, 1.1, 0.05, 0.02, 0.3], [1.3, -0.05, 0.9, -0.1, 0.03, 2.0]])
    n, nv = len(vxvv), len(vxvv[0])
    dxdv = np.random.default_rng(5).normal(size=(n, nv)) * 1e-3
    ts = np.linspace(0, 5, 51)
    o = Orbit(vxvv)
    o.integrate_dxdv(dxdv, ts, MWPotential2014, method="dop853_cuda", rectIn=rect,
                     rectOut=rect, rtol=1e-12, atol=1e-12)
    assert [c[0] for c in host_engine] == ["dxdv"]  # one batched call
    assert host_engine[0][2] == (n, 2 * nv)
    ref = Orbit(vxvv)
    ref.integrate_dxdv(dxdv, ts, MWPotential2014, method="dop853", rectIn=rect, rectOut=rect,
                       rtol=1e-12, atol=1e-12)
    got, want = o.getOrbit_dxdv(), ref.getOrbit_dxdv()
    assert got.shape == want.shape
    d = np.abs(got - want)
    k = nv - 1  # phi of the base orbit, compared modulo 2 pi
    d[..., k] = np.abs((got[..., k] - want[..., k] + np.pi) % (2 * np.pi) - np.pi)
    scale = np.abs(want).max(axis=1, keepdims=True)
    assert (d / scale).max() < 1e-8, (d / scale).max()


def test_lyapunov_routes(host_engine):
    """Orbit.lyapunov with dop853_cuda runs its renormalisation segments
    through the routed integrate_dxdv and agrees with galpy's pure-Python
    dop853 estimate."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    vxvv = [[1.0, 0.1, 1.1, 0.05, 0.02, 0.3], [1.3, -0.05, 0.9, -0.1, 0.03, 2.0]]
    ts = np.linspace(0, 20, 41)
    lam = Orbit(vxvv).lyapunov(ts, MWPotential2014, method="dop853_cuda", renorm_every=10,
                               rtol=1e-12, atol=1e-12)
    assert sum(c[0] == "dxdv" for c in host_engine) == 4  # one call per segment
    ref = Orbit(vxvv).lyapunov(ts, MWPotential2014, method="dop853", renorm_every=10,
                               rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(lam[:, 1:], ref[:, 1:], rtol=1e-7, atol=1e-10)


def test_energy_and_jacobi_route_potential_sums(host_engine):
    """Orbit.E and Orbit.Jacobi over many stored points take the potential
    sum from the engine (here its oracle stand-in); few points stay with
    galpy."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    from galpy_b200 import galpy_hooks

    rng = np.random.default_rng(9)
    n = 64
    vxvv = np.stack([rng.uniform(0.5, 2, n), rng.normal(0, 0.1, n), 1 + rng.normal(0, 0.1, n),
                     rng.normal(0, 0.05, n), rng.normal(0, 0.05, n),
                     rng.uniform(0, 2 * np.pi, n)], 1)
    ts = np.linspace(0, 2, 101)  # 64 x 101 = 6,464 points: above the threshold
    o = Orbit(vxvv)
    o.integrate(ts, MWPotential2014, method="dop853")  # galpy's own integrator
    E = o.E(ts)
    J = o.Jacobi(ts, OmegaP=0.3)
    assert sum(c[0] == "phi" for c in host_engine) == 2
    galpy_hooks.uninstall()
    Eref, Jref = o.E(ts), o.Jacobi(ts, OmegaP=0.3)
    galpy_hooks.install()
    np.testing.assert_allclose(E, Eref, rtol=1e-13)
    np.testing.assert_allclose(J, Jref, rtol=1e-13)
    host_engine.clear()
    o.E(ts[:2])  # 128 points: galpy's own sum
    assert not host_engine


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("backward", [False, True])
def test_orbit_call_between_times_routes_interpolation(host_engine, planar, backward):
    """Orbit.__call__ (and o.R(t), o.phi(t), ...) at times between the
    integration times of many orbits takes the interpolation from the engine
    (here its oracle stand-in, pinned against scipy's FITPACK in
    tests/test_oracle.py); the integration times themselves, times outside
    the integrated range and small requests stay with galpy."""
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    from galpy_b200 import galpy_hooks

    rng = np.random.default_rng(12)
    n = 64
    vxvv = np.stack([rng.uniform(0.5, 2, n), rng.normal(0, 0.1, n), 1 + rng.normal(0, 0.1, n),
                     rng.normal(0, 0.05, n), rng.normal(0, 0.05, n),
                     rng.uniform(0, 2 * np.pi, n)], 1)
    if planar:
        vxvv = vxvv[:, [0, 1, 2, 5]]
    ts = np.linspace(0, 3, 61)
    if backward:
        ts = -ts
    o = Orbit(vxvv)
    pot = MWPotential2014 if not planar else [p.toPlanar() for p in MWPotential2014]
    o.integrate(ts, pot, method="dop853")  # galpy's own integrator
    tq = np.sort(rng.uniform(ts.min(), ts.max(), 80))  # 64 x 80 = 5,120 pairs
    host_engine.clear()
    got = o._call_internal(tq)
    R, phi = o.R(tq), o.phi(tq)
    assert [c[0] for c in host_engine] == ["interp"] * 3
    galpy_hooks.uninstall()
    ref = o._call_internal(tq)
    Rref, phiref = o.R(tq), o.phi(tq)
    galpy_hooks.install()
    assert got.shape == ref.shape == ((4 if planar else 6), 80, n)
    np.testing.assert_allclose(got[:-1], ref[:-1], rtol=1e-10, atol=1e-12)
    dphi = np.mod(got[-1] - ref[-1] + np.pi, 2 * np.pi) - np.pi
    assert np.abs(dphi).max() < 1e-10
    np.testing.assert_allclose(R, Rref, rtol=1e-10)
    assert np.abs(np.mod(phi - phiref + np.pi, 2 * np.pi) - np.pi).max() < 1e-10
    host_engine.clear()
    o._call_internal(ts)  # the integration times: galpy's fast path
    o._call_internal(tq[:10])  # 640 pairs: galpy's own splines
    with pytest.raises(ValueError):
        o._call_internal(np.array([ts.max() + 1.0, 0.5]) * (-1 if backward else 1) * 10)
    assert not host_engine
