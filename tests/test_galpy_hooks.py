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
                 max_attempts, return_nsteps, device):
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
    from galpy.potential import SCFPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    o.integrate(np.linspace(0, 1, 11), SCFPotential(normalize=1.0), method="dop853_cuda")
    assert hooks == []  # galpy's own integrator ran


def test_spherical_potential_routes(hooks):
    from galpy.orbit import Orbit
    from galpy.potential import PlummerPotential

    o = Orbit([1.0, 0.1, 1.1, 0.0, 0.1, 0.0])
    o.integrate(np.linspace(0, 1, 11), PlummerPotential(normalize=1.0), method="dopr54_cuda")
    assert len(hooks) == 1 and hooks[-1]["method"] == "dopr54_cuda"
    assert type(hooks[-1]["pot"]).__name__ == "PlummerPotential"


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
