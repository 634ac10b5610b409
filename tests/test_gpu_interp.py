"""Orbit interpolation between stored rows on a B200
(galpy_cuda_orbit_interp_device) against the oracle's restatement of the
not-a-knot interpolating spline (oracle/spline.py, pinned against scipy's
FITPACK in tests/test_oracle.py), and galpy's own Orbit.__call__ through the
hooks."""
import numpy as np
import pytest
from galpy_stub import import_galpy
from helpers import seeded_ics

import galpy_b200 as gb
from galpy_b200 import _lib
from galpy_b200.orbit_quantities import interpolate

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "GPU tests need a GPU"


def _rows(golden, n, t, planar, seed):
    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    ics = seeded_ics(n, seed, planar=planar)
    rows, err = gb.integrateFullOrbit_cuda((pt, pa), ics, t, "dop853_cuda", progressbar=False) \
        if not planar else gb.integratePlanarOrbit_cuda((pt, pa), ics, t, "dop853_cuda",
                                                         progressbar=False)
    assert not err.any()
    return rows


def _close(got, ref, nv):
    d = np.abs(got - ref)
    d[..., nv - 1] = np.abs(np.mod(got[..., -1] - ref[..., -1] + np.pi, 2 * np.pi) - np.pi)
    scale = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1.0)
    scale[..., nv - 1] = 1.0
    return (d / scale).max()


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("nt", [2, 3, 4, 5, 101])
def test_interpolation_vs_oracle_shared_times(golden, planar, nt):
    from oracle import spline

    t = np.linspace(0.0, 6.0, nt)
    rows = _rows(golden, 300, t, planar, 40 + nt)
    rng = np.random.default_rng(nt)
    # inside, at the rows, and a little outside (extrapolation by the end pieces)
    tq = np.concatenate([rng.uniform(0, 6, 50), t, [-0.05, 6.05]])
    got = interpolate(rows, t, tq)
    ref = spline.interpolate(rows, t, tq)
    assert _close(got, ref, rows.shape[-1]) < 1e-11
    # at the integration times the rows come back
    at = interpolate(rows, t, t)
    assert _close(at, rows, rows.shape[-1]) < 1e-12


def test_interpolation_per_orbit_times_and_queries(golden):
    from oracle import spline

    n = 257
    rng = np.random.default_rng(5)
    tend = np.exp(rng.normal(np.log(5.0), 0.5, n))
    t = np.linspace(0, 1, 41)[None, :] * tend[:, None]
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    rows, err = gb.integrateFullOrbit_cuda((pt, pa), seeded_ics(n, 6), t, "dop853_cuda",
                                           progressbar=False)
    assert not err.any()
    tq = rng.uniform(0, 1, (n, 17)) * tend[:, None]
    got = interpolate(rows, t, tq)
    ref = spline.interpolate(rows, t, tq)
    assert _close(got, ref, 6) < 1e-11
    # a shared query grid with per-orbit rows
    tq1 = np.linspace(0.1, 2.0, 9)
    assert _close(interpolate(rows, t, tq1), spline.interpolate(rows, t, tq1), 6) < 1e-11


def test_interpolation_of_a_backward_grid(golden):
    from oracle import spline

    t = -np.linspace(0, 4, 31)
    rows = _rows(golden, 64, t, False, 8)
    tq = -np.linspace(0.05, 3.95, 23)
    got = interpolate(rows, t, tq)
    ref = spline.interpolate(rows[:, ::-1], t[::-1], tq)
    assert _close(got, ref, 6) < 1e-11


def test_orbit_call_through_the_hooks():
    """galpy's own Orbit.__call__ between integration times with the real
    engine behind the hooks, against galpy's scipy path."""
    galpy = import_galpy()
    if galpy is None:
        pytest.skip("galpy not importable")
    from galpy.orbit import Orbit
    from galpy.potential import MWPotential2014

    from galpy_b200 import galpy_hooks

    ics = seeded_ics(200, 9)
    ts = np.linspace(0, 5, 51)
    tq = np.sort(np.random.default_rng(9).uniform(0, 5, 40))  # 8,000 pairs
    galpy_hooks.install()
    try:
        o = Orbit(ics)
        o.integrate(ts, MWPotential2014, method="dop853_cuda")
        got = o._call_internal(tq)
        R = o.R(tq)
    finally:
        galpy_hooks.uninstall()
    ref = o._call_internal(tq)
    assert got.shape == ref.shape == (6, 40, 200)
    d = np.abs(got[:5] - ref[:5]).max()
    dphi = np.abs(np.mod(got[5] - ref[5] + np.pi, 2 * np.pi) - np.pi).max()
    assert d < 1e-10 and dphi < 1e-10, (d, dphi)
    np.testing.assert_allclose(R, o.R(tq), rtol=1e-10)
