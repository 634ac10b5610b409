"""The CPU oracle (oracle/galpy_oracle.c) pinned against the reference.

* bit-for-bit against the reference's own C integrators built from its
  sources (oracle/_ref), when that build is present;
* against the committed golden vectors made from the reference's C build and
  from galpy's Python (tests/golden/make_golden.py), everywhere;
* against scipy for the incomplete gamma function of the bulge mass (the
  reference calls GSL there, which is not part of the reference tree).
"""
import numpy as np
import pytest
from helpers import ADDED_POTS, cyl_to_rect, golden_pot, seeded_ics

METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
def test_oracle_bitwise_vs_reference_build(oracle, mw14, mw14_planar, method, planar):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built here (needs the reference tree)")
    pt, pa = mw14_planar if planar else mw14
    ics = seeded_ics(16, 3, planar=planar)
    t = np.linspace(0, 20, 201)
    a, ea, _, _ = oracle.integrate(ics, t, pt, pa, method, planar=planar)
    b, eb, _, _ = oracle.integrate(ics, t, pt, pa, method, planar=planar, impl="ref")
    assert np.array_equal(a, b)
    assert np.array_equal(ea, eb)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
def test_oracle_dxdv_bitwise_vs_reference_build(oracle, mw14, mw14_planar, method, planar):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built here (needs the reference tree)")
    pt, pa = mw14_planar if planar else mw14
    dim = 2 if planar else 3
    ics = seeded_ics(2 * dim, 4, planar=planar)
    w = np.zeros((2 * dim, 4 * dim))
    w[:, :2 * dim] = cyl_to_rect(ics)
    w[np.arange(2 * dim), 2 * dim + np.arange(2 * dim)] = 1.0
    t = np.linspace(0, 4, 41)
    a, _, _ = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar)
    b, _, _ = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, impl="ref")
    assert np.array_equal(a, b)


@pytest.mark.parametrize("method", METHODS)
def test_oracle_matches_golden_c_vectors(oracle, golden, method):
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    t = np.linspace(0, 5, 51)
    a, _, _, _ = oracle.integrate(golden["c_ics"], t, pt, pa, method)
    np.testing.assert_allclose(a, golden[f"c_{method}_3d"], rtol=0, atol=1e-13)
    pt2, pa2 = golden["mw14_planar_type"], golden["mw14_planar_args"]
    a, _, _, _ = oracle.integrate(golden["c_ics_planar"], t, pt2, pa2, method, planar=True)
    np.testing.assert_allclose(a, golden[f"c_{method}_planar"], rtol=0, atol=1e-13)
    t = np.linspace(0, 3, 31)
    a, _, _ = oracle.integrate_dxdv(golden["c_dxdv_w3"], t, pt, pa, method)
    np.testing.assert_allclose(a, golden[f"c_{method}_dxdv3"], rtol=0, atol=1e-12)
    a, _, _ = oracle.integrate_dxdv(golden["c_dxdv_w2"], t, pt2, pa2, method, planar=True)
    np.testing.assert_allclose(a, golden[f"c_{method}_dxdv2"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("method", ["dop853", "dopr54"])
def test_oracle_indiv_t_golden(oracle, golden, method):
    a, _, _, _ = oracle.integrate(golden["c_ics"], golden["c_indiv_t"], golden["mw14_type"],
                                  golden["mw14_args"], method, rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(a, golden[f"c_{method}_indiv"], rtol=0, atol=1e-13)


def test_oracle_dopr54_forced_steps_golden(oracle, golden):
    """dopr54's smallest-step rule (bovy_rk.c:598-604): an unreachable
    tolerance forces every step to the interval's first step / 10000 and
    flags err = 1, as the reference's own C does on the same input."""
    a, err, nsteps, _ = oracle.integrate(golden["c_ics"], np.array([0.0, 50.0]),
                                         golden["mw14_type"], golden["mw14_args"], "dopr54",
                                         dt=50.0, rtol=1e-20, atol=1e-20)
    np.testing.assert_array_equal(err, golden["c_dopr54_forced_err"])
    assert np.all(err == 1)
    assert np.all(nsteps == 10000)
    np.testing.assert_allclose(a, golden["c_dopr54_forced"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("method", ["rk6", "symplec6", "dopr54"])
def test_oracle_bitwise_vs_reference_build_edge_cases(oracle, mw14, method):
    """Backward integration over per-orbit time grids and an explicit step."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built here (needs the reference tree)")
    pt, pa = mw14
    ics = seeded_ics(8, 6)
    tt = -np.linspace(0, 1, 21)[None, :] * np.linspace(3.0, 9.0, 8)[:, None]
    for kw in ({"rtol": 1e-9, "atol": 1e-9}, {"dt": -0.01}):
        a, ea, _, _ = oracle.integrate(ics, tt, pt, pa, method, **kw)
        b, eb, _, _ = oracle.integrate(ics, tt, pt, pa, method, impl="ref", **kw)
        assert np.array_equal(a, b)
        assert np.array_equal(ea, eb)


def test_incomplete_gamma_vs_scipy(oracle):
    from scipy.special import gammainc

    worst = 0.0
    for a in (0.1, 0.6, 0.9, 1.2, 2.5, 7.0):
        for x in np.concatenate([np.geomspace(1e-6, 300, 400), [a + 1 - 1e-12, a + 1]]):
            ref = gammainc(a, x)
            got = oracle.gammainc_P(a, x)
            worst = max(worst, abs(got - ref) / max(ref, 1e-300))
    assert worst < 5e-14, worst


def test_exponential_integral_vs_scipy(oracle):
    """E1 for ExpTruncNFW (the reference calls GSL's gsl_sf_expint_E1)."""
    from scipy.special import exp1

    xs = np.concatenate([np.geomspace(1e-8, 1.0, 300), np.geomspace(1.0, 600.0, 300)])
    worst = max(abs(oracle.expint_E1(x) - exp1(x)) / exp1(x) for x in xs)
    assert worst < 2e-14, worst


@pytest.mark.parametrize("name", ["mw14", "hernquist", "loghalo", "logtri", "nfw", "mn", "pswc"]
                         + ADDED_POTS)
def test_oracle_forces_vs_galpy_python(oracle, golden, name):
    """C-side formulas restated in the oracle agree with galpy's Python
    potentials (different code, same mathematics)."""
    pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
    R, z, phi = golden["pts_R"], golden["pts_z"], golden["pts_phi"]
    py = golden[f"{name}_pyforces"]
    f = oracle.forces(R, z, phi, pt, pa)
    pot = oracle.potential(R, z, phi, pt, pa)
    got = np.stack([f[:, 0], f[:, 1], f[:, 2], f[:, 3], f[:, 4], f[:, 5], pot], 1)
    if name == "null":  # zero forces; galpy's Python value is the constant amp, C has none
        assert not got[:, :6].any() and np.all(py[:, :6] == 0)
        return
    scale = np.abs(py).max(0) + 1e-300
    err = np.abs(got - py) / scale
    assert err.max() < 1e-11, err.max(0)


@pytest.mark.parametrize("name", ADDED_POTS)
def test_oracle_spherical_potentials(oracle, golden, name):
    """The reference's own C in each spherical potential: golden vectors
    (dop853 3D, symplec4 planar, dop853 variational) and, where the reference
    build is present, bit for bit over all methods."""
    pt, pa = golden_pot(golden, name)
    pt2, pa2 = golden_pot(golden, name, planar=True)
    t = np.linspace(0, 5, 51)
    a, _, _, _ = oracle.integrate(golden["c_ics"], t, pt, pa, "dop853")
    np.testing.assert_allclose(a, golden[f"sph_{name}_3d"], rtol=0, atol=1e-13)
    a, _, _, _ = oracle.integrate(golden["c_ics_planar"], t, pt2, pa2, "symplec4", planar=True)
    np.testing.assert_allclose(a, golden[f"sph_{name}_planar"], rtol=0, atol=1e-13)
    a, _, _ = oracle.integrate_dxdv(golden["sph_dxdv_w3"], t, pt, pa, "dop853")
    np.testing.assert_allclose(a, golden[f"sph_{name}_dxdv3"], rtol=0, atol=1e-12)
    if not oracle.ref_available():
        return
    ics = seeded_ics(6, 7)
    ics2 = seeded_ics(6, 8, planar=True)
    t = np.linspace(0, 8, 41)
    for m in ("leapfrog", "symplec4", "symplec6", "rk4", "rk6", "dopr54", "dop853"):
        a, ea, _, _ = oracle.integrate(ics, t, pt, pa, m, rtol=1e-10, atol=1e-10)
        b, eb, _, _ = oracle.integrate(ics, t, pt, pa, m, rtol=1e-10, atol=1e-10, impl="ref")
        assert np.array_equal(a, b) and np.array_equal(ea, eb), m
        a, _, _, _ = oracle.integrate(ics2, t, pt2, pa2, m, planar=True, rtol=1e-10, atol=1e-10)
        b, _, _, _ = oracle.integrate(ics2, t, pt2, pa2, m, planar=True, rtol=1e-10, atol=1e-10,
                                      impl="ref")
        assert np.array_equal(a, b), m
    w = np.zeros((4, 8))
    w[:, :4] = cyl_to_rect(ics2[:4])
    w[np.arange(4), 4 + np.arange(4)] = 1.0
    for m in ("symplec4", "dop853"):
        a, _, _ = oracle.integrate_dxdv(w, t, pt2, pa2, m, planar=True)
        b, _, _ = oracle.integrate_dxdv(w, t, pt2, pa2, m, planar=True, impl="ref")
        assert np.array_equal(a, b), m


def test_oracle_dop853_vs_galpy_python_dop853(oracle, golden):
    """The C DOP853 (default tol 1e-12) against galpy's pure-Python DOP853."""
    a, _, _, _ = oracle.integrate(golden["pydop_ics"], golden["pydop_t"], golden["mw14_type"],
                                  golden["mw14_args"], "dop853")
    d = np.abs(a - golden["pydop_orbit"])
    d[..., 5] = np.abs((a[..., 5] - golden["pydop_orbit"][..., 5] + np.pi) % (2 * np.pi) - np.pi)
    assert d.max() < 1e-7, d.max()


def test_oracle_dop853_vs_galpy_python_dop853_added_potentials(oracle, golden):
    """The C DOP853 against galpy's pure-Python DOP853 in the planar
    HenonHeiles and the 3D TriaxialHernquist potentials."""
    ts = np.linspace(0.0, 10.0, 51)
    a, _, _, _ = oracle.integrate(golden["hh_ics"][:3], ts, golden["hh_type"],
                                  golden["hh_args"], "dop853", planar=True)
    ref = golden["pydop_hh_orbit"]
    d = np.abs(a - ref)
    d[..., 3] = np.abs((a[..., 3] - ref[..., 3] + np.pi) % (2 * np.pi) - np.pi)
    assert d.max() < 1e-7, d.max()
    a, _, _, _ = oracle.integrate(golden["pydop_trihern_ics"], ts, golden["ell_trihern_type"],
                                  golden["ell_trihern_args"], "dop853")
    ref = golden["pydop_trihern_orbit"]
    d = np.abs(a - ref)
    d[..., 5] = np.abs((a[..., 5] - ref[..., 5] + np.pi) % (2 * np.pi) - np.pi)
    assert d.max() < 1e-7, d.max()


@pytest.mark.parametrize("method", METHODS)
def test_oracle_energy_conservation(oracle, mw14, method):
    """galpy's test_energy_jacobi_conservation criterion
    (tests/test_orbit.py:111, conftest.py:656): (std E / mean E)^2 < 1e-10."""
    pt, pa = mw14
    ics = seeded_ics(4, 5)
    t = np.linspace(0, 14, 501)
    res, err, _, _ = oracle.integrate(ics, t, pt, pa, method)
    assert not err.any()
    E = oracle.energy_cyl(res, pt, pa)
    assert np.all((E.std(1) / E.mean(1)) ** 2 < 1e-10)


SOS_METHODS = ["rk4", "rk6", "dopr54", "dop853"]


@pytest.mark.parametrize("method", SOS_METHODS)
def test_oracle_surface_of_section(oracle, golden, method):
    """integrateFullOrbit_sos (integrateFullOrbit.c:1151-1233, evalSOSDeriv
    :1353-1390): golden vectors of the reference's C, and bit for bit
    against the reference build (MWPotential2014, the triaxial logarithmic
    halo, per-orbit increments) where it is present."""
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    a, err, _ = oracle.integrate_sos(golden["sos_yo"], golden["sos_psi"], pt, pa, method,
                                     rtol=1e-10, atol=1e-10)
    assert not err.any()
    np.testing.assert_allclose(a, golden[f"sos_{method}"], rtol=0, atol=1e-12)
    if method == "dop853":
        a, _, _ = oracle.integrate_sos(golden["sos_yo"], golden["sos_psi_indiv"], pt, pa,
                                       method, rtol=1e-10, atol=1e-10)
        np.testing.assert_allclose(a, golden["sos_dop853_indiv"], rtol=0, atol=1e-12)
    if not oracle.ref_available():
        return
    # (not the Plummer sphere: one of these orbits makes the reference's
    # dop853 reject its smallest step forever)
    for name in ("mw14", "logtri", "flatpower"):
        pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
        yo = np.concatenate([seeded_ics(6, 9), np.zeros((6, 1))], 1)
        psi = np.linspace(0.0, 12.0 * np.pi, 7)
        for kw in ({"rtol": 1e-9, "atol": 1e-9}, {"dpsi": 0.05}):
            a, ea, _ = oracle.integrate_sos(yo, psi, pt, pa, method, **kw)
            b, eb, _ = oracle.integrate_sos(yo, psi, pt, pa, method, impl="ref", **kw)
            assert np.array_equal(a, b) and np.array_equal(ea, eb), (name, kw)


@pytest.mark.parametrize("surface", [0, 1])
def test_oracle_planar_surface_of_section(oracle, golden, surface):
    """integratePlanarOrbit_sos (integratePlanarOrbit.c:848-939, 1056-1123)
    for the surfaces x = 0 and y = 0: golden vectors of the reference's C and,
    where the reference build is present, bit for bit."""
    pt, pa = golden["mw14_planar_type"], golden["mw14_planar_args"]
    for m in SOS_METHODS:
        a, err, _ = oracle.integrate_sos(golden["sos_planar_yo"], golden["sos_psi"], pt, pa, m,
                                         rtol=1e-10, atol=1e-10, planar=True, surface=surface)
        assert not err.any()
        np.testing.assert_allclose(a, golden[f"sos_planar{surface}_{m}"], rtol=0, atol=1e-12)
    if not oracle.ref_available():
        return
    yo = np.concatenate([seeded_ics(6, 10, planar=True), np.zeros((6, 1))], 1)
    psi = np.linspace(0.0, 12.0 * np.pi, 7)
    for name in ("logtri", "flatpower"):
        ptn = golden.get(f"{name}_planar_type", golden[f"{name}_type"])
        pan = golden.get(f"{name}_planar_args", golden[f"{name}_args"])
        for m in SOS_METHODS:
            a, ea, _ = oracle.integrate_sos(yo, psi, ptn, pan, m, rtol=1e-9, atol=1e-9,
                                            planar=True, surface=surface)
            b, eb, _ = oracle.integrate_sos(yo, psi, ptn, pan, m, rtol=1e-9, atol=1e-9,
                                            planar=True, surface=surface, impl="ref")
            assert np.array_equal(a, b) and np.array_equal(ea, eb), (name, m)


# --- orbit interpolation between stored rows (oracle/spline.py) ----------

@pytest.mark.parametrize("m", [2, 3, 4, 5, 11, 101])
def test_spline_oracle_vs_scipy_fitpack(m):
    """The restated interpolant against scipy's FITPACK splines, which
    galpy's Orbit.__call__ evaluates: InterpolatedUnivariateSpline with
    k = min(3, m - 1) (per-orbit grids) and RectBivariateSpline(kx=3, ky=1,
    s=0) at integer orbit indices (shared grids, m >= 4)."""
    from scipy import interpolate as si

    from oracle import spline

    rng = np.random.default_rng(m)
    t = np.sort(rng.uniform(0, 10, m)) if m > 4 else np.linspace(0, 3, m)
    ys = np.stack([np.sin(1.3 * t + k) * (1 + 0.1 * k) for k in range(5)])
    tq = np.concatenate([rng.uniform(t[0], t[-1], 40), t, [t[0], t[-1]]])
    for y in ys:
        ref = si.InterpolatedUnivariateSpline(t, y, k=min(3, m - 1))(tq)
        got = spline.interp1(t, y, tq)
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(y).max()), m
    if m >= 4:
        rb = si.RectBivariateSpline(t, np.arange(5), ys.T, ky=1, s=0.0)
        ref2 = rb(np.sort(tq), np.arange(5))
        got2 = np.stack([spline.interp1(t, y, np.sort(tq)) for y in ys], 1)
        assert np.allclose(got2, ref2, rtol=1e-11, atol=1e-12)


def test_spline_oracle_unpacks_like_galpy():
    """R and phi are interpolated as x = R cos phi and y = R sin phi and
    unpacked with sqrt and atan2, as Orbit.__call__ does (phase wrapping of
    phi between rows does not matter)."""
    from scipy import interpolate as si

    from oracle import spline

    t = np.linspace(0, 5, 21)
    R = 1 + 0.2 * np.sin(t)
    phi = np.mod(1.7 * t, 2 * np.pi) - np.pi  # wraps
    rows = np.stack([R, 0.1 * np.cos(t), R * 1.7, phi], 1)[None]
    tq = np.linspace(0.05, 4.95, 33)
    got = spline.interpolate(rows, t, tq)[0]
    x = si.InterpolatedUnivariateSpline(t, R * np.cos(phi), k=3)(tq)
    y = si.InterpolatedUnivariateSpline(t, R * np.sin(phi), k=3)(tq)
    assert np.allclose(got[:, 0], np.sqrt(x * x + y * y), rtol=1e-12)
    assert np.allclose(got[:, 3], np.arctan2(y, x), atol=1e-12)
    assert np.allclose(got[:, 1], si.InterpolatedUnivariateSpline(t, rows[0, :, 1], k=3)(tq),
                       atol=1e-13)
