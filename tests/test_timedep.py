"""The oracle's DehnenBarPotential (time-dependent) and SCFPotential against
the reference's own C (oracle/_ref, built from DehnenBarPotential.c and
SCFPotential.c with the stand-in Gegenbauer / Legendre arrays) and against
galpy's Python potentials (scipy's special functions).

The time the reference hands each force evaluation follows its steppers'
own bookkeeping (leapfrog's to + dt/2, the symplectic drifts summed into
`to`, the RK stage offsets tn + c dt, dop853's t_current + c h and t_old +
c h, the state's time in a surface of section); the oracle restates it, so
the comparison is bit for bit."""
import numpy as np
import pytest

import timedep_pots as TP
from oracle import oracle

METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def ics(n, planar, seed=11):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.5, 1.5, n)
    vR = rng.normal(0, 0.1, n)
    vT = rng.uniform(0.8, 1.1, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    if planar:
        return np.stack([R, vR, vT, phi], 1)
    return np.stack([R, vR, vT, rng.normal(0, 0.1, n), rng.normal(0, 0.1, n), phi], 1)


def tol(method):
    return dict(rtol=1e-10, atol=1e-10) if method in ("dopr54", "dop853") else {}


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.NAMES)
@pytest.mark.parametrize("method", METHODS)
def test_orbits_bit_exact_vs_reference_build(name, planar, method):
    pt, pa = TP.potential(name, planar)
    yo = ics(8, planar)
    t = np.linspace(0.0, 8.0, 41)
    a, ea, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, **tol(method))
    b, eb, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, impl="ref", **tol(method))
    np.testing.assert_array_equal(ea, eb)
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["bar_growing+mw14", "scf_nonaxi"])
@pytest.mark.parametrize("method", METHODS)
def test_dxdv_bit_exact_vs_reference_build(name, planar, method):
    pt, pa = TP.potential(name, planar)
    dim = 2 if planar else 3
    rng = np.random.default_rng(5)
    w = np.concatenate([rng.uniform(0.6, 1.2, (4, dim)), rng.normal(0, 0.2, (4, dim)),
                        rng.normal(0, 1, (4, 2 * dim))], 1)
    w[:, dim + 1] += 1.0
    t = np.linspace(0.0, 4.0, 17)
    a = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, **tol(method))[0]
    b = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, impl="ref", **tol(method))[0]
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("method", ["rk4", "dop853"])
def test_sos_time_from_state_vs_reference_build(method):
    """The surface of section's force time is the state's (integrated) time."""
    pt, pa = TP.potential("bar_growing+mw14")
    yo = np.concatenate([ics(4, False), np.full((4, 1), 0.5)], 1)
    psi = np.linspace(0.0, 6 * np.pi, 25)
    a, _, _ = oracle.integrate_sos(yo, psi, pt, pa, method, **tol(method))
    b, _, _ = oracle.integrate_sos(yo, psi, pt, pa, method, impl="ref", **tol(method))
    np.testing.assert_array_equal(a, b)


def test_bar_force_follows_time():
    """The bar's force at a point changes with its pattern rotation and its
    growth; zero before tform."""
    pt, pa = TP.potential("bar_growing+mw14")
    R, z, phi = np.array([0.7]), np.array([0.1]), np.array([0.3])
    f_early = oracle.forces(R, z, phi, pt[3:], pa[-6:], t=0.5)
    assert np.all(f_early == 0.0)
    f1 = oracle.forces(R, z, phi, pt[3:], pa[-6:], t=2.0)
    f2 = oracle.forces(R, z, phi, pt[3:], pa[-6:], t=2.3)
    assert np.all(np.abs(f1[0, :3]) > 0) and not np.allclose(f1, f2)


def galpy_or_skip():
    import galpy_stub

    if galpy_stub.import_galpy() is None:
        pytest.skip("galpy not importable")
    from galpy import potential as P

    return P


@pytest.mark.parametrize("planar", [False, True])
def test_argument_layouts_match_galpy(planar):
    P = galpy_or_skip()
    if planar:
        from galpy.orbit.integratePlanarOrbit import _parse_pot
    else:
        from galpy.orbit.integrateFullOrbit import _parse_pot
    bar = P.DehnenBarPotential(omegab=1.85, rb=0.8, Af=0.01, tform=-2.0, tsteady=3.0, barphi=0.4)
    pots = [bar] if not planar else [P.toPlanarPotential(bar)]
    _, pt, pa, _ = _parse_pot(pots)
    assert list(pt) == [1]
    # galpy keeps tform / tsteady in absolute times (given in bar periods)
    np.testing.assert_array_equal(
        pa, TP.dehnen_bar_args(bar._amp * bar._af, bar._tform, bar._tsteady, bar._rb,
                               bar._omegab, bar._barphi))
    Acos, Asin = TP.scf_coefficients(nonaxi=True)
    scf = P.SCFPotential(amp=1.0, Acos=Acos, Asin=Asin, a=1.1)
    _, pt, pa, _ = _parse_pot([scf] if not planar else [P.toPlanarPotential(scf)])
    assert list(pt) == [24]
    # galpy folds its spherical-harmonic normalisation into the coefficients
    np.testing.assert_array_equal(np.asarray(pa),
                                  TP.scf_args(scf._Acos, scf._Asin, a=scf._a, amp=scf._amp))


@pytest.mark.parametrize("nonaxi", [True, False])
def test_scf_forces_vs_galpy_python(nonaxi):
    """Forces and second derivatives of the oracle's SCF (own Gegenbauer and
    Legendre recurrences) against galpy's Python SCFPotential (scipy)."""
    P = galpy_or_skip()
    Acos, Asin = TP.scf_coefficients(nonaxi=nonaxi)
    pot = P.SCFPotential(amp=1.0, Acos=Acos, Asin=Asin, a=1.1)
    rng = np.random.default_rng(2)
    R, z, phi = rng.uniform(0.3, 2, 60), rng.normal(0, 0.5, 60), rng.uniform(0, 6.2, 60)
    args = TP.scf_args(pot._Acos, pot._Asin if nonaxi else None, a=pot._a, amp=pot._amp)
    got = oracle.forces(R, z, phi, np.array([24], np.int32), np.array(args))
    names = ["Rforce", "zforce", "phitorque", "R2deriv", "z2deriv", "Rzderiv", "phi2deriv",
             "Rphideriv", "phizderiv"]
    for k, nm in enumerate(names):
        ref = np.array([getattr(pot, nm)(R[i], z[i], phi=phi[i], use_physical=False)
                        for i in range(R.size)])
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got[:, k] - ref).max() <= 1e-13 * scale, nm


# ---- the engine's machines and forces, compiled as host C++ (harness) -------
def c2r(v, planar):
    if planar:
        R, vR, vT, p = v.T
        c, s = np.cos(p), np.sin(p)
        return np.stack([R * c, R * s, vR * c - vT * s, vR * s + vT * c], 1)
    R, vR, vT, z, vz, p = v.T
    c, s = np.cos(p), np.sin(p)
    return np.stack([R * c, R * s, z, vR * c - vT * s, vR * s + vT * c, vz], 1)


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.NAMES)
def test_engine_forces_at_times(harness, name, planar):
    """The engine's Cartesian forces (the bar's quadratic form, the SCF
    recurrences) against the oracle's cylindrical restatement at several
    times."""
    pt, pa = TP.potential(name, planar)
    rng = np.random.default_rng(6)
    R = rng.uniform(0.3, 2.0, 200)
    z = np.zeros(200) if planar else rng.normal(0, 0.4, 200)
    phi = rng.uniform(0, 2 * np.pi, 200)
    for t in (0.0, 2.5, 7.0):
        f = oracle.forces(R, z, phi, pt, pa, planar=planar, t=t)
        tq = f[:, 1] if planar else f[:, 2]
        ax = np.cos(phi) * f[:, 0] - np.sin(phi) * tq / R
        ay = np.sin(phi) * f[:, 0] + np.cos(phi) * tq / R
        acc, _, _ = harness.forces(R * np.cos(phi), R * np.sin(phi), z, pt, pa, planar=planar,
                                   t=t)
        ref = np.stack([ax, ay] + ([] if planar else [f[:, 1]]), 1)
        scale = np.abs(ref).max()
        assert np.abs(acc[:, :ref.shape[1]] - ref).max() < 1e-14 * scale, t


@pytest.mark.parametrize("planar", [False, True])
def test_engine_bar_tidal_tensor(harness, planar):
    """K = -grad grad Phi of the bar (engine: Cartesian closed form) against
    the oracle's cylindrical second derivatives."""
    pt, pa = np.array([1], np.int32), np.array(TP.dehnen_bar_args())
    rng = np.random.default_rng(8)
    R = rng.uniform(0.3, 2.0, 100)
    z = np.zeros(100) if planar else rng.normal(0, 0.4, 100)
    phi = rng.uniform(0, 2 * np.pi, 100)
    x, y = R * np.cos(phi), R * np.sin(phi)
    _, K, _ = harness.forces(x, y, z, pt, pa, planar=planar, t=1.3)
    # central differences of the engine's own accelerations
    h = 1e-6
    cols = [(0, 0), (0, 1), (1, 1)] + ([] if planar else [(0, 2), (1, 2), (2, 2)])
    for k, (i, j) in enumerate(cols):
        dp = [x, y, z]
        dm = [x, y, z]
        dp = [v + (h if m == j else 0) for m, v in enumerate(dp)]
        dm = [v - (h if m == j else 0) for m, v in enumerate(dm)]
        ap, _, _ = harness.forces(*dp, pt, pa, planar=planar, t=1.3)
        am, _, _ = harness.forces(*dm, pt, pa, planar=planar, t=1.3)
        fd = (ap[:, i] - am[:, i]) / (2 * h)
        assert np.abs(K[:, k] - fd).max() < 1e-6 * max(np.abs(fd).max(), 1e-3), (i, j)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["bar+mw14", "bar_growing+mw14", "scf_axi+mn"])
def test_engine_machines_vs_oracle(harness, name, planar, method):
    """The engine's stepper machines with their force times (host build)
    against the oracle: same step sizes; DOP853 the same steps on orbits
    that stay on one side of the bar radius."""
    pt, pa = TP.potential(name, planar)
    y0 = ics(24, planar, seed=21)
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, _, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar, **tol(method))
    out, err, ns = harness.integrate(c2r(y0, planar), t, pt, pa, method, planar=planar,
                                     **tol(method))
    assert not err.any()
    ref_r = np.stack([c2r(ref[:, j], planar) for j in range(len(t))], 1)
    d = np.abs(out - ref_r).reshape(len(y0), -1).max(1)
    same = ns == nref
    kink = TP.crosses_bar_radius(ref) if name.startswith("bar") and method == "dop853" else \
        np.zeros(len(ns), bool)
    assert same[~kink].all()
    strict = same & ~kink
    assert np.median(d[strict]) < 1e-12 and d[strict].max() < 1e-9, d[strict].max()
    assert (d < 1e-6).all()


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["scf_nonaxi", "scf_axi+mn"])
def test_engine_scf_tidal_tensor(harness, name, planar):
    """K = -grad grad Phi of the SCF expansion (engine: second derivatives
    by the recurrences, chain rule to cylindrical, then Cartesian) against
    the oracle's cylindrical second derivatives (the reference's
    compute_scf_hessian_cyl, bit-exact with it)."""
    pt, pa = TP.potential(name, planar)
    rng = np.random.default_rng(12)
    R = rng.uniform(0.3, 2.0, 150)
    z = np.zeros(150) if planar else rng.normal(0, 0.4, 150)
    phi = rng.uniform(0, 2 * np.pi, 150)
    c, s = np.cos(phi), np.sin(phi)
    _, K, _ = harness.forces(R * c, R * s, z, pt, pa, planar=planar)
    f = oracle.forces(R, z, phi, pt, pa, planar=planar)
    if planar:
        Rf, tq, R2, p2, Rp = f.T
        z2 = Rz = zp = np.zeros_like(R)
    else:
        Rf, zf, tq, R2, z2, Rz, p2, Rp, zp = f.T
    # Cartesian -Hessian from the cylindrical derivatives (Rf = -Phi_R, tq = -Phi_phi)
    PR, Pf = -Rf, -tq
    Kxx = -(c * c * R2 - 2 * c * s / R * Rp + s * s / R**2 * p2 + s * s / R * PR +
            2 * c * s / R**2 * Pf)
    Kxy = -(c * s * R2 + (c * c - s * s) / R * Rp - c * s / R**2 * p2 - c * s / R * PR -
            (c * c - s * s) / R**2 * Pf)
    Kyy = -(s * s * R2 + 2 * c * s / R * Rp + c * c / R**2 * p2 + c * c / R * PR -
            2 * c * s / R**2 * Pf)
    ref = [Kxx, Kxy, Kyy]
    if not planar:
        ref += [-(c * Rz - s / R * zp), -(s * Rz + c / R * zp), -z2]
    ref = np.stack(ref, 1)
    scale = np.abs(ref).max()
    assert np.abs(K[:, :ref.shape[1]] - ref).max() < 1e-12 * scale


@pytest.mark.parametrize("method", ["leapfrog", "rk4", "symplec4", "dopr54", "dop853"])
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["scf_axi+mn", "scf_nonaxi", "bar_growing+mw14"])
def test_engine_variational_vs_oracle(harness, name, planar, method):
    from helpers import unit_deviations

    pt, pa = TP.potential(name, planar)
    dim = 2 if planar else 3
    w = unit_deviations(c2r(ics(6, planar, seed=7), planar), dim)
    t = np.linspace(0.0, 2.0, 17)
    with oracle.phi_from_atan2():
        ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar,
                                                **tol(method))
    out, err, ns = harness.integrate(w, t, pt, pa, method, planar=planar, var=True,
                                     **tol(method))
    assert np.array_equal(err, eref) and np.array_equal(ns, nref)
    rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max()
    assert rel < 1e-10, rel


# ---- wrappers: DehnenSmooth, SolidBodyRotation, GaussianAmplitude ----------
@needs_ref
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.WRAPPED)
@pytest.mark.parametrize("method", ["leapfrog", "rk6", "symplec6", "dopr54", "dop853"])
def test_wrapped_orbits_bit_exact_vs_reference_build(name, planar, method):
    pt, pa, npot = TP.wrapped(name, planar)
    yo = ics(8, planar)
    t = np.linspace(0.0, 8.0, 41)
    a, ea, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, npot=npot, **tol(method))
    b, eb, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, npot=npot, impl="ref",
                                   **tol(method))
    np.testing.assert_array_equal(ea, eb)
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["smooth(bar)+mw14", "rotate(loghalo)+mw14",
                                  "kuzmin(plummer)+mw14", "corot(needle)+mw14"])
def test_wrapped_dxdv_bit_exact_vs_reference_build(name, planar):
    pt, pa, npot = TP.wrapped(name, planar)
    dim = 2 if planar else 3
    rng = np.random.default_rng(5)
    w = np.concatenate([rng.uniform(0.6, 1.2, (4, dim)), rng.normal(0, 0.2, (4, dim)),
                        rng.normal(0, 1, (4, 2 * dim))], 1)
    w[:, dim + 1] += 1.0
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4", "dop853"):
        a = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, npot=npot,
                                  **tol(method))[0]
        b = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, npot=npot, impl="ref",
                                  **tol(method))[0]
        np.testing.assert_array_equal(a, b)


def cyl_to_K(f, R, phi, planar):
    """Cartesian K = -grad grad Phi from the oracle's cylindrical forces and
    second derivatives (Rf = -Phi_R, tq = -Phi_phi)."""
    c, s = np.cos(phi), np.sin(phi)
    if planar:
        Rf, tq, R2, p2, Rp = f.T
    else:
        Rf, zf, tq, R2, z2, Rz, p2, Rp, zp = f.T
    PR, Pf = -Rf, -tq
    K = [-(c * c * R2 - 2 * c * s / R * Rp + s * s / R**2 * p2 + s * s / R * PR +
           2 * c * s / R**2 * Pf),
         -(c * s * R2 + (c * c - s * s) / R * Rp - c * s / R**2 * p2 - c * s / R * PR -
           (c * c - s * s) / R**2 * Pf),
         -(s * s * R2 + 2 * c * s / R * Rp + c * c / R**2 * p2 + c * c / R * PR -
           2 * c * s / R**2 * Pf)]
    if not planar:
        K += [-(c * Rz - s / R * zp), -(s * Rz + c / R * zp), -z2]
    return np.stack(K, 1)


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.WRAPPED)
def test_engine_wrapped_forces_and_tidal(harness, name, planar):
    """The engine's wrapper frames (records evaluated at the rotated point,
    rotated back and scaled) against the oracle's wrapped sums, at several
    times."""
    pt, pa, npot = TP.wrapped(name, planar)
    rng = np.random.default_rng(14)
    R = rng.uniform(0.3, 2.0, 120)
    z = np.zeros(120) if planar else rng.normal(0, 0.4, 120)
    phi = rng.uniform(0, 2 * np.pi, 120)
    for t in (0.2, 2.5, 7.0):
        f = oracle.forces(R, z, phi, pt, pa, planar=planar, t=t, npot=npot)
        tq = f[:, 1] if planar else f[:, 2]
        ax = np.cos(phi) * f[:, 0] - np.sin(phi) * tq / R
        ay = np.sin(phi) * f[:, 0] + np.cos(phi) * tq / R
        acc, K, _ = harness.forces(R * np.cos(phi), R * np.sin(phi), z, pt, pa, planar=planar,
                                   t=t, npot=npot)
        ref = np.stack([ax, ay] + ([] if planar else [f[:, 1]]), 1)
        assert np.abs(acc[:, :ref.shape[1]] - ref).max() < 1e-14 * np.abs(ref).max(), t
        Kref = cyl_to_K(f, R, phi, planar)
        assert np.abs(K[:, :Kref.shape[1]] - Kref).max() < 1e-12 * np.abs(Kref).max(), t


@pytest.mark.parametrize("method", ["leapfrog", "symplec4", "rk4", "dopr54", "dop853"])
@pytest.mark.parametrize("name", TP.WRAPPED)
def test_engine_wrapped_machines_vs_oracle(harness, name, method):
    pt, pa, npot = TP.wrapped(name)
    y0 = ics(24, False, seed=23)
    t = np.linspace(0.0, 8.0, 33)
    with oracle.phi_from_atan2():
        ref, _, nref, _ = oracle.integrate(y0, t, pt, pa, method, npot=npot, **tol(method))
    out, err, ns = harness.integrate(c2r(y0, False), t, pt, pa, method, npot=npot,
                                     **tol(method))
    assert not err.any()
    ref_r = np.stack([c2r(ref[:, j], False) for j in range(len(t))], 1)
    d = np.abs(out - ref_r).reshape(len(y0), -1).max(1)
    same = ns == nref
    kink = TP.crosses_bar_radius(ref) if "bar" in name and method == "dop853" else \
        np.zeros(len(ns), bool)
    assert same[~kink].all()
    strict = same & ~kink
    assert np.median(d[strict]) < 1e-12 and d[strict].max() < 1e-9, d[strict].max()
    assert (d < 1e-6).all()


def test_nested_wrappers_refused():
    import galpy_b200 as gb

    mt, ma = TP.mw14()
    inner = [1] + TP.loghalo_triaxial_args() + [1.0, 0.6, 0.3]  # a rotating halo
    pt = np.array(mt + [-1, -2, 0], np.int32)
    pa = np.array(ma + [1] + inner + [1.0, 0.5, 4.0, 1.0])  # ... smoothly grown
    with pytest.raises(gb.PotentialNotSupported):
        gb.compile_potential((pt, pa, len(mt) + 1))


# ---- planar disk perturbations: log spirals, elliptical / lopsided / cos(m phi) disks
def pert_kink(name, ref):
    """Orbits crossing a radius where the potential's second derivative
    jumps: CosmphiDisk's break radius rb = 0.6."""
    if not name.startswith("cosmphi"):
        return np.zeros(len(ref), bool)
    R = ref[..., 0]
    return (R.min(axis=1) < 0.6) & (R.max(axis=1) > 0.6)


@needs_ref
@pytest.mark.parametrize("name", TP.PLANAR_PERTURBATIONS)
@pytest.mark.parametrize("method", METHODS)
def test_perturbation_orbits_bit_exact_vs_reference_build(name, method):
    pt, pa = TP.planar_perturbation(name)
    yo = ics(8, True)
    t = np.linspace(0.0, 8.0, 41)
    a, ea, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=True, **tol(method))
    b, eb, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=True, impl="ref", **tol(method))
    np.testing.assert_array_equal(ea, eb)
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("name", TP.PLANAR_PERTURBATIONS)
def test_perturbation_dxdv_bit_exact_vs_reference_build(name):
    pt, pa = TP.planar_perturbation(name)
    rng = np.random.default_rng(5)
    w = np.concatenate([rng.uniform(0.6, 1.2, (4, 2)), rng.normal(0, 0.2, (4, 2)),
                        rng.normal(0, 1, (4, 4))], 1)
    w[:, 3] += 1.0
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4", "dop853"):
        a = oracle.integrate_dxdv(w, t, pt, pa, method, planar=True, **tol(method))[0]
        b = oracle.integrate_dxdv(w, t, pt, pa, method, planar=True, impl="ref",
                                  **tol(method))[0]
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", TP.PLANAR_PERTURBATIONS)
def test_engine_perturbation_forces_and_tidal(harness, name):
    pt, pa = TP.planar_perturbation(name)
    rng = np.random.default_rng(15)
    R, phi = rng.uniform(0.3, 2.0, 120), rng.uniform(0, 2 * np.pi, 120)
    z = np.zeros(120)
    for t in (0.2, 3.0, 7.0):
        f = oracle.forces(R, z, phi, pt, pa, planar=True, t=t)
        ax = np.cos(phi) * f[:, 0] - np.sin(phi) * f[:, 1] / R
        ay = np.sin(phi) * f[:, 0] + np.cos(phi) * f[:, 1] / R
        acc, K, _ = harness.forces(R * np.cos(phi), R * np.sin(phi), z, pt, pa, planar=True,
                                   t=t)
        ref = np.stack([ax, ay], 1)
        assert np.abs(acc[:, :2] - ref).max() < 1e-14 * np.abs(ref).max(), t
        Kref = cyl_to_K(f, R, phi, True)
        assert np.abs(K[:, :3] - Kref).max() < 1e-12 * np.abs(Kref).max(), t


@pytest.mark.parametrize("method", ["leapfrog", "symplec4", "rk4", "dopr54", "dop853"])
@pytest.mark.parametrize("name", TP.PLANAR_PERTURBATIONS)
def test_engine_perturbation_machines_vs_oracle(harness, name, method):
    pt, pa = TP.planar_perturbation(name)
    y0 = ics(24, True, seed=29)
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, _, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=True, **tol(method))
    out, err, ns = harness.integrate(c2r(y0, True), t, pt, pa, method, planar=True,
                                     **tol(method))
    assert not err.any()
    ref_r = np.stack([c2r(ref[:, j], True) for j in range(len(t))], 1)
    d = np.abs(out - ref_r).reshape(len(y0), -1).max(1)
    same = ns == nref
    kink = pert_kink(name, ref) if method == "dop853" else np.zeros(len(ns), bool)
    assert same[~kink].all()
    strict = same & ~kink
    assert np.median(d[strict]) < 1e-12 and d[strict].max() < 1e-9, d[strict].max()
    assert (d < 1e-6).all()


# ---- SpiralArmsPotential: the oracle differentiates its potential by dual numbers
@pytest.mark.parametrize("planar", [False, True])
def test_spiral_arms_layout_and_forces_vs_galpy_python(planar):
    """The argument layout galpy's integrators build, and the oracle's forces
    and second derivatives against galpy's Python SpiralArmsPotential (its
    hand-written derivatives), at two times."""
    P = galpy_or_skip()
    pot = P.SpiralArmsPotential(amp=0.8, N=4, alpha=np.deg2rad(12), r_ref=1.1, phi_ref=0.3,
                                Rs=0.4, H=0.1, omega=0.55, Cs=[8 / (3 * np.pi), 0.5,
                                                              8 / (15 * np.pi)])
    if planar:
        from galpy.orbit.integratePlanarOrbit import _parse_pot
        gp = P.toPlanarPotential(pot)
    else:
        from galpy.orbit.integrateFullOrbit import _parse_pot
        gp = pot
    _, pt, pa, _ = _parse_pot([gp])
    assert list(pt) == [27]
    _, ref_a = TP.spiral_arms("spiral3+mw14", planar)
    np.testing.assert_allclose(pa, ref_a[-len(pa):], rtol=1e-15, atol=0)
    rng = np.random.default_rng(4)
    R, phi = rng.uniform(0.3, 2.0, 50), rng.uniform(0, 2 * np.pi, 50)
    z = np.zeros(50) if planar else rng.normal(0, 0.3, 50)
    names = (["Rforce", "phitorque", "R2deriv", "phi2deriv", "Rphideriv"] if planar else
             ["Rforce", "zforce", "phitorque", "R2deriv", "z2deriv", "Rzderiv", "phi2deriv",
              "Rphideriv", "phizderiv"])
    for t in (0.0, 1.7):
        got = oracle.forces(R, z, phi, np.array([27], np.int32), np.asarray(pa), planar=planar,
                            t=t)
        for k, nm in enumerate(names):
            ref = np.array([getattr(gp, nm)(R[i], *([] if planar else [z[i]]), phi=phi[i], t=t,
                                            use_physical=False) for i in range(R.size)])
            assert np.abs(got[:, k] - ref).max() <= 5e-14 * np.abs(ref).max(), (nm, t)
    if not planar:
        pv = oracle.potential(R, z, phi, np.array([27], np.int32), np.asarray(pa))
        ref = np.array([pot(R[i], z[i], phi=phi[i], use_physical=False) for i in range(50)])
        assert np.abs(pv - ref).max() <= 1e-14 * np.abs(ref).max()


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.SPIRAL_ARMS)
@pytest.mark.parametrize("method", METHODS)
def test_spiral_orbits_vs_reference_build(name, planar, method):
    """The reference differentiates the spiral potential by hand, the oracle
    by dual numbers: orbits agree to each orbit's own one-ulp response."""
    from helpers import cyl_diff

    pt, pa = TP.spiral_arms(name, planar)
    yo = ics(8, planar)
    t = np.linspace(0.0, 8.0, 41)
    a, ea, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, **tol(method))
    b, eb, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, impl="ref",
                                   **tol(method))
    np.testing.assert_array_equal(ea, eb)
    u = TP.ulp_response(oracle, yo, t, pt, pa, method, planar, a, **tol(method))
    d = cyl_diff(a, b).max(axis=(1, 2))
    assert (d <= 30 * np.maximum(u, 1e-15)).all(), (d / np.maximum(u, 1e-15)).max()


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
def test_spiral_dxdv_vs_reference_build(planar):
    pt, pa = TP.spiral_arms("spiral3+mw14", planar)
    dim = 2 if planar else 3
    rng = np.random.default_rng(5)
    w = np.concatenate([rng.uniform(0.6, 1.2, (4, dim)), rng.normal(0, 0.2, (4, dim)),
                        rng.normal(0, 1, (4, 2 * dim))], 1)
    w[:, dim + 1] += 1.0
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4", "dop853"):
        a = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, **tol(method))[0]
        b = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, impl="ref",
                                  **tol(method))[0]
        assert np.abs(a - b).max() < 1e-9 * max(1.0, np.abs(a).max()), method


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.SPIRAL_ARMS)
def test_engine_spiral_forces_and_tidal(harness, name, planar):
    """The engine's spiral arms (second-order forward differentiation in
    Cartesian form) against the oracle's cylindrical derivatives."""
    pt, pa = TP.spiral_arms(name, planar)
    rng = np.random.default_rng(16)
    R = rng.uniform(0.3, 2.0, 120)
    z = np.zeros(120) if planar else rng.normal(0, 0.4, 120)
    phi = rng.uniform(0, 2 * np.pi, 120)
    for t in (0.0, 2.5, 7.0):
        f = oracle.forces(R, z, phi, pt, pa, planar=planar, t=t)
        tq = f[:, 1] if planar else f[:, 2]
        ax = np.cos(phi) * f[:, 0] - np.sin(phi) * tq / R
        ay = np.sin(phi) * f[:, 0] + np.cos(phi) * tq / R
        acc, K, _ = harness.forces(R * np.cos(phi), R * np.sin(phi), z, pt, pa, planar=planar,
                                   t=t)
        ref = np.stack([ax, ay] + ([] if planar else [f[:, 1]]), 1)
        assert np.abs(acc[:, :ref.shape[1]] - ref).max() < 1e-14 * np.abs(ref).max(), t
        Kref = cyl_to_K(f, R, phi, planar)
        assert np.abs(K[:, :Kref.shape[1]] - Kref).max() < 1e-12 * np.abs(Kref).max(), t


@pytest.mark.parametrize("method", ["leapfrog", "symplec4", "rk4", "dopr54", "dop853"])
@pytest.mark.parametrize("planar", [False, True])
def test_engine_spiral_machines_vs_oracle(harness, planar, method):
    pt, pa = TP.spiral_arms("spiral3+mw14", planar)
    y0 = ics(24, planar, seed=31)
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, _, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar, **tol(method))
    out, err, ns = harness.integrate(c2r(y0, planar), t, pt, pa, method, planar=planar,
                                     **tol(method))
    assert not err.any()
    ref_r = np.stack([c2r(ref[:, j], planar) for j in range(len(t))], 1)
    d = np.abs(out - ref_r).reshape(len(y0), -1).max(1)
    same = ns == nref
    assert same.mean() > 0.9
    assert np.median(d[same]) < 1e-12 and d[same].max() < 1e-9, d[same].max()
    assert (d < 1e-6).all()


def test_spiral_arms_term_limit():
    import galpy_b200 as gb

    mt, ma = TP.mw14()
    a = TP.spiral_arms_args(Cs=[1.0] * 7)
    with pytest.raises(gb.PotentialNotSupported):
        gb.compile_potential((np.array(mt + [27], np.int32), np.array(ma + a)))


# ---- SoftenedNeedleBarPotential: a rotating softened needle ------------------
@pytest.mark.parametrize("planar", [False, True])
def test_needle_bar_layout_and_forces_vs_galpy_python(planar):
    """galpy's argument layout, and the oracle's forces and second
    derivatives against galpy's Python SoftenedNeedleBarPotential, at two
    times."""
    P = galpy_or_skip()
    pot = P.SoftenedNeedleBarPotential(amp=0.08, a=0.4, b=0.1, c=0.2, pa=-0.3, omegab=1.5)
    if planar:
        from galpy.orbit.integratePlanarOrbit import _parse_pot
        gp = P.toPlanarPotential(pot)
    else:
        from galpy.orbit.integrateFullOrbit import _parse_pot
        gp = pot
    _, pt, pa, _ = _parse_pot([gp])
    assert list(pt) == [25]
    _, ref_a = TP.needle_bar("needle_thick+mw14", planar)
    np.testing.assert_allclose(pa, ref_a[-len(pa):], rtol=1e-15, atol=0)
    rng = np.random.default_rng(8)
    R, phi = rng.uniform(0.2, 2.0, 50), rng.uniform(0, 2 * np.pi, 50)
    z = np.zeros(50) if planar else rng.normal(0, 0.3, 50)
    names = (["Rforce", "phitorque", "R2deriv", "phi2deriv", "Rphideriv"] if planar else
             ["Rforce", "zforce", "phitorque", "R2deriv", "z2deriv", "Rzderiv", "phi2deriv",
              "Rphideriv", "phizderiv"])
    for t in (0.0, 1.3):
        got = oracle.forces(R, z, phi, np.array([25], np.int32), np.asarray(pa), planar=planar,
                            t=t)
        for k, nm in enumerate(names):
            ref = np.array([getattr(gp, nm)(R[i], *([] if planar else [z[i]]), phi=phi[i], t=t,
                                            use_physical=False) for i in range(R.size)])
            assert np.abs(got[:, k] - ref).max() <= 1e-12 * np.abs(ref).max(), (nm, t)
    if not planar:
        pv = oracle.potential(R, z, phi, np.array([25], np.int32), np.asarray(pa))
        ref = np.array([pot(R[i], z[i], phi=phi[i], use_physical=False) for i in range(50)])
        assert np.abs(pv - ref).max() <= 1e-14 * np.abs(ref).max()


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.NEEDLE_BARS)
@pytest.mark.parametrize("method", METHODS)
def test_needle_orbits_bit_exact_vs_reference_build(name, planar, method):
    pt, pa = TP.needle_bar(name, planar)
    yo = ics(8, planar)
    t = np.linspace(0.0, 8.0, 41)
    a, ea, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, **tol(method))
    b, eb, _, _ = oracle.integrate(yo, t, pt, pa, method, planar=planar, impl="ref",
                                   **tol(method))
    np.testing.assert_array_equal(ea, eb)
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("planar", [False, True])
def test_needle_dxdv_bit_exact_vs_reference_build(planar):
    pt, pa = TP.needle_bar("needle_thick+mw14", planar)
    dim = 2 if planar else 3
    rng = np.random.default_rng(5)
    w = np.concatenate([rng.uniform(0.6, 1.2, (4, dim)), rng.normal(0, 0.2, (4, dim)),
                        rng.normal(0, 1, (4, 2 * dim))], 1)
    w[:, dim + 1] += 1.0
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4", "dop853"):
        a = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, **tol(method))[0]
        b = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar, impl="ref",
                                  **tol(method))[0]
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.NEEDLE_BARS)
def test_engine_needle_forces_and_tidal(harness, name, planar):
    """The engine's needle bar (bar-frame Cartesian gradient and Hessian in
    cancellation-free forms, rotated back) against the oracle."""
    pt, pa = TP.needle_bar(name, planar)
    rng = np.random.default_rng(18)
    R = rng.uniform(0.2, 2.0, 120)
    z = np.zeros(120) if planar else rng.normal(0, 0.4, 120)
    phi = rng.uniform(0, 2 * np.pi, 120)
    for t in (0.0, 2.5, 7.0):
        f = oracle.forces(R, z, phi, pt, pa, planar=planar, t=t)
        tq = f[:, 1] if planar else f[:, 2]
        ax = np.cos(phi) * f[:, 0] - np.sin(phi) * tq / R
        ay = np.sin(phi) * f[:, 0] + np.cos(phi) * tq / R
        acc, K, _ = harness.forces(R * np.cos(phi), R * np.sin(phi), z, pt, pa, planar=planar,
                                   t=t)
        ref = np.stack([ax, ay] + ([] if planar else [f[:, 1]]), 1)
        assert np.abs(acc[:, :ref.shape[1]] - ref).max() < 1e-14 * np.abs(ref).max(), t
        Kref = cyl_to_K(f, R, phi, planar)
        assert np.abs(K[:, :Kref.shape[1]] - Kref).max() < 1e-12 * np.abs(Kref).max(), t


@pytest.mark.parametrize("method", ["leapfrog", "symplec4", "rk4", "dopr54", "dop853"])
@pytest.mark.parametrize("planar", [False, True])
def test_engine_needle_machines_vs_oracle(harness, planar, method):
    pt, pa = TP.needle_bar("needle_thick+mw14", planar)
    y0 = ics(24, planar, seed=37)
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, _, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar, **tol(method))
    out, err, ns = harness.integrate(c2r(y0, planar), t, pt, pa, method, planar=planar,
                                     **tol(method))
    assert not err.any()
    ref_r = np.stack([c2r(ref[:, j], planar) for j in range(len(t))], 1)
    d = np.abs(out - ref_r).reshape(len(y0), -1).max(1)
    same = ns == nref
    assert same.mean() > 0.9
    assert np.median(d[same]) < 1e-12 and d[same].max() < 1e-9, d[same].max()
    assert (d < 1e-6).all()


def test_needle_bar_arguments_checked():
    """A needle of zero length is refused; an unsoftened one (b = c = 0,
    singular on the needle only, as in the reference) compiles."""
    import galpy_b200 as gb
    from galpy_b200 import _lib

    mt, ma = TP.mw14()
    pt = np.array(mt + [25], np.int32)
    with pytest.raises(_lib.CudaError, match="invalid potential arguments"):
        gb.compile_potential((pt, np.array(ma + TP.needle_bar_args(a=0.0))))
    gb.compile_potential((pt, np.array(ma + TP.needle_bar_args(b=0.0, c=0.0))))


@pytest.mark.parametrize("planar", [False, True])
def test_kuzmin_like_layout_and_forces_vs_galpy_python(planar):
    """galpy's layout of a KuzminLikeWrapperPotential around a Plummer
    sphere, and the oracle's forces, second derivatives and potential
    against galpy's Python wrapper."""
    P = galpy_or_skip()
    pot = P.KuzminLikeWrapperPotential(pot=P.PlummerPotential(amp=0.8, b=0.5), a=0.3,
                                       b=np.sqrt(0.4))
    if planar:
        from galpy.orbit.integratePlanarOrbit import _parse_pot
        gp = P.toPlanarPotential(pot)
    else:
        from galpy.orbit.integrateFullOrbit import _parse_pot
        gp = pot
    npot, pt, pa, _ = _parse_pot([gp])
    assert npot == 1 and list(pt) == [-10, 17]
    np.testing.assert_allclose(pa, [1, 0.8, 0.5, 1.0, 0.3, 0.4], rtol=1e-15)
    rng = np.random.default_rng(10)
    R, phi = rng.uniform(0.1, 2.0, 40), rng.uniform(0, 2 * np.pi, 40)
    z = np.zeros(40) if planar else rng.normal(0, 0.4, 40)
    names = (["Rforce", "phitorque", "R2deriv"] if planar else
             ["Rforce", "zforce", "phitorque", "R2deriv", "z2deriv", "Rzderiv"])
    cols = [0, 1, 2] if planar else [0, 1, 2, 3, 4, 5]
    got = oracle.forces(R, z, phi, pt, np.asarray(pa), planar=planar, npot=1)
    for k, nm in zip(cols, names):
        ref = np.array([getattr(gp, nm)(R[i], *([] if planar else [z[i]]), phi=phi[i],
                                        use_physical=False) for i in range(R.size)])
        assert np.abs(got[:, k] - ref).max() <= 1e-13 * max(np.abs(ref).max(), 1e-300), nm
    if not planar:
        pv = oracle.potential(R, z, phi, pt, np.asarray(pa), npot=1)
        ref = np.array([pot(R[i], z[i], phi=phi[i], use_physical=False) for i in range(40)])
        assert np.abs(pv - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("planar", [False, True])
def test_corotating_rotation_layout_and_forces_vs_galpy_python(planar):
    """galpy's layout of a CorotatingRotationWrapperPotential around a
    triaxial halo, and the oracle's forces and second derivatives against
    galpy's Python wrapper, at two times."""
    P = galpy_or_skip()
    halo = P.LogarithmicHaloPotential(amp=0.5, q=0.9, core=0.1, b=0.8)
    pot = P.CorotatingRotationWrapperPotential(pot=halo, vpo=0.7, beta=0.8, pa=0.2, to=0.5)
    if planar:
        from galpy.orbit.integratePlanarOrbit import _parse_pot
        gp = P.toPlanarPotential(pot)
    else:
        from galpy.orbit.integrateFullOrbit import _parse_pot
        gp = pot
    npot, pt, pa, _ = _parse_pot([gp])
    assert npot == 1 and list(pt) == [-4, 0]
    np.testing.assert_allclose(pa[-5:], [1.0, 0.7, 0.8, 0.2, 0.5], rtol=1e-15)
    rng = np.random.default_rng(13)
    R, phi = rng.uniform(0.3, 2.0, 40), rng.uniform(0, 2 * np.pi, 40)
    z = np.zeros(40) if planar else rng.normal(0, 0.4, 40)
    names = (["Rforce", "phitorque", "R2deriv", "phi2deriv", "Rphideriv"] if planar else
             ["Rforce", "zforce", "phitorque", "R2deriv", "z2deriv", "Rzderiv", "phi2deriv",
              "Rphideriv", "phizderiv"])
    for t in (0.0, 2.3):
        got = oracle.forces(R, z, phi, pt, np.asarray(pa), planar=planar, t=t, npot=1)
        for k, nm in enumerate(names):
            ref = np.array([getattr(gp, nm)(R[i], *([] if planar else [z[i]]), phi=phi[i],
                                            t=t, use_physical=False) for i in range(R.size)])
            assert np.abs(got[:, k] - ref).max() <= 1e-12 * np.abs(ref).max(), (nm, t)
