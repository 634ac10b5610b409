"""The engine's device code (galpy_b200/csrc: force library + per-orbit
stepper state machines), compiled as host C++ by the test-only harness,
against the CPU oracle.  This checks the kernel logic on every CPU-only run;
tests/test_gpu_parity.py checks the compiled kernels on the GPU."""
import numpy as np
import pytest
from helpers import ADDED_POTS, KINKED, cyl_diff, cyl_to_sos, golden_pot, polar_to_sos, sos_diff, sos_to_cyl, sos_to_polar, cyl_to_rect, rect_to_cyl, seeded_ics, unit_deviations

METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]
POTS = ["mw14", "hernquist", "loghalo", "logtri", "nfw", "mn", "pswc"] + ADDED_POTS


@pytest.mark.parametrize("alpha", [0.5, 1.2, 1.8, 2.6])
def test_gamma_star_table_vs_mpmath(harness, alpha):
    """The bulge's Chebyshev table of gamma*(a, u) = P(a, u) / u^a against
    mpmath at 30 digits, a = 1.5 - alpha/2."""
    import ctypes

    import mpmath as mp

    mp.mp.dps = 30
    a = 1.5 - alpha / 2
    u = np.concatenate([[0.0, 1e-12], np.geomspace(1e-6, 45.0, 300), np.linspace(0.1, 44.9, 300)])
    out = np.zeros_like(u)
    dp = ctypes.POINTER(ctypes.c_double)
    assert harness.lib.harness_gamma_star(ctypes.c_double(alpha), ctypes.c_double(0.3), len(u),
                                          u.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    am = mp.mpf(a)
    ref = np.array([float(1 / mp.gamma(am + 1)) if x == 0 else
                    float(mp.gammainc(am, 0, mp.mpf(x), regularized=True) / mp.mpf(x) ** am)
                    for x in u])
    U = 20.0  # table cutoff, as in compile_potential.h (the kernel uses P = 1 beyond)
    while mp.e ** -U * U ** (a - 1) / mp.gamma(a) > 1e-18:
        U += 1.0
    sel = u < U
    assert (np.abs(out[sel] - ref[sel]) / ref[sel]).max() < 1e-15


@pytest.mark.parametrize("name", POTS)
def test_forces_and_tidal_tensor(harness, oracle, golden, name):
    pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
    R, z, phi = golden["pts_R"], golden["pts_z"], golden["pts_phi"]
    x, y = R * np.cos(phi), R * np.sin(phi)
    acc, K, a32 = harness.forces(x, y, z, pt, pa)
    if name == "null":
        assert not acc.any() and not K.any() and not a32.any()
        return
    f = oracle.forces(R, z, phi, pt, pa)
    Rf, zf, ptq, R2, z2, Rz, p2, Rp, zp = f.T
    c, s = x / R, y / R
    ref = np.stack([c * Rf - s / R * ptq, s * Rf + c / R * ptq, zf], 1)
    # NFW at r << a cancels two terms; the reference (log(1+x)) is the less
    # accurate side there (this code uses log1p).  Einasto: the reference
    # forms the enclosed-mass fraction as Q - 1, which loses ~eps / P digits
    # where P(3n, (r/h)^(1/n)) is small; this code evaluates P directly.
    tol = 1e-10 if name == "einasto" else 1e-12
    assert (np.abs(acc - ref).max(1) / np.abs(ref).max(1)).max() < tol
    Kxx = -c * c * R2 + 2 * c * s / R / R * ptq + s * s / R * Rf + 2 * s * c / R * Rp - s * s / R / R * p2
    Kxy = (-s * c * R2 + (s * s - c * c) / R / R * ptq - c * s / R * Rf - (c * c - s * s) / R * Rp
           + c * s / R / R * p2)
    Kyy = -s * s * R2 - 2 * s * c / R / R * ptq - 2 * s * c / R * Rp + c * c / R * Rf - c * c / R / R * p2
    Kref = np.stack([Kxx, Kxy, Kyy, -c * Rz + s / R * zp, -s * Rz - c / R * zp, -z2], 1)
    assert (np.abs(K - Kref).max(1) / np.abs(Kref).max(1)).max() < tol
    # float32 force evaluation: single-precision accuracy
    assert (np.abs(a32 - ref).max(1) / np.abs(ref).max(1)).max() < 3e-5


@pytest.mark.parametrize("name", POTS)
def test_potential_values(harness, oracle, golden, name):
    """The energy kernel's potential against the oracle (reference formulas)."""
    import ctypes

    pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
    R, z, phi = golden["pts_R"], golden["pts_z"], golden["pts_phi"]
    x, y = R * np.cos(phi), R * np.sin(phi)
    out = np.zeros_like(R)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    pti = np.ascontiguousarray(pt, np.int32)
    pad = np.ascontiguousarray(pa, np.float64)
    assert harness.lib.harness_potential(len(R), x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                         z.ctypes.data_as(dp), len(pti), pti.ctypes.data_as(ip),
                                         pad.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    ref = oracle.potential(R, z, phi, pt, pa)
    assert (np.abs(out - ref) / max(np.abs(ref).max(), 1e-300)).max() < 1e-13


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
def test_orbits_vs_oracle(harness, oracle, mw14, mw14_planar, method, planar):
    pt, pa = mw14_planar if planar else mw14
    ics = seeded_ics(24, 8, planar=planar)
    t = np.linspace(0, 20, 201)
    ref, eref, nref, _ = oracle.integrate(ics, t, pt, pa, method, planar=planar)
    out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, method, planar=planar)
    assert not err.any() and not eref.any()
    assert np.array_equal(ns, nref), "step sequence differs from the reference"
    assert cyl_diff(ref, rect_to_cyl(out)).max() < 1e-11


@pytest.mark.parametrize("name", ADDED_POTS)
def test_spherical_potential_orbits(harness, oracle, golden, name):
    """Orbits in each spherical potential: the same step sequence as the
    oracle and agreement to the orbits' conditioning, 3D, planar and
    variational."""
    pt, pa = golden_pot(golden, name)
    t = np.linspace(0, 8, 41)
    for planar, m in ((False, "dop853"), (False, "symplec6"), (True, "dopr54"), (True, "rk4")):
        pt, pa = golden_pot(golden, name, planar)
        ics = seeded_ics(8, 17, planar=planar)
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, m, planar=planar, rtol=1e-10,
                                           atol=1e-10)
        out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, m, planar=planar,
                                         rtol=1e-10, atol=1e-10)
        assert not err.any(), m
        d = cyl_diff(ref, rect_to_cyl(out)).max(axis=(1, 2))
        same = ns == nref
        if name in KINKED:
            # at the kink (jump) an adaptive step's accept / reject follows
            # rounding: each orbit is bounded by the oracle's own response to
            # a 1-ulp change of its initial conditions
            ulp = 1 + np.finfo(float).eps * np.random.default_rng(1).choice([-1, 1], ics.shape)
            pert, _, _, _ = oracle.integrate(ics * ulp, t, pt, pa, m, planar=planar,
                                             rtol=1e-10, atol=1e-10)
            bound = np.maximum(1e-10, 10 * cyl_diff(ref, pert).max(axis=(1, 2)))
            assert (d <= bound).all(), (m, same, d.max())
        else:
            assert same.all(), m
            assert d.max() < 1e-10, m
    pt, pa = golden_pot(golden, name)
    w = unit_deviations(cyl_to_rect(seeded_ics(2, 18)), 3)
    ref, _, nref = oracle.integrate_dxdv(w, t, pt, pa, "dop853")
    out, err, ns = harness.integrate(w, t, pt, pa, "dop853", var=True)
    assert not err.any()
    # scaled per orbit: inside the homogeneous sphere some deviation
    # components vanish exactly (the reference's formulas leave 1e-16 there)
    rel = (np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)).max(axis=(1, 2))
    assert rel[ns == nref].max(initial=0) < 1e-10 and rel.max() < 1e-6


def test_config0_symplec4_conditioning(harness, oracle, mw14):
    """t in [0,100], 1001 outputs: same step size per orbit, and differences
    at the level of the orbits' own sensitivity to 1e-16 perturbations."""
    pt, pa = mw14
    ics = seeded_ics(48, 0)
    t = np.linspace(0, 100, 1001)
    ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, "symplec4")
    out, _, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, "symplec4")
    assert np.array_equal(ns, nref)
    per_orbit = cyl_diff(ref, rect_to_cyl(out)).max(axis=(1, 2))
    assert np.median(per_orbit) < 1e-12
    assert per_orbit.max() < 1e-10


@pytest.mark.parametrize("name", ["hernquist", "loghalo", "logtri", "nfw", "mn", "pswc"]
                         + ADDED_POTS)
def test_planar_variational_added_potentials(harness, oracle, golden, name):
    """Planar variational runs (integratePlanarOrbit_dxdv) in each
    potential: the planar tidal tensor against the reference's planar second
    derivatives, restated in the oracle (for KuzminDisk that includes the
    reference's sign of PlanarR2deriv)."""
    pt, pa = golden_pot(golden, name, planar=True)
    if int(pt[0]) == 15:  # planar PowerSphericalwCutoff: (amp, alpha, rc)
        pa = np.asarray(pa, float)[:3]
    w = unit_deviations(cyl_to_rect(seeded_ics(2, 18, planar=True)), 2)
    t = np.linspace(0, 8, 41)
    for m in ("rk4",) if name in KINKED else ("rk4", "dop853"):
        ref, _, nref = oracle.integrate_dxdv(w, t, pt, pa, m, planar=True)
        out, err, ns = harness.integrate(w, t, pt, pa, m, planar=True, var=True)
        assert not err.any() and np.array_equal(ns, nref), m
        rel = np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)
        assert rel.max() < 1e-10, (m, rel.max())


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
def test_variational_vs_oracle(harness, oracle, mw14, mw14_planar, method, planar):
    pt, pa = mw14_planar if planar else mw14
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(seeded_ics(2, 9, planar=planar)), dim)
    t = np.linspace(0, 5, 51)
    ref, _, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar)
    out, err, ns = harness.integrate(w, t, pt, pa, method, planar=planar, var=True)
    assert not err.any()
    assert np.array_equal(ns, nref)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert (np.abs(out - ref) / scale).max() < 1e-10


@pytest.mark.parametrize("method", ["dop853", "dopr54"])
def test_adaptive_per_orbit_times(harness, oracle, golden, method):
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    ics = golden["c_ics"]
    out, err, _ = harness.integrate(cyl_to_rect(ics), golden["c_indiv_t"], pt, pa, method,
                                    rtol=1e-10, atol=1e-10)
    assert not err.any()
    assert cyl_diff(golden[f"c_{method}_indiv"], rect_to_cyl(out)).max() < 1e-10


def test_dopr54_forced_steps(harness, oracle, golden):
    """The smallest-step rule: err = 1 and 10,000 forced steps per orbit, as
    in the reference's own C (golden vectors)."""
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    out, err, ns = harness.integrate(cyl_to_rect(golden["c_ics"]), np.array([0.0, 50.0]), pt, pa,
                                     "dopr54", dt=50.0, rtol=1e-20, atol=1e-20)
    assert np.all(err == 1) and np.all(ns == 10000)
    assert cyl_diff(golden["c_dopr54_forced"], rect_to_cyl(out)).max() < 1e-11


def test_backward_integration(harness, oracle, mw14):
    pt, pa = mw14
    ics = seeded_ics(8, 12)
    t = np.linspace(0, -10, 101)
    for method in METHODS:
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, method)
        out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, method)
        assert np.array_equal(ns, nref)
        assert cyl_diff(ref, rect_to_cyl(out)).max() < 1e-11


def test_fixed_dt(harness, oracle, mw14):
    pt, pa = mw14
    ics = seeded_ics(8, 13)
    t = np.linspace(0, 10, 11)
    for method in ("leapfrog", "symplec4", "symplec6", "rk4", "rk6"):
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, method, dt=0.01)
        out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, method, dt=0.01)
        assert np.array_equal(ns, nref) and nref[0] == 1000
        assert cyl_diff(ref, rect_to_cyl(out)).max() < 1e-11
    # dopr54: dt is only its first step
    ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, "dopr54", dt=0.01)
    out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, "dopr54", dt=0.01)
    assert np.array_equal(ns, nref) and not err.any()
    assert cyl_diff(ref, rect_to_cyl(out)).max() < 1e-11


def test_attempt_budget_and_nonfinite(harness, mw14):
    pt, pa = mw14
    ics = seeded_ics(3, 14)
    t = np.linspace(0, 50, 51)
    for method in ("dop853", "dopr54"):
        out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, method, max_attempts=20)
        assert np.all(err == 2)
        assert np.isnan(out[:, -1]).all() and np.isfinite(out[:, 0]).all()
    w = cyl_to_rect(ics)
    w[1, 0] = np.nan
    for method in METHODS:
        out, err, ns = harness.integrate(w, t[:5], pt, pa, method, dt=0.01)
        assert err[1] == 3 and err[0] == 0 and err[2] == 0
        assert np.isnan(out[1, 1:]).all()


def test_dopr54_stalled_time_ends_the_orbit(harness, mw14):
    """Output times near 1e17 (ulp 16) and a first step of 1: the accepted
    step leaves the time unchanged, where the reference loops forever; the
    machine stops the orbit with err 2 after that one step."""
    pt, pa = mw14
    w = cyl_to_rect(seeded_ics(2, 16))
    t = 1e17 + np.array([0.0, 128.0, 256.0])
    out, err, ns = harness.integrate(w, t, pt, pa, "dopr54", dt=1.0)
    assert np.all(err == 2) and np.all(ns == 1)
    assert np.array_equal(out[:, 0], w) and np.isnan(out[:, 1:]).all()


def test_single_output_row(harness, mw14):
    pt, pa = mw14
    w = cyl_to_rect(seeded_ics(2, 15))
    out, err, ns = harness.integrate(w, np.array([0.0]), pt, pa, "dop853")
    assert np.array_equal(out[:, 0], w) and not err.any()


def test_binade_tables_match_mpmath(harness):
    """The FP64 force path's branch-free (r^2)^(-alpha/2) and log1p (binade
    tables built on the host) against 120-bit references."""
    import ctypes

    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 120
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(0)
    x = np.exp(rng.uniform(np.log(1e-10), np.log(1e8), 4000))
    for alpha in (1.8, 1.0, 2.5, 0.3):
        out = np.zeros_like(x)
        assert harness.lib.harness_binade(0, ctypes.c_double(alpha), len(x),
                                          x.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
        ref = np.array([float(mpmath.mpf(v) ** (-alpha / 2)) for v in x])
        assert np.abs(out / ref - 1).max() < 3 * 2.3e-16
    xs = np.concatenate([np.exp(rng.uniform(np.log(1e-12), np.log(1e6), 4000)),
                         np.linspace(0, 2, 201)])
    out = np.zeros_like(xs)
    assert harness.lib.harness_binade(1, ctypes.c_double(0), len(xs), xs.ctypes.data_as(dp),
                                      out.ctypes.data_as(dp)) == 0
    ref = np.array([float(mpmath.log1p(mpmath.mpf(v))) for v in xs])
    pos = ref > 0
    assert np.abs(out[pos] / ref[pos] - 1).max() < 3 * 2.3e-16
    assert out[xs == 0].tolist() == [0.0]
    xf = xs.astype(np.float32).astype(np.float64)
    assert harness.lib.harness_binade(2, ctypes.c_double(0), len(xf), xf.ctypes.data_as(dp),
                                      out.ctypes.data_as(dp)) == 0
    ref = np.array([float(mpmath.log1p(mpmath.mpf(v))) for v in xf])
    pos = ref > 0
    assert np.abs(out[pos] / ref[pos] - 1).max() < 4 * 6e-8


@pytest.mark.parametrize("method", ["rk4", "rk6", "dopr54", "dop853"])
def test_surface_of_section_machines(harness, oracle, golden, method):
    """The SOS system on the RK-type machines against the oracle: same step
    sequence, agreement well inside the tolerance."""
    for name in ("mw14", "logtri"):
        pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
        yo = np.concatenate([seeded_ics(8, 19), np.linspace(0, 2, 8)[:, None]], 1)
        psi = np.linspace(0.0, 12.0 * np.pi, 7)
        ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-10, atol=1e-10)
        raw, err, ns = harness.integrate_sos(cyl_to_sos(yo), psi, pt, pa, method, rtol=1e-10,
                                             atol=1e-10)
        assert not err.any() and np.array_equal(ns, nref), (name, ns, nref)
        assert sos_diff(ref, sos_to_cyl(raw)).max() < 1e-10, name


@pytest.mark.parametrize("surface", [0, 1])
@pytest.mark.parametrize("method", ["rk4", "rk6", "dopr54", "dop853"])
def test_planar_surface_of_section_machines(harness, oracle, golden, method, surface):
    pt, pa = golden["mw14_planar_type"], golden["mw14_planar_args"]
    yo = np.concatenate([seeded_ics(8, 20, planar=True), np.linspace(0, 2, 8)[:, None]], 1)
    psi = np.linspace(0.0, 12.0 * np.pi, 7)
    ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-10, atol=1e-10,
                                        planar=True, surface=surface)
    raw, err, ns = harness.integrate_sos(polar_to_sos(yo, surface), psi, pt, pa, method,
                                         rtol=1e-10, atol=1e-10, surface=surface)
    assert not err.any() and np.array_equal(ns, nref)
    got = sos_to_polar(raw, surface)
    d = np.abs(got - ref)
    d[..., 3] = np.abs((got[..., 3] - ref[..., 3] + np.pi) % (2 * np.pi) - np.pi)
    assert d.max() < 1e-10


@pytest.mark.parametrize("planar", [False, True])
def test_dop853_queued_dense_output(harness, oracle, golden, planar):
    """The kernels' queued dense output (request record written at the
    accepted step, dense stages run later from the record) gives the in-slot
    dense output's rows bit for bit: shared grids, ragged per-orbit grids
    with several outputs in one step, backward integration, a generic
    component list, and orbits stopped by the attempt budget."""
    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    ics = seeded_ics(24, 61, planar=planar, r_range=(0.05, 3.0), log_r=True)
    w = cyl_to_rect(ics)
    rng = np.random.default_rng(61)
    grids = [np.linspace(0, 20, 201), np.linspace(0, -15, 31),
             np.sort(rng.uniform(0, 1, (len(w), 41)), axis=1) * rng.uniform(2, 30, (len(w), 1))]
    grids[2][:, 0] = 0.0
    for t in grids:
        ref, eref, nref = harness.integrate(w, t, pt, pa, "dop853", planar=planar, rtol=1e-10,
                                            atol=1e-10)
        out, err, ns = harness.dop853_queued(w, t, pt, pa, planar=planar, rtol=1e-10, atol=1e-10)
        assert np.array_equal(err, eref) and np.array_equal(ns, nref)
        assert np.array_equal(out, ref)
    # a generic list (triaxial halo + Hernquist) and the attempt budget
    pt2 = np.concatenate([golden["logtri_type"], golden["hernquist_type"]])
    pa2 = np.concatenate([golden["logtri_args"], golden["hernquist_args"]])
    t = np.linspace(0, 50, 51)
    for ma in (0, 40):
        ref, eref, nref = harness.integrate(w, t, pt2, pa2, "dop853", planar=planar,
                                            max_attempts=ma)
        out, err, ns = harness.dop853_queued(w, t, pt2, pa2, planar=planar, max_attempts=ma)
        assert np.array_equal(err, eref) and np.array_equal(ns, nref)
        assert np.array_equal(out, ref, equal_nan=True)
    assert (eref == 2).all()  # the budget stops every orbit


@pytest.mark.parametrize("planar", [False, True])
def test_mixed_precision_forces(harness, golden, planar):
    """The mixed float64 / float32 MWPotential2014 forces against the
    float64 force over the radii the integrations visit (0.01 to 30, all
    polynomial intervals of the tables): the float32 tails of the table
    polynomials (F64_TAIL32) move the force by < 1e-11 relative; the float32
    bulge term (F32BULGE) by the single-precision log2 / exp2 of its power
    law, up to ~1e-6 of the total where the bulge dominates (r < 0.1)."""
    import ctypes

    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    rng = np.random.default_rng(17)
    n = 20000
    r = np.exp(rng.uniform(np.log(0.01), np.log(30.0), n))
    th = np.arccos(rng.uniform(-1, 1, n)) if not planar else np.full(n, np.pi / 2)
    ph = rng.uniform(0, 2 * np.pi, n)
    x, y, z = r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)
    ref, _, _ = harness.forces(x, y, z, pt, pa, planar=planar)
    pa_c = np.ascontiguousarray(pa, np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    for mix, tol in ((1, 1e-11), (2, 3e-6)):
        acc = np.zeros((n, 3))
        rc = harness.lib.harness_forces_mixed(
            mix, int(planar), n, np.ascontiguousarray(x).ctypes.data_as(dp),
            np.ascontiguousarray(y).ctypes.data_as(dp), np.ascontiguousarray(z).ctypes.data_as(dp),
            pa_c.ctypes.data_as(dp), acc.ctypes.data_as(dp))
        assert rc == 0
        rel = np.abs(acc - ref).max(axis=1) / np.abs(ref).max(axis=1)
        assert rel.max() < tol, (mix, rel.max())
        if mix == 1:
            assert rel.max() > 0  # the tails are in float32 indeed
