"""The CUDA engine in the time-dependent DehnenBarPotential and the
SCFPotential against the oracle (bit-exact with the reference's C for these
potentials: tests/test_timedep.py), through galpy's C-ABI entry points.

Force times follow the reference steppers' bookkeeping, so the engine takes
the reference's step sizes; its force is Cartesian (the bar as a quadratic
form, the SCF sums by recurrences), so results differ by the force's
rounding, which each orbit amplifies by its own conditioning: the bound per
orbit is the oracle's response to a one-ulp change of its initial
conditions (times 30, the larger of two such responses), never looser
than 1e-10.  DOP853 orbits that cross the bar radius (a jump of the
potential's second derivative) may flip accept / reject decisions at that
rounding level; they agree to the tolerance's scale instead.  The random
non-axisymmetric SCF expansion makes many orbits chaotic (the oracle's own
orbits move by O(1) at t = 10 under a one-ulp change of their initial
conditions), so it is compared over t <= 3."""
import numpy as np
import pytest
from helpers import cyl_diff, cyl_to_rect, sos_diff, unit_deviations

import galpy_b200 as gb
import timedep_pots as TP
from galpy_b200 import _lib

pytestmark = pytest.mark.gpu
METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "GPU tests need a GPU"


def ics(n, planar, seed):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.5, 1.5, n)
    vR, vT, phi = rng.normal(0, 0.1, n), rng.uniform(0.8, 1.1, n), rng.uniform(0, 2 * np.pi, n)
    if planar:
        return np.stack([R, vR, vT, phi], 1)
    return np.stack([R, vR, vT, rng.normal(0, 0.1, n), rng.normal(0, 0.1, n), phi], 1)


def tol(method):
    return dict(rtol=1e-10, atol=1e-10) if method in ("dopr54", "dop853") else {}


T_END = {"scf_nonaxi": 3.0}  # chaotic orbits: a short window


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.NAMES)
def test_orbits_vs_oracle(oracle, name, planar, method):
    pt, pa = TP.potential(name, planar)
    y0 = ics(128, planar, 17 + TP.NAMES.index(name))
    t = np.linspace(0.0, T_END.get(name, 10.0), 41)
    with oracle.phi_from_atan2():
        ref, eref, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar, **tol(method))
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    out, err, ns = fn((pt, pa), y0.copy(), t, method + "_cuda", progressbar=False,
                      return_nsteps=True, **tol(method))
    assert not err.any() and not eref.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    same = ns == nref
    kink = TP.crosses_bar_radius(ref) if name.startswith("bar") and method == "dop853" else \
        np.zeros(len(ns), bool)
    assert same[~kink].mean() >= 0.99, same[~kink].mean()
    far = same & ~kink & (d > 1e-10)
    if far.any():
        with oracle.phi_from_atan2():
            resp = np.maximum(*[TP.ulp_response(oracle, y0[far], t, pt, pa, method, planar,
                                                ref[far], seed=sd, **tol(method))
                                for sd in (3, 4)])
        assert (d[far] <= 30 * resp).all(), (d[far], resp)
    assert (d[~same | kink] < 1e-6).all(), d[~same | kink]


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
def test_variational_in_growing_bar(oracle, method, planar):
    pt, pa = TP.potential("bar_growing+mw14", planar)
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(ics(6, planar, 5)), dim)
    t = np.linspace(0.0, 6.0, 25)
    with oracle.phi_from_atan2():
        ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar,
                                                **tol(method))
    out, err, ns = gb.integrate_dxdv_batch((pt, pa), w, t, method + "_cuda", planar=planar,
                                           return_nsteps=True, **tol(method))
    # err 1: dopr54's forced smallest step, flagged by the reference too
    assert np.array_equal(err, eref)
    r = np.sqrt((ref[..., :dim] ** 2).sum(-1))
    kink = (r.min(axis=1) < 0.8) & (r.max(axis=1) > 0.8) if method == "dop853" else \
        np.zeros(len(ns), bool)
    assert np.array_equal(ns[~kink], nref[~kink])
    rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max(axis=(1, 2))
    assert rel[~kink].max() < 1e-9 and (rel[kink] < 1e-5).all(), rel


@pytest.mark.parametrize("method", ["leapfrog", "rk4", "symplec4", "dop853"])
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["scf_axi+mn", "scf_nonaxi"])
def test_variational_in_scf(oracle, name, method, planar):
    """The SCF expansion's tidal tensor (second derivatives by the
    recurrences, the reference's spherical-to-cylindrical chain rule, then
    Cartesian) drives the deviations like the reference's."""
    pt, pa = TP.potential(name, planar)
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(ics(6, planar, 7)), dim)
    t = np.linspace(0.0, 2.0, 17)
    with oracle.phi_from_atan2():
        ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar,
                                                **tol(method))
    out, err, ns = gb.integrate_dxdv_batch((pt, pa), w, t, method + "_cuda", planar=planar,
                                           return_nsteps=True, **tol(method))
    assert np.array_equal(err, eref) and np.array_equal(ns, nref)
    rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max()
    assert rel < 1e-9, rel


@pytest.mark.parametrize("method", ["rk4", "dop853"])
def test_surface_of_section_in_growing_bar(oracle, method):
    """The surface of section's force time is the integrated time in the
    state."""
    pt, pa = TP.potential("bar_growing+mw14")
    y0 = ics(64, False, 9)
    yo = np.concatenate([y0, np.full((64, 1), 0.5)], 1)
    psi = np.linspace(0.0, 6 * np.pi, 13)
    with oracle.phi_from_atan2():
        ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-10, atol=1e-10)
    out, err, ns = gb.integrateFullOrbit_sos_cuda((pt, pa), y0, psi, 0.5, method + "_cuda",
                                                  rtol=1e-10, atol=1e-10, progressbar=False,
                                                  return_nsteps=True)
    assert not err.any()
    same = ns == nref
    assert same.mean() >= 0.8, same.mean()
    d = sos_diff(ref, out).max(axis=(1, 2))
    assert np.median(d) < 1e-10 and d.max() < 1e-6, (np.median(d), d.max())


def test_device_forces_and_potential(oracle):
    """Accelerations of the device kernel (galpy_cuda_accel_device) and SCF
    potential values (galpy_cuda_energy_device) against the oracle."""
    import torch

    rng = np.random.default_rng(4)
    R, z, phi = rng.uniform(0.2, 2.0, 500), rng.normal(0, 0.4, 500), rng.uniform(0, 6.28, 500)
    for name in ["scf_nonaxi", "scf_axi+mn"]:
        pt, pa = TP.potential(name)
        comps, nrec = gb.compile_potential((pt, pa))
        dev = torch.device("cuda", 0)
        pos = torch.tensor(np.stack([R * np.cos(phi), R * np.sin(phi), z]), device=dev)
        acc = torch.empty_like(pos)
        gb.accel_device(torch.from_numpy(comps).to(dev), nrec, pos, acc)
        f = oracle.forces(R, z, phi, pt, pa)
        ax = np.cos(phi) * f[:, 0] - np.sin(phi) * f[:, 2] / R
        ay = np.sin(phi) * f[:, 0] + np.cos(phi) * f[:, 2] / R
        a = acc.cpu().numpy()
        scale = np.abs(np.stack([ax, ay, f[:, 1]])).max()
        assert np.abs(a - np.stack([ax, ay, f[:, 1]])).max() < 1e-13 * scale, name
        # potential: the energy at rest
        w = torch.zeros((6, R.size), dtype=torch.float64, device=dev)
        w[:3] = pos
        E = torch.empty(R.size, dtype=torch.float64, device=dev)
        gb.energy_device(torch.from_numpy(comps).to(dev), nrec, w, E)
        ref = oracle.potential(R, z, phi, pt, pa)
        assert np.abs(E.cpu().numpy() - ref).max() < 1e-13 * np.abs(ref).max(), name


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.WRAPPED)
def test_wrapped_orbits_vs_oracle(oracle, name, planar, method):
    """Wrappers (DehnenSmooth, SolidBodyRotation, GaussianAmplitude) around
    a bar or a triaxial halo, next to MWPotential2014, through galpy's entry
    points with galpy's (pot_type, pot_args, npot)."""
    pt, pa, npot = TP.wrapped(name, planar)
    y0 = ics(128, planar, 31 + TP.WRAPPED.index(name))
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, eref, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar, npot=npot,
                                              **tol(method))
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    out, err, ns = fn((pt, pa, npot), y0.copy(), t, method + "_cuda", progressbar=False,
                      return_nsteps=True, **tol(method))
    assert not err.any() and not eref.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    same = ns == nref
    kink = TP.crosses_bar_radius(ref) if "bar" in name and method == "dop853" else \
        np.zeros(len(ns), bool)
    # the growth factors' third derivatives jump at tform and tsteady too, and
    # the 41 sampled rows can miss a brief crossing of the bar radius: a few
    # DOP853 flips beyond the detected crossings
    floor = 0.97 if "bar" in name and method == "dop853" else 0.99
    assert same[~kink].mean() >= floor, same[~kink].mean()
    far = same & ~kink & (d > 1e-10)
    if far.any():
        with oracle.phi_from_atan2():
            resp = np.maximum(*[TP.ulp_response(oracle, y0[far], t, pt, pa, method, planar,
                                                ref[far], seed=sd, npot=npot, **tol(method))
                                for sd in (3, 4)])
        assert (d[far] <= 30 * resp).all(), (d[far], resp)
    assert (d[~same | kink] < 1e-6).all(), d[~same | kink]


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", ["smooth(bar)+mw14", "rotate(loghalo)+mw14",
                                  "kuzmin(plummer)+mw14", "corot(needle)+mw14"])
def test_wrapped_variational(oracle, name, planar):
    pt, pa, npot = TP.wrapped(name, planar)
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(ics(6, planar, 5)), dim)
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4"):
        with oracle.phi_from_atan2():
            ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar,
                                                    npot=npot)
        out, err, ns = gb.integrate_dxdv_batch((pt, pa, npot), w, t, method + "_cuda",
                                               planar=planar, return_nsteps=True)
        assert np.array_equal(err, eref) and np.array_equal(ns, nref)
        rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max()
        assert rel < 1e-9, (method, rel)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("name", TP.PLANAR_PERTURBATIONS)
def test_planar_perturbation_orbits_vs_oracle(oracle, name, method):
    """galpy's planar disk perturbations (log spirals, elliptical, lopsided
    and cos(m phi) disks) over MWPotential2014 in the plane.  CosmphiDisk's
    second derivative jumps at its break radius rb = 0.6: DOP853 orbits
    crossing it may flip decisions at the rounding level."""
    pt, pa = TP.planar_perturbation(name)
    y0 = ics(128, True, 41 + TP.PLANAR_PERTURBATIONS.index(name))
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, eref, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=True, **tol(method))
    out, err, ns = gb.integratePlanarOrbit_cuda((pt, pa), y0.copy(), t, method + "_cuda",
                                                progressbar=False, return_nsteps=True,
                                                **tol(method))
    assert not err.any() and not eref.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    same = ns == nref
    R = ref[..., 0]
    kink = ((R.min(axis=1) < 0.6) & (R.max(axis=1) > 0.6)) if (
        name.startswith("cosmphi") and method == "dop853") else np.zeros(len(ns), bool)
    assert same[~kink].mean() >= 0.98, same[~kink].mean()
    far = same & ~kink & (d > 1e-10)
    if far.any():
        with oracle.phi_from_atan2():
            resp = np.maximum(*[TP.ulp_response(oracle, y0[far], t, pt, pa, method, True,
                                                ref[far], seed=sd, **tol(method))
                                for sd in (3, 4)])
        assert (d[far] <= 30 * resp).all(), (d[far], resp)
    assert (d[~same | kink] < 1e-6).all(), d[~same | kink]


@pytest.mark.parametrize("name", TP.PLANAR_PERTURBATIONS)
def test_planar_perturbation_variational(oracle, name):
    pt, pa = TP.planar_perturbation(name)
    w = unit_deviations(cyl_to_rect(ics(6, True, 5)), 2)
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4"):
        with oracle.phi_from_atan2():
            ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=True)
        out, err, ns = gb.integrate_dxdv_batch((pt, pa), w, t, method + "_cuda", planar=True,
                                               return_nsteps=True)
        assert np.array_equal(err, eref) and np.array_equal(ns, nref)
        rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max()
        assert rel < 1e-9, (method, rel)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.SPIRAL_ARMS)
def test_spiral_arms_orbits_vs_oracle(oracle, name, planar, method):
    """SpiralArmsPotential (one rotating term, or four arms with three
    terms) over MWPotential2014.  The potential is smooth: every orbit takes
    the oracle's steps."""
    pt, pa = TP.spiral_arms(name, planar)
    y0 = ics(128, planar, 51 + TP.SPIRAL_ARMS.index(name))
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, eref, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar,
                                              **tol(method))
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    out, err, ns = fn((pt, pa), y0.copy(), t, method + "_cuda", progressbar=False,
                      return_nsteps=True, **tol(method))
    assert not err.any() and not eref.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    same = ns == nref
    assert same.mean() >= 0.98, same.mean()
    far = same & (d > 1e-10)
    if far.any():
        with oracle.phi_from_atan2():
            resp = np.maximum(*[TP.ulp_response(oracle, y0[far], t, pt, pa, method, planar,
                                                ref[far], seed=sd, **tol(method))
                                for sd in (3, 4)])
        assert (d[far] <= 30 * resp).all(), (d[far], resp)
    assert (d[~same] < 1e-6).all(), d[~same]


@pytest.mark.parametrize("planar", [False, True])
def test_spiral_arms_variational(oracle, planar):
    pt, pa = TP.spiral_arms("spiral3+mw14", planar)
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(ics(6, planar, 5)), dim)
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4"):
        with oracle.phi_from_atan2():
            ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar)
        out, err, ns = gb.integrate_dxdv_batch((pt, pa), w, t, method + "_cuda",
                                               planar=planar, return_nsteps=True)
        assert np.array_equal(err, eref) and np.array_equal(ns, nref)
        rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max()
        assert rel < 1e-9, (method, rel)


def test_spiral_arms_device_forces_and_potential(oracle):
    """Accelerations (at t = 0, the device force entry's time) and potential
    values of the spiral arms on the device against the oracle."""
    import torch

    rng = np.random.default_rng(6)
    R, z, phi = rng.uniform(0.2, 2.0, 500), rng.normal(0, 0.4, 500), rng.uniform(0, 6.28, 500)
    pt, pa = TP.spiral_arms("spiral3+mw14")
    comps, nrec = gb.compile_potential((pt, pa))
    dev = torch.device("cuda", 0)
    pos = torch.tensor(np.stack([R * np.cos(phi), R * np.sin(phi), z]), device=dev)
    acc = torch.empty_like(pos)
    gb.accel_device(torch.from_numpy(comps).to(dev), nrec, pos, acc)
    f = oracle.forces(R, z, phi, pt, pa)
    ref = np.stack([np.cos(phi) * f[:, 0] - np.sin(phi) * f[:, 2] / R,
                    np.sin(phi) * f[:, 0] + np.cos(phi) * f[:, 2] / R, f[:, 1]])
    assert np.abs(acc.cpu().numpy() - ref).max() < 1e-13 * np.abs(ref).max()
    w = torch.zeros((6, R.size), dtype=torch.float64, device=dev)
    w[:3] = pos
    E = torch.empty(R.size, dtype=torch.float64, device=dev)
    gb.energy_device(torch.from_numpy(comps).to(dev), nrec, w, E)
    pv = oracle.potential(R, z, phi, pt, pa)
    assert np.abs(E.cpu().numpy() - pv).max() < 1e-13 * np.abs(pv).max()


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("name", TP.NEEDLE_BARS)
def test_needle_bar_orbits_vs_oracle(oracle, name, planar, method):
    """A rotating softened needle bar (galpy's default shape, and a thick
    one) over MWPotential2014: a smooth potential, every orbit takes the
    oracle's steps."""
    pt, pa = TP.needle_bar(name, planar)
    y0 = ics(128, planar, 61 + TP.NEEDLE_BARS.index(name))
    t = np.linspace(0.0, 10.0, 41)
    with oracle.phi_from_atan2():
        ref, eref, nref, _ = oracle.integrate(y0, t, pt, pa, method, planar=planar,
                                              **tol(method))
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    out, err, ns = fn((pt, pa), y0.copy(), t, method + "_cuda", progressbar=False,
                      return_nsteps=True, **tol(method))
    assert not err.any() and not eref.any()
    d = cyl_diff(ref, out).max(axis=(1, 2))
    same = ns == nref
    assert same.mean() >= 0.98, same.mean()
    far = same & (d > 1e-10)
    if far.any():
        with oracle.phi_from_atan2():
            resp = np.maximum(*[TP.ulp_response(oracle, y0[far], t, pt, pa, method, planar,
                                                ref[far], seed=sd, **tol(method))
                                for sd in (3, 4)])
        assert (d[far] <= 30 * resp).all(), (d[far], resp)
    assert (d[~same] < 1e-6).all(), d[~same]


@pytest.mark.parametrize("planar", [False, True])
def test_needle_bar_variational(oracle, planar):
    pt, pa = TP.needle_bar("needle_thick+mw14", planar)
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(ics(6, planar, 5)), dim)
    t = np.linspace(0.0, 4.0, 17)
    for method in ("rk4", "symplec4"):
        with oracle.phi_from_atan2():
            ref, eref, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar)
        out, err, ns = gb.integrate_dxdv_batch((pt, pa), w, t, method + "_cuda",
                                               planar=planar, return_nsteps=True)
        assert np.array_equal(err, eref) and np.array_equal(ns, nref)
        rel = (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max()
        assert rel < 1e-9, (method, rel)


def test_needle_bar_device_forces_and_potential(oracle):
    import torch

    rng = np.random.default_rng(9)
    R, z, phi = rng.uniform(0.2, 2.0, 500), rng.normal(0, 0.4, 500), rng.uniform(0, 6.28, 500)
    pt, pa = TP.needle_bar("needle_thick+mw14")
    comps, nrec = gb.compile_potential((pt, pa))
    dev = torch.device("cuda", 0)
    pos = torch.tensor(np.stack([R * np.cos(phi), R * np.sin(phi), z]), device=dev)
    acc = torch.empty_like(pos)
    gb.accel_device(torch.from_numpy(comps).to(dev), nrec, pos, acc)
    f = oracle.forces(R, z, phi, pt, pa)
    ref = np.stack([np.cos(phi) * f[:, 0] - np.sin(phi) * f[:, 2] / R,
                    np.sin(phi) * f[:, 0] + np.cos(phi) * f[:, 2] / R, f[:, 1]])
    assert np.abs(acc.cpu().numpy() - ref).max() < 1e-13 * np.abs(ref).max()
    w = torch.zeros((6, R.size), dtype=torch.float64, device=dev)
    w[:3] = pos
    E = torch.empty(R.size, dtype=torch.float64, device=dev)
    gb.energy_device(torch.from_numpy(comps).to(dev), nrec, w, E)
    pv = oracle.potential(R, z, phi, pt, pa)
    assert np.abs(E.cpu().numpy() - pv).max() < 1e-13 * np.abs(pv).max()


def test_kuzmin_like_device_forces_and_potential(oracle):
    """KuzminLike frames on the device: accelerations and potential values
    (the wrapped list at (xi, 0, 0)) against the oracle."""
    import torch

    rng = np.random.default_rng(12)
    R, z, phi = rng.uniform(0.1, 2.0, 500), rng.normal(0, 0.4, 500), rng.uniform(0, 6.28, 500)
    pt, pa, npot = TP.wrapped("kuzmin(hernquist,plummer)")
    comps, nrec = gb.compile_potential((pt, pa, npot))
    dev = torch.device("cuda", 0)
    pos = torch.tensor(np.stack([R * np.cos(phi), R * np.sin(phi), z]), device=dev)
    acc = torch.empty_like(pos)
    gb.accel_device(torch.from_numpy(comps).to(dev), nrec, pos, acc)
    f = oracle.forces(R, z, phi, pt, pa, npot=npot)
    ref = np.stack([np.cos(phi) * f[:, 0], np.sin(phi) * f[:, 0], f[:, 1]])
    assert np.abs(acc.cpu().numpy() - ref).max() < 1e-13 * np.abs(ref).max()
    w = torch.zeros((6, R.size), dtype=torch.float64, device=dev)
    w[:3] = pos
    E = torch.empty(R.size, dtype=torch.float64, device=dev)
    gb.energy_device(torch.from_numpy(comps).to(dev), nrec, w, E)
    pv = oracle.potential(R, z, phi, pt, pa, npot=npot)
    assert np.abs(E.cpu().numpy() - pv).max() < 1e-13 * np.abs(pv).max()
