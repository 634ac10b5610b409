"""The EllipsoidalPotential family: TriaxialHernquist (21), TriaxialNFW (22),
TriaxialJaffe (23), PerfectEllipsoid (30), TriaxialGaussian (37),
PowerTriaxial (38) and TwoPowerTriaxial (43), aligned and rotated.

The force is a Gauss-Legendre integral over the ellipsoidal shells
(EllipsoidalPotential.c:38-76) with each member's density function.  Oracle:
the restatement pinned on galpy's Python forces, second derivatives (galpy
implements them for aligned potentials only) and values, and on the
reference's C orbits (golden vectors; bit for bit where the reference build
is present).  The reference's C second derivatives are evaluated in the
principal-axis form at the unrotated point (EllipsoidalPotential.c:414-421);
the engine's tidal tensor does the same, so variational runs of rotated
potentials follow the reference.  TwoPowerTriaxial's potential value needs
the Gauss hypergeometric function, which neither the oracle nor the engine
carries: it is NaN in both.
"""
import ctypes

import numpy as np
import pytest
from helpers import cyl_diff, cyl_to_rect, golden_pot, rect_to_cyl, seeded_ics

ELL = ["trihern", "trinfw", "trijaffe", "perfell", "trigauss", "powertri", "twopowtri"]
METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]


def _pot(golden, name, planar=False):
    return golden_pot(golden, f"ell_{name}", planar)


def _cart_K(f, x, y):
    """Cartesian tidal tensor (xx, xy, yy, xz, yz, zz) from the oracle's
    cylindrical forces and second derivatives."""
    R = np.hypot(x, y)
    Rf, zf, ptq, R2, z2, Rz, p2, Rp, zp = f.T
    c, s = x / R, y / R
    Kxx = -c * c * R2 + 2 * c * s / R / R * ptq + s * s / R * Rf + 2 * s * c / R * Rp - s * s / R / R * p2
    Kxy = (-s * c * R2 + (s * s - c * c) / R / R * ptq - c * s / R * Rf - (c * c - s * s) / R * Rp
           + c * s / R / R * p2)
    Kyy = -s * s * R2 - 2 * s * c / R / R * ptq - 2 * s * c / R * Rp + c * c / R * Rf - c * c / R / R * p2
    return np.stack([Kxx, Kxy, Kyy, -c * Rz + s / R * zp, -s * Rz - c / R * zp, -z2], 1)


@pytest.mark.parametrize("name", ELL)
def test_oracle_vs_galpy_python(oracle, golden, name):
    pt, pa = _pot(golden, name)
    R, z, phi = golden["pts_R"], golden["pts_z"], golden["pts_phi"]
    py = golden[f"ell_{name}_pyforces"]
    f = oracle.forces(R, z, phi, pt, pa)
    np.testing.assert_allclose(f[:, :3], py[:, :3], rtol=1e-12, atol=1e-14)
    hess = py[:, 3:9]
    ok = ~np.isnan(hess)
    aligned = name in ("trihern", "perfell", "trigauss", "twopowtri")
    assert ok.all() if aligned else not ok.any()
    if aligned:
        assert (np.abs(f[:, 3:9] - hess) / np.abs(hess).max()).max() < 1e-12
    v = oracle.potential(R, z, phi, pt, pa)
    if name == "twopowtri":
        assert np.isnan(v).all()
    else:
        np.testing.assert_allclose(v, py[:, 9], rtol=1e-12)


@pytest.mark.parametrize("name", ELL)
def test_oracle_golden_and_bitwise(oracle, golden, name):
    pt, pa = _pot(golden, name)
    pt2, pa2 = _pot(golden, name, planar=True)
    t = np.linspace(0, 5, 51)
    a, _, _, _ = oracle.integrate(golden["c_ics"], t, pt, pa, "dop853")
    np.testing.assert_allclose(a, golden[f"ell_{name}_3d"], rtol=0, atol=1e-13)
    a, _, _, _ = oracle.integrate(golden["c_ics_planar"], t, pt2, pa2, "symplec4", planar=True)
    np.testing.assert_allclose(a, golden[f"ell_{name}_planar"], rtol=0, atol=1e-13)
    a, _, _ = oracle.integrate_dxdv(golden["sph_dxdv_w3"], t, pt, pa, "dop853")
    np.testing.assert_allclose(a, golden[f"ell_{name}_dxdv3"], rtol=0, atol=1e-12)
    if not oracle.ref_available():
        return
    ics = seeded_ics(4, 7)
    ics2 = seeded_ics(4, 8, planar=True)
    t = np.linspace(0, 4, 21)
    for m in METHODS:
        a, ea, _, _ = oracle.integrate(ics, t, pt, pa, m, rtol=1e-9, atol=1e-9)
        b, eb, _, _ = oracle.integrate(ics, t, pt, pa, m, rtol=1e-9, atol=1e-9, impl="ref")
        assert np.array_equal(a, b) and np.array_equal(ea, eb), m
        a, _, _, _ = oracle.integrate(ics2, t, pt2, pa2, m, planar=True, rtol=1e-9, atol=1e-9)
        b, _, _, _ = oracle.integrate(ics2, t, pt2, pa2, m, planar=True, rtol=1e-9, atol=1e-9,
                                      impl="ref")
        assert np.array_equal(a, b), m
    w = np.zeros((2, 8))
    w[:, :4] = cyl_to_rect(ics2[:2])
    w[0, 4] = w[1, 6] = 1.0
    a, _, _ = oracle.integrate_dxdv(w, t, pt2, pa2, "dop853", planar=True)
    b, _, _ = oracle.integrate_dxdv(w, t, pt2, pa2, "dop853", planar=True, impl="ref")
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ELL)
@pytest.mark.parametrize("planar", [False, True])
def test_harness_forces_and_tidal_tensor(harness, oracle, golden, name, planar):
    pt, pa = _pot(golden, name, planar)
    R, phi = golden["pts_R"], golden["pts_phi"]
    z = 0 * R if planar else golden["pts_z"]
    x, y = R * np.cos(phi), R * np.sin(phi)
    acc, K, a32 = harness.forces(x, y, z, pt, pa, planar=planar)
    if planar:
        f = oracle.forces(R, z, phi, pt, pa, planar=True)
        Rf, ptq, R2, p2, Rp = f.T
        f = np.stack([Rf, 0 * Rf, ptq, R2, 0 * R2, 0 * R2, p2, Rp, 0 * R2], 1)
    else:
        f = oracle.forces(R, z, phi, pt, pa)
    Rf, zf, ptq = f[:, 0], f[:, 1], f[:, 2]
    c, s = x / R, y / R
    ref = np.stack([c * Rf - s / R * ptq, s * Rf + c / R * ptq, zf], 1)
    assert (np.abs(acc - ref).max(1) / np.abs(ref).max(1)).max() < 1e-12
    Kref = _cart_K(f, x, y)
    cols = [0, 1, 2] if planar else list(range(6))
    assert (np.abs(K - Kref)[:, cols].max(1) / np.abs(Kref).max(1)).max() < 1e-11
    assert (np.abs(a32 - ref).max(1) / np.abs(ref).max(1)).max() < 1e-6


@pytest.mark.parametrize("name", ELL)
def test_harness_potential_values(harness, golden, name):
    pt, pa = _pot(golden, name)
    R, z, phi = golden["pts_R"], golden["pts_z"], golden["pts_phi"]
    x, y = R * np.cos(phi), R * np.sin(phi)
    out = np.zeros_like(R)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    pti = np.ascontiguousarray(pt, np.int32)
    pad = np.ascontiguousarray(pa, np.float64)
    assert harness.lib.harness_potential(len(R), x.ctypes.data_as(dp), y.ctypes.data_as(dp),
                                         z.ctypes.data_as(dp), len(pti), pti.ctypes.data_as(ip),
                                         pad.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    ref = golden[f"ell_{name}_pyforces"][:, 9]
    if name == "twopowtri":
        assert np.isnan(out).all()
    else:
        assert (np.abs(out - ref) / np.abs(ref).max()).max() < 1e-13


@pytest.mark.parametrize("name", ELL)
def test_harness_orbits(harness, oracle, golden, name):
    """The machines on the host: the oracle's step sequence and orbits, 3D,
    planar and variational."""
    t = np.linspace(0, 6, 31)
    for planar, m in ((False, "dop853"), (False, "symplec4"), (True, "dopr54"), (True, "rk6")):
        pt, pa = _pot(golden, name, planar)
        ics = seeded_ics(6, 17, planar=planar)
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, m, planar=planar, rtol=1e-10,
                                           atol=1e-10)
        out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, m, planar=planar,
                                         rtol=1e-10, atol=1e-10)
        assert not err.any() and np.array_equal(ns, nref), m
        assert cyl_diff(ref, rect_to_cyl(out)).max() < 1e-10, m
    pt, pa = _pot(golden, name)
    w = golden["sph_dxdv_w3"]
    ref, _, nref = oracle.integrate_dxdv(w, t, pt, pa, "dop853")
    out, err, ns = harness.integrate(w, t, pt, pa, "dop853", var=True)
    assert not err.any() and np.array_equal(ns, nref)
    assert (np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)).max() < 1e-10
    # planar variational (the planar second derivatives of
    # EllipsoidalPotential.c:232-410)
    pt, pa = _pot(golden, name, planar=True)
    w = golden["c_dxdv_w2"]
    ref, _, nref = oracle.integrate_dxdv(w, t, pt, pa, "dop853", planar=True)
    out, err, ns = harness.integrate(w, t, pt, pa, "dop853", planar=True, var=True)
    assert not err.any() and np.array_equal(ns, nref)
    assert (np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)).max() < 1e-10


# ------------------------------------------------------------------ GPU ---
@pytest.fixture(scope="module")
def engine():
    from galpy_b200 import _lib, build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "no CUDA device: GPU tests need a GPU"
    return _lib.lib()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ELL)
def test_gpu_ellipsoidal(engine, oracle, golden, name):
    """The engine against the reference's C (golden: dop853 3D, symplec4
    planar, dop853 variational) and the oracle on a larger batch."""
    import galpy_b200 as gb

    pt, pa = _pot(golden, name)
    t = np.linspace(0, 5, 51)
    out, err = gb.integrateFullOrbit_cuda((pt, pa), golden["c_ics"].copy(), t, "dop853_cuda",
                                          progressbar=False)
    assert not err.any() and cyl_diff(golden[f"ell_{name}_3d"], out).max() < 1e-10
    out, err = gb.integratePlanarOrbit_cuda(_pot(golden, name, True),
                                            golden["c_ics_planar"].copy(), t, "symplec4_cuda",
                                            progressbar=False)
    assert not err.any() and cyl_diff(golden[f"ell_{name}_planar"], out).max() < 1e-10
    ref = golden[f"ell_{name}_dxdv3"]
    out, err = gb.integrate_dxdv_batch((pt, pa), golden["sph_dxdv_w3"], t, "dop853_cuda")
    assert not err.any()
    assert (np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)).max() < 1e-8
    ics = seeded_ics(256, 37)
    t = np.linspace(0, 6, 31)
    # each orbit's own conditioning: the oracle's response to a 1-ulp change
    # of the initial conditions (orbits through the PowerTriaxial cusp with
    # a fixed rk6 step reach 1e-8)
    ulp = 1 + np.finfo(float).eps * np.random.default_rng(1).choice([-1, 1], ics.shape)
    for m in ("rk6", "dopr54"):
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, m, rtol=1e-10, atol=1e-10)
        pert, _, _, _ = oracle.integrate(ics * ulp, t, pt, pa, m, rtol=1e-10, atol=1e-10)
        bound = np.maximum(1e-9, 10 * cyl_diff(ref, pert).max(axis=(1, 2)))
        out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, m + "_cuda",
                                                  rtol=1e-10, atol=1e-10, progressbar=False,
                                                  return_nsteps=True)
        same = ns == nref
        d = cyl_diff(ref, out).max(axis=(1, 2))
        assert not err.any() and same.mean() >= 0.9, m
        assert (d[same] < bound[same]).all() and np.median(d) < 1e-11, (m, d.max())


SOS_SAFE = {  # (potential, methods) whose every orbit below completes in the oracle
    "ell_powertri": ("rk4", "rk6", "dopr54", "dop853"),
    "ell_trigauss": ("rk4", "rk6"),
    "ell_perfell": ("rk4", "rk6"),
    "ell_twopowtri": ("rk4", "rk6"),
    "kuzmindisk": ("rk4", "rk6"),
}


def _sos_yo():
    return np.concatenate([seeded_ics(6, 21), np.zeros((6, 1))], 1)


@pytest.mark.parametrize("key", sorted(SOS_SAFE))
def test_oracle_surface_of_section_bitwise(oracle, golden, key):
    """integrateFullOrbit_sos in potentials symmetric about z = 0 (aligned or
    rotated about z only), bit for bit against the reference build.  Only
    runs whose every orbit completes in the oracle are given to the reference:
    where the oracle stops an orbit at dop853's smallest step (err 2; here
    orbits that escape, and tilted potentials, whose z = 0 is no symmetry
    plane) the reference's loop never returns."""
    pt, pa = golden[f"{key}_type"], golden[f"{key}_args"]
    psi = np.linspace(0.0, 12.0 * np.pi, 7)
    for m in SOS_SAFE[key]:
        a, ea, _ = oracle.integrate_sos(_sos_yo(), psi, pt, pa, m, rtol=1e-9, atol=1e-9)
        assert not ea.any(), m
        if oracle.ref_available():
            b, eb, _ = oracle.integrate_sos(_sos_yo(), psi, pt, pa, m, rtol=1e-9, atol=1e-9,
                                            impl="ref")
            assert np.array_equal(a, b) and np.array_equal(ea, eb), m


@pytest.mark.parametrize("method", ["rk4", "rk6", "dopr54", "dop853"])
def test_harness_surface_of_section(harness, oracle, golden, method):
    """The device's SOS machine (force at (x, y, A sin psi) through the
    ellipsoidal integral) against the oracle: same steps, same crossings."""
    from helpers import cyl_to_sos, sos_diff, sos_to_cyl

    pt, pa = golden["ell_powertri_type"], golden["ell_powertri_args"]
    yo = _sos_yo()
    psi = np.linspace(0.0, 12.0 * np.pi, 7)
    ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-9, atol=1e-9)
    raw, err, ns = harness.integrate_sos(cyl_to_sos(yo), psi, pt, pa, method, rtol=1e-9,
                                         atol=1e-9)
    assert not err.any() and np.array_equal(ns, nref)
    assert sos_diff(ref, sos_to_cyl(raw)).max() < 1e-9
