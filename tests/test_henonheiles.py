"""HenonHeilesPotential (galpy type 29, a planarPotential only).

Its force is not axisymmetric and a_y carries a term that is not
proportional to y (-amp x^2), so the device force library takes it through
its additive accumulator.  Oracle: HenonHeilesPotential.c restated, pinned
on galpy's Python forces and the reference's C orbits (golden vectors and,
where the reference build is present, bit for bit).  Host harness: the
device force and tidal-tensor code compiled for the CPU.  GPU: the engine
against the golden vectors and the oracle.
"""
import numpy as np
import pytest
from helpers import cyl_diff, cyl_to_rect, polar_to_sos, rect_to_cyl, sos_to_polar

METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]
T = np.linspace(0, 30, 61)


def _pot(golden):
    return golden["hh_type"], golden["hh_args"]


def _pts(golden):
    R, phi = golden["pts_R"], golden["pts_phi"]
    return R, phi, R * np.cos(phi), R * np.sin(phi)


def _angle_diff(a, b, k=3):
    d = np.abs(a - b)
    d[..., k] = np.abs((a[..., k] - b[..., k] + np.pi) % (2 * np.pi) - np.pi)
    return d


def test_oracle_forces_vs_galpy_python(oracle, golden):
    """Rforce, phitorque, R2deriv, phi2deriv, Rphideriv of
    HenonHeilesPotential.c:6-53 against galpy's Python methods."""
    pt, pa = _pot(golden)
    R, phi, _, _ = _pts(golden)
    f = oracle.forces(R, 0 * R, phi, pt, pa, planar=True)
    py = golden["hh_pyforces"]
    np.testing.assert_allclose(f[:, :5], py[:, :5], rtol=1e-13, atol=1e-13)


def test_oracle_golden_and_bitwise(oracle, golden):
    """The reference's C orbits in the potential: golden vectors for every
    method, the variational DOP853 and the x = 0 surface of section, and bit
    for bit against the reference build where it is present."""
    pt, pa = _pot(golden)
    ics = golden["hh_ics"]
    for m in METHODS:
        a, err, _, _ = oracle.integrate(ics, T, pt, pa, m, planar=True, rtol=1e-10, atol=1e-10)
        assert not err.any()
        np.testing.assert_allclose(a, golden[f"hh_{m}"], rtol=0, atol=1e-12, err_msg=m)
    a, _, _ = oracle.integrate_dxdv(golden["hh_dxdv_w2"], np.linspace(0, 10, 21), pt, pa,
                                    "dop853", planar=True)
    np.testing.assert_allclose(a, golden["hh_dop853_dxdv2"], rtol=0, atol=1e-11)
    yo = np.concatenate([ics, np.zeros((len(ics), 1))], 1)
    psi = np.linspace(0.0, 20.0 * np.pi, 11)
    for m in ("rk6", "dop853"):
        a, err, _ = oracle.integrate_sos(yo, psi, pt, pa, m, rtol=1e-10, atol=1e-10, planar=True,
                                         surface=0)
        assert not err.any()
        np.testing.assert_allclose(a, golden[f"hh_sos0_{m}"], rtol=0, atol=1e-12, err_msg=m)
    if not oracle.ref_available():
        return
    ics2 = np.stack([np.full(6, 0.25), np.linspace(-0.3, 0.3, 6), np.full(6, 0.3),
                     np.linspace(0.5, 5.5, 6)], 1)
    for m in METHODS:
        a, ea, _, _ = oracle.integrate(ics2, T, pt, pa, m, planar=True, rtol=1e-9, atol=1e-9)
        b, eb, _, _ = oracle.integrate(ics2, T, pt, pa, m, planar=True, rtol=1e-9, atol=1e-9,
                                       impl="ref")
        assert np.array_equal(a, b) and np.array_equal(ea, eb), m


def test_harness_forces_and_tidal_tensor(harness, oracle, golden):
    """The device force code (additive a_y term) and the Cartesian tidal
    tensor against the oracle's polar forces and Hessian."""
    pt, pa = _pot(golden)
    R, phi, x, y = _pts(golden)
    acc, K, a32 = harness.forces(x, y, 0 * x, pt, pa, planar=True)
    f = oracle.forces(R, 0 * R, phi, pt, pa, planar=True)
    Rf, ptq, R2, p2, Rp = f.T
    c, s = x / R, y / R
    ref = np.stack([c * Rf - s / R * ptq, s * Rf + c / R * ptq], 1)
    scale = np.abs(ref).max(1)
    assert (np.abs(acc[:, :2] - ref).max(1) / scale).max() < 1e-13
    assert not acc[:, 2].any()
    Kxx = -c * c * R2 + 2 * c * s / R / R * ptq + s * s / R * Rf + 2 * s * c / R * Rp - s * s / R / R * p2
    Kxy = (-s * c * R2 + (s * s - c * c) / R / R * ptq - c * s / R * Rf - (c * c - s * s) / R * Rp
           + c * s / R / R * p2)
    Kyy = -s * s * R2 - 2 * s * c / R / R * ptq - 2 * s * c / R * Rp + c * c / R * Rf - c * c / R / R * p2
    Kref = np.stack([Kxx, Kxy, Kyy], 1)
    assert (np.abs(K[:, :3] - Kref).max(1) / np.abs(Kref).max(1)).max() < 1e-12
    assert (np.abs(a32[:, :2] - ref).max(1) / scale).max() < 3e-5


def test_harness_potential_value(harness, golden):
    """The energy kernel's potential against galpy's Python value."""
    import ctypes

    pt, pa = _pot(golden)
    R, phi, x, y = _pts(golden)
    out = np.zeros_like(R)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    pti = np.ascontiguousarray(pt, np.int32)
    pad = np.ascontiguousarray(pa, np.float64)
    z = np.zeros_like(R)
    assert harness.lib.harness_potential_in(1, len(R), x.ctypes.data_as(dp),
                                            y.ctypes.data_as(dp), z.ctypes.data_as(dp),
                                            len(pti), pti.ctypes.data_as(ip),
                                            pad.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    ref = golden["hh_pyforces"][:, 5]
    assert (np.abs(out - ref) / np.abs(ref).max()).max() < 1e-13


@pytest.mark.parametrize("method", METHODS)
def test_harness_orbits(harness, oracle, golden, method):
    """The machines on the host: the oracle's step sequence and its orbits
    to their conditioning (a chaotic potential: short span)."""
    pt, pa = _pot(golden)
    ics = golden["hh_ics"]
    t = np.linspace(0, 10, 21)
    ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, method, planar=True, rtol=1e-10,
                                       atol=1e-10)
    out, err, ns = harness.integrate(cyl_to_rect(ics), t, pt, pa, method, planar=True,
                                     rtol=1e-10, atol=1e-10)
    assert not err.any() and np.array_equal(ns, nref)
    assert cyl_diff(ref, rect_to_cyl(out)).max() < 1e-10


@pytest.mark.parametrize("method", ["rk6", "dop853"])
def test_harness_surface_of_section(harness, oracle, golden, method):
    pt, pa = _pot(golden)
    yo = np.concatenate([golden["hh_ics"], np.zeros((8, 1))], 1)
    psi = np.linspace(0.0, 20.0 * np.pi, 11)
    ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-10, atol=1e-10,
                                        planar=True, surface=0)
    raw, err, ns = harness.integrate_sos(polar_to_sos(yo, 0), psi, pt, pa, method, rtol=1e-10,
                                         atol=1e-10, surface=0)
    assert not err.any() and np.array_equal(ns, nref)
    assert _angle_diff(sos_to_polar(raw, 0), ref).max() < 1e-9


# ------------------------------------------------------------------ GPU ---
@pytest.fixture(scope="module")
def engine():
    from galpy_b200 import _lib, build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "no CUDA device: GPU tests need a GPU"
    return _lib.lib()


@pytest.mark.gpu
@pytest.mark.parametrize("method", METHODS)
def test_gpu_golden_orbits(engine, golden, method):
    """integratePlanarOrbit_cuda against the reference's C orbits; the
    golden span is a few dynamical times of a chaotic potential, so the
    bound is the adaptive methods' agreement plus its growth."""
    import galpy_b200 as gb

    out, err = gb.integratePlanarOrbit_cuda(_pot(golden), golden["hh_ics"].copy(), T,
                                            method + "_cuda", rtol=1e-10, atol=1e-10,
                                            progressbar=False)
    assert not err.any() and cyl_diff(golden[f"hh_{method}"], out).max() < 1e-8


@pytest.mark.gpu
def test_gpu_oracle_batch_variational_and_sos(engine, oracle, golden):
    """A larger batch against the oracle (same step sequence), the
    variational DOP853 against the reference's C, and the x = 0 surface of
    section against the reference's C."""
    import galpy_b200 as gb

    pt, pa = _pot(golden)
    rng = np.random.default_rng(41)
    n = 512
    ics = np.stack([rng.uniform(0.1, 0.4, n), rng.uniform(-0.25, 0.25, n),
                    rng.uniform(0.1, 0.3, n), rng.uniform(0, 2 * np.pi, n)], 1)
    t = np.linspace(0, 10, 21)
    for m in ("rk6", "dopr54", "dop853"):
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, m, planar=True, rtol=1e-10,
                                           atol=1e-10)
        out, err, ns = gb.integratePlanarOrbit_cuda((pt, pa), ics.copy(), t, m + "_cuda",
                                                    rtol=1e-10, atol=1e-10, progressbar=False,
                                                    return_nsteps=True)
        same = ns == nref
        d = cyl_diff(ref, out).max(axis=(1, 2))
        assert not err.any() and same.mean() >= 0.9 and d[same].max() < 1e-9, m
    ref = golden["hh_dop853_dxdv2"]
    out, err = gb.integrate_dxdv_batch((pt, pa), golden["hh_dxdv_w2"], np.linspace(0, 10, 21),
                                       "dop853_cuda", planar=True)
    assert not err.any()
    assert (np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)).max() < 1e-8
    ics = golden["hh_ics"]
    psi = np.linspace(0.0, 20.0 * np.pi, 11)
    for m in ("rk6", "dop853"):
        out, err = gb.integratePlanarOrbit_sos_cuda((pt, pa), ics, psi, 0.0, m + "_cuda",
                                                    surface="x", rtol=1e-10, atol=1e-10,
                                                    progressbar=False)
        assert not err.any() and _angle_diff(out, golden[f"hh_sos0_{m}"]).max() < 1e-8, m
