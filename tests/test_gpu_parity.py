"""CUDA engine vs the CPU oracle on a B200, through the C ABI.

Tolerances: fixed-step methods take the same step size per orbit as the
reference and agree to the orbits' own conditioning (differences of 1e-16
in the force grow to ~1e-13 over 1e4 steps; the oracle shows the same growth
under 1e-16 perturbations of the initial conditions); DOP853 takes the same
accepted step sequence and agrees well inside its tolerance.
"""
import ctypes

import numpy as np
import pytest
from helpers import ADDED_POTS, KINKED, cyl_diff, golden_pot, sos_diff, cyl_to_rect, rect_to_cyl, seeded_ics, unit_deviations

import galpy_b200 as gb
from galpy_b200 import _lib

pytestmark = pytest.mark.gpu
METHODS = ["leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"]


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    n = _lib.lib().galpy_cuda_device_count()
    assert n > 0, "no CUDA device: GPU tests need a GPU"
    return _lib.lib()


def cuda(method):
    return method + "_cuda"


def test_config0_symplec4_parity(oracle, mw14):
    """Config 0 at full size: all 10,000 orbits, symplec4 with galpy's
    estimated step, MWPotential2014, t in [0,100] with 1001 outputs, step
    for step against the oracle (bit-identical to the reference's C).

    Every orbit takes the reference's step size (the same estimator
    decisions).  The results then differ only by the force's rounding (the
    engine's special functions are not GSL's), which each orbit amplifies
    by its own conditioning; the bound per orbit is the oracle's own
    response to a one-ulp change of that orbit's initial conditions (times
    30: the engine's force differs from the reference's by a few ulp at each
    of ~50,000 evaluations, not once), and never looser than 1e-10."""
    pt, pa = mw14
    ics = seeded_ics(10000, 0)
    t = np.linspace(0, 100, 1001)
    ref, eref, nref, _ = oracle.integrate(ics, t, pt, pa, "symplec4")
    out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "symplec4_cuda",
                                              progressbar=False, return_nsteps=True)
    assert not err.any() and not eref.any()
    same = ns == nref
    assert same.mean() >= 0.999, same.mean()
    per = cyl_diff(ref, out).max(axis=(1, 2))
    assert np.median(per[same]) < 1e-12, np.median(per[same])
    ulp = 1 + np.finfo(float).eps * np.random.default_rng(0).choice([-1, 1], ics.shape)
    pert, _, npert, _ = oracle.integrate(ics * ulp, t, pt, pa, "symplec4")
    resp = cyl_diff(ref, pert).max(axis=(1, 2))
    bound = np.minimum(np.maximum(1e-12, 30 * resp), 1e-10)
    bad = same & (per > bound)
    assert not bad.any(), (bad.sum(), per[bad][:10], resp[bad][:10])


def test_config0_full_size_energy(mw14, oracle):
    """All 10,000 config-0 orbits: size-independent checks (energy
    conservation per orbit, agreement with a 2x smaller step)."""
    pt, pa = mw14
    ics = seeded_ics(10000, 0)
    t = np.linspace(0, 100, 1001)
    out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "symplec4_cuda",
                                              progressbar=False, return_nsteps=True)
    assert not err.any() and np.isfinite(out).all()
    E = oracle.energy_cyl(out[:, ::50], pt, pa)
    rel = np.abs(E / E[:, :1] - 1)
    assert rel.max() < 1e-8, rel.max()


NAMED_POTS = ["mw14", "hernquist", "loghalo", "logtri"]


def named_pot(golden, name, planar):
    """The potentials the plain form is specified for: MWPotential2014, a
    Hernquist sphere and the logarithmic halo (axisymmetric and triaxial).
    galpy's planar argument lists of the last three equal the 3D ones
    (galpy/orbit/integratePlanarOrbit.py:67-79, 148-153)."""
    if name == "mw14":
        return ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
                else (golden["mw14_type"], golden["mw14_args"]))
    return golden[f"{name}_type"], golden[f"{name}_args"]


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("potname", NAMED_POTS)
def test_methods_vs_oracle(oracle, golden, method, planar, potname):
    pt, pa = named_pot(golden, potname, planar)
    ics = seeded_ics(257, 8 + NAMED_POTS.index(potname), planar=planar)
    t = np.linspace(0, 20, 201)
    ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, method, planar=planar)
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    out, err, ns = fn((pt, pa), ics.copy(), t, cuda(method), progressbar=False,
                      return_nsteps=True)
    assert not err.any()
    same = ns == nref
    assert same.mean() >= 0.99
    d = cyl_diff(ref, out).max(axis=(1, 2))
    far = same & (d >= 1e-10)
    if far.any():
        # The reference takes the angle of its Cartesian force routes as
        # acos(x / R) (integratePlanarOrbit.c:1022, integrateFullOrbit.c:1313),
        # ill-conditioned near the x axis: in the triaxial halo a step that
        # lands within ~1e-8 rad of the axis moves its force by up to ~1e-8,
        # and the orbit by ~1e-10 after it.  The engine's force is Cartesian
        # (no angle); with the angle from atan2 -- the only change -- the
        # oracle agrees with it again.  What is left beyond 1e-10 is bounded
        # by that oracle's response to a one-ulp change of the orbit's
        # initial conditions.
        with oracle.phi_from_atan2():
            ref2, _, nref2, _ = oracle.integrate(ics[far], t, pt, pa, method, planar=planar)
            d2 = cyl_diff(ref2, out[far]).max(axis=(1, 2))
            still = (d2 >= 1e-10) | (nref2 != ns[far])
            if still.any():
                ulp = 1 + np.finfo(float).eps * np.random.default_rng(3).choice(
                    [-1, 1], ics[far][still].shape)
                pert, _, _, _ = oracle.integrate(ics[far][still] * ulp, t, pt, pa, method,
                                                 planar=planar)
                resp = cyl_diff(ref2[still], pert).max(axis=(1, 2))
                assert (d2[still] <= np.maximum(1e-10, 30 * resp)).all(), (d2[still], resp)


@pytest.mark.parametrize("method", METHODS)
def test_golden_reference_vectors(golden, method):
    """The committed outputs of the reference's own C build."""
    t = np.linspace(0, 5, 51)
    out, err = gb.integrateFullOrbit_cuda((golden["mw14_type"], golden["mw14_args"]),
                                          golden["c_ics"].copy(), t, cuda(method),
                                          progressbar=False)
    assert cyl_diff(golden[f"c_{method}_3d"], out).max() < 1e-11
    out, err = gb.integratePlanarOrbit_cuda(
        (golden["mw14_planar_type"], golden["mw14_planar_args"]), golden["c_ics_planar"].copy(),
        t, cuda(method), progressbar=False)
    assert cyl_diff(golden[f"c_{method}_planar"], out).max() < 1e-11


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("planar", [False, True])
def test_variational_vs_oracle(oracle, mw14, mw14_planar, method, planar):
    pt, pa = mw14_planar if planar else mw14
    dim = 2 if planar else 3
    w = unit_deviations(cyl_to_rect(seeded_ics(4, 9, planar=planar)), dim)
    t = np.linspace(0, 5, 51)
    ref, _, nref = oracle.integrate_dxdv(w, t, pt, pa, method, planar=planar)
    out, err, ns = gb.integrate_dxdv_batch((pt, pa), w, t, cuda(method), planar=planar,
                                           return_nsteps=True)
    assert not err.any() and np.array_equal(ns, nref)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert (np.abs(out - ref) / scale).max() < 1e-10
    # galpy's single-orbit entry points
    single = gb.integratePlanarOrbit_dxdv_cuda if planar else gb.integrateFullOrbit_dxdv_cuda
    res, e = single((pt, pa), w[0, :2 * dim], w[0, 2 * dim:], t, cuda(method))
    assert e == 0 and np.allclose(res, out[0], rtol=0, atol=1e-12)


def test_golden_variational_vectors(golden):
    t = np.linspace(0, 3, 31)
    for method in METHODS:
        out, err = gb.integrate_dxdv_batch((golden["mw14_type"], golden["mw14_args"]),
                                           golden["c_dxdv_w3"], t, cuda(method))
        ref = golden[f"c_{method}_dxdv3"]
        assert (np.abs(out - ref) / np.abs(ref).max(axis=1, keepdims=True)).max() < 1e-10


def test_dop853_ragged_times(oracle, mw14):
    """Config-1 style: log-uniform radii down to 0.05, per-orbit end times,
    101 snapshots, rtol = atol = 1e-10."""
    pt, pa = mw14
    ics = seeded_ics(400, 1, r_range=(0.05, 3.0), log_r=True)
    rng = np.random.default_rng(1)
    tend = np.exp(rng.normal(np.log(50), 0.7, len(ics)))
    t = np.linspace(0, 1, 101)[None, :] * tend[:, None]
    ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, "dop853", rtol=1e-10, atol=1e-10)
    out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "dop853_cuda",
                                              rtol=1e-10, atol=1e-10, progressbar=False,
                                              return_nsteps=True)
    assert not err.any()
    same = ns == nref
    assert same.mean() >= 0.98, same.mean()
    d = cyl_diff(ref, out)[same]
    scale = np.maximum(np.abs(ref[same]), 1.0)
    assert (d / scale).max() < 1e-7


def test_dopr54_golden_vectors(golden):
    """dopr54 against the reference's own C: per-orbit time grids, and the
    smallest-step rule (every step forced at the interval's first step /
    10000, err = 1 on every orbit)."""
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), golden["c_ics"].copy(),
                                              golden["c_indiv_t"], "dopr54_cuda", rtol=1e-10,
                                              atol=1e-10, progressbar=False, return_nsteps=True)
    assert not err.any()
    assert cyl_diff(golden["c_dopr54_indiv"], out).max() < 1e-10
    out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), golden["c_ics"].copy(),
                                              np.array([0.0, 50.0]), "dopr54_cuda", dt=50.0,
                                              rtol=1e-20, atol=1e-20, progressbar=False,
                                              return_nsteps=True)
    assert np.array_equal(err, golden["c_dopr54_forced_err"]) and np.all(ns == 10000)
    assert cyl_diff(golden["c_dopr54_forced"], out).max() < 1e-10


@pytest.mark.parametrize("method", ["rk6", "symplec6", "dopr54"])
def test_generic_potentials_and_fixed_dt(oracle, golden, method):
    """Kernels that walk the component list at run time (a triaxial
    logarithmic halo plus a Hernquist sphere), an explicit dt, and the
    float32-force variant."""
    pt = np.concatenate([golden["logtri_type"], golden["hernquist_type"]])
    pa = np.concatenate([golden["logtri_args"], golden["hernquist_args"]])
    ics = seeded_ics(128, 36)
    t = np.linspace(0, 10, 41)
    for dt in (None, 0.01):
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, method, dt=dt)
        out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, cuda(method), dt=dt,
                                                  progressbar=False, return_nsteps=True)
        assert not err.any()
        same = ns == nref
        assert same.mean() >= 0.99
        assert cyl_diff(ref, out).max(axis=(1, 2))[same].max() < 1e-10
    f32, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, cuda(method), dt=0.01,
                                          progressbar=False, precision="f32force")
    d = cyl_diff(out, f32)[..., :5].max()
    assert not err.any() and 0 < d < 1e-4, d


@pytest.mark.parametrize("name", ADDED_POTS)
def test_spherical_potentials(oracle, golden, name):
    """Orbits in each spherical potential: the reference's own C (golden
    vectors: dop853 3D, symplec4 planar, dop853 variational) and the oracle
    with rk6 / dopr54, FP64 and FP32 force."""
    pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
    # the homogeneous sphere's force has a kink at its surface and the Kuzmin
    # disk's a jump at its plane, where an adaptive step's accept / reject can
    # follow a rounding difference
    tol = 1e-8 if name in KINKED else 1e-10
    t = np.linspace(0, 5, 51)
    out, err = gb.integrateFullOrbit_cuda((pt, pa), golden["c_ics"].copy(), t, "dop853_cuda",
                                          progressbar=False)
    assert not err.any() and cyl_diff(golden[f"sph_{name}_3d"], out).max() < tol
    out, err = gb.integratePlanarOrbit_cuda(golden_pot(golden, name, True),
                                            golden["c_ics_planar"].copy(), t, "symplec4_cuda",
                                            progressbar=False)
    assert not err.any() and cyl_diff(golden[f"sph_{name}_planar"], out).max() < tol
    ref = golden[f"sph_{name}_dxdv3"]
    out, err = gb.integrate_dxdv_batch((pt, pa), golden["sph_dxdv_w3"], t, "dop853_cuda")
    assert (np.abs(out - ref) / np.abs(ref).max(axis=(1, 2), keepdims=True)).max() < 100 * tol
    ics = seeded_ics(256, 37)
    t = np.linspace(0, 10, 41)
    for m in ("rk6", "dopr54"):
        ref, _, nref, _ = oracle.integrate(ics, t, pt, pa, m, rtol=1e-10, atol=1e-10)
        out, err, ns = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, cuda(m), rtol=1e-10,
                                                  atol=1e-10, progressbar=False,
                                                  return_nsteps=True)
        same = ns == nref
        d = cyl_diff(ref, out).max(axis=(1, 2))
        if name in KINKED:
            # at the kink (jump) an adaptive step's accept / reject follows
            # rounding, and dopr54 forces its smallest step at the Kuzmin
            # disk's plane (err 1, as the reference): each orbit is bounded
            # by the oracle's own response to a 1-ulp change of its
            # initial conditions
            ulp = 1 + np.finfo(float).eps * np.random.default_rng(1).choice([-1, 1], ics.shape)
            pert, _, _, _ = oracle.integrate(ics * ulp, t, pt, pa, m, rtol=1e-10, atol=1e-10)
            bound = np.maximum(1e-9, 10 * cyl_diff(ref, pert).max(axis=(1, 2)))
            assert np.isin(err, (0, 1)).all() and (d <= bound).all(), (m, d.max())
        else:
            assert not err.any() and same.mean() >= 0.9, m
            assert d[same].max() < 1e-9 and d.max() < 1e-6, (m, d.max())
    f32, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "symplec4_cuda", dt=0.01,
                                          progressbar=False, precision="f32force")
    f64, _ = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "symplec4_cuda", dt=0.01,
                                        progressbar=False)
    # single-precision forces over 1,000 steps (the strong power-law orbits
    # cover the most periods)
    d = cyl_diff(f64, f32)[..., :5].max(axis=(1, 2))
    assert not err.any()
    if name == "kuzmindisk":
        # the vertical force changes sign at the disk's plane: a kick taken
        # within rounding of z = 0 flips, so a few orbits in a hundred
        # depart by ~0.1 in FP32 (FP64 orbits do the same under a 1e-7 change
        # of their initial conditions); the rest agree to single precision
        assert (d > 1e-2).mean() <= 0.06 and np.median(d) < 1e-5, (d > 1e-2).sum()
    else:
        assert d.max() < 1e-2


@pytest.mark.parametrize("method", ["rk4", "rk6", "dopr54", "dop853"])
def test_surface_of_section(oracle, golden, method):
    """integrateFullOrbit_sos_cuda against the reference's C (golden) and the
    oracle on a larger batch with per-orbit increments."""
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    yo = golden["sos_yo"].copy()
    out, err = gb.integrateFullOrbit_sos_cuda((pt, pa), yo[:, :6], golden["sos_psi"],
                                              yo[:, 6], cuda(method), rtol=1e-10, atol=1e-10,
                                              progressbar=False)
    assert not err.any()
    assert sos_diff(golden[f"sos_{method}"], out).max() < 1e-9
    ics = seeded_ics(300, 38)
    yo = np.concatenate([ics, np.zeros((300, 1))], 1)
    psi = np.linspace(0.0, 1.0, 9)[None, :] * np.linspace(6.0, 40.0, 300)[:, None]
    ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-10, atol=1e-10)
    out, err, ns = gb.integrateFullOrbit_sos_cuda((pt, pa), ics, psi, 0.0, cuda(method),
                                                  rtol=1e-10, atol=1e-10, progressbar=False,
                                                  return_nsteps=True)
    same = ns == nref
    assert not err.any() and same.mean() >= 0.95, same.mean()
    d = sos_diff(ref, out).max(axis=(1, 2))
    assert d[same].max() < 1e-8 and d.max() < 1e-6, d.max()
    # the symplectic methods are not integrated in psi (as in the reference)
    with pytest.raises(gb.MethodNotSupported):
        gb.integrateFullOrbit_sos_cuda((pt, pa), ics[:2], psi[0], 0.0, "symplec4_cuda")


@pytest.mark.parametrize("surface", ["x", "y"])
@pytest.mark.parametrize("method", ["rk4", "dop853"])
def test_planar_surface_of_section(oracle, golden, method, surface):
    """integratePlanarOrbit_sos_cuda against the reference's C (golden) and
    the oracle on a larger batch."""
    pt, pa = golden["mw14_planar_type"], golden["mw14_planar_args"]
    s = 1 if surface == "y" else 0
    yo = golden["sos_planar_yo"]
    out, err = gb.integratePlanarOrbit_sos_cuda((pt, pa), yo[:, :4], golden["sos_psi"],
                                                yo[:, 4], cuda(method), surface=surface,
                                                rtol=1e-10, atol=1e-10, progressbar=False)
    ref = golden[f"sos_planar{s}_{method}"]
    d = np.abs(out - ref)
    d[..., 3] = np.abs((out[..., 3] - ref[..., 3] + np.pi) % (2 * np.pi) - np.pi)
    assert not err.any() and d.max() < 1e-9
    ics = seeded_ics(300, 39, planar=True)
    yo = np.concatenate([ics, np.zeros((300, 1))], 1)
    psi = np.linspace(0.0, 12.0 * np.pi, 7)
    ref, _, nref = oracle.integrate_sos(yo, psi, pt, pa, method, rtol=1e-10, atol=1e-10,
                                        planar=True, surface=s)
    out, err, ns = gb.integratePlanarOrbit_sos_cuda((pt, pa), ics, psi, 0.0, cuda(method),
                                                    surface=surface, rtol=1e-10, atol=1e-10,
                                                    progressbar=False, return_nsteps=True)
    same = ns == nref
    d = np.abs(out - ref)
    d[..., 3] = np.abs((out[..., 3] - ref[..., 3] + np.pi) % (2 * np.pi) - np.pi)
    d = d.max(axis=(1, 2))
    assert not err.any() and same.mean() >= 0.95 and d[same].max() < 1e-8 and d.max() < 1e-6


def test_device_api_surface_of_section(golden):
    """The surface-of-section systems through the device-resident entry point
    (SoA rows, galpy-coordinate output) agree with the host entry points."""
    import torch

    from helpers import cyl_to_sos, polar_to_sos

    dev = torch.device("cuda:0")
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    yo = golden["sos_yo"]
    psi = golden["sos_psi"]
    ref, _ = gb.integrateFullOrbit_sos_cuda((pt, pa), yo[:, :6], psi, yo[:, 6], "dop853_cuda",
                                            rtol=1e-10, atol=1e-10, progressbar=False)
    comps, n = gb.compile_potential((pt, pa))
    w0 = torch.tensor(cyl_to_sos(yo).T.copy(), device=dev)
    out = torch.empty((7, len(psi), len(yo)), dtype=torch.float64, device=dev)
    e = torch.empty(len(yo), dtype=torch.int32, device=dev)
    gb.integrate_device(torch.tensor(comps, device=dev), n, w0, torch.tensor(psi, device=dev),
                        out, e, "dop853_cuda", out_layout="soa_cyl", rtol=1e-10, atol=1e-10,
                        system="sos")
    torch.cuda.synchronize()
    got = out.cpu().numpy().transpose(2, 1, 0)
    assert not e.cpu().numpy().any() and sos_diff(ref, got).max() < 1e-13
    # planar, surface y = 0
    pt2, pa2 = golden["mw14_planar_type"], golden["mw14_planar_args"]
    yo5 = golden["sos_planar_yo"]
    ref, _ = gb.integratePlanarOrbit_sos_cuda((pt2, pa2), yo5[:, :4], psi, yo5[:, 4],
                                              "rk4_cuda", surface="y", rtol=1e-10, atol=1e-10,
                                              progressbar=False)
    comps, n = gb.compile_potential((pt2, pa2), planar=True)
    w0 = torch.tensor(polar_to_sos(yo5, 1).T.copy(), device=dev)
    out = torch.empty((5, len(psi), len(yo5)), dtype=torch.float64, device=dev)
    e = torch.empty(len(yo5), dtype=torch.int32, device=dev)
    gb.integrate_device(torch.tensor(comps, device=dev), n, w0, torch.tensor(psi, device=dev),
                        out, e, "rk4_cuda", planar=True, out_layout="soa_cyl", rtol=1e-10,
                        atol=1e-10, system="sos_planar_y")
    torch.cuda.synchronize()
    got = out.cpu().numpy().transpose(2, 1, 0)
    d = np.abs(got - ref)
    d[..., 3] = np.abs((got[..., 3] - ref[..., 3] + np.pi) % (2 * np.pi) - np.pi)
    assert not e.cpu().numpy().any() and d.max() < 1e-13
    # inconsistent requests are refused before any work
    with pytest.raises(gb.CudaError):
        gb.integrate_device(torch.tensor(comps, device=dev), n, w0,
                            torch.tensor(psi, device=dev), out, e, "symplec4_cuda", planar=True,
                            system="sos_planar_y")
    with pytest.raises(gb.CudaError):
        gb.integrate_device(torch.tensor(comps, device=dev), n, w0,
                            torch.tensor(psi, device=dev), out, e, "rk4_cuda", planar=False,
                            system="sos_planar_y")


def test_device_api_soa_matches_galpy_layout(mw14):
    import torch

    pt, pa = mw14
    ics = seeded_ics(1000, 21)
    t = np.linspace(0, 10, 11)
    res, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "dop853_cuda",
                                          progressbar=False)
    comps, n = gb.compile_potential((pt, pa))
    dev = torch.device("cuda:0")
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    tt = torch.tensor(t, device=dev)
    out = torch.empty((6, 11, len(ics)), dtype=torch.float64, device=dev)
    e = torch.empty(len(ics), dtype=torch.int32, device=dev)
    # same kernel specialisation as the galpy-facing call
    gb.integrate_device(torch.tensor(comps, device=dev), n, w0, tt, out, e, "dop853_cuda",
                        signature=gb.signature((pt, pa)), comps_host=comps)
    torch.cuda.synchronize()
    got = rect_to_cyl(out.cpu().numpy().transpose(2, 1, 0))
    assert cyl_diff(res, got).max() < 1e-14 and not e.cpu().numpy().any()


def test_potential_groups(oracle, mw14):
    """Ragged multi-potential batch: every orbit uses its own group's
    parameters (config-4 style variants of MWPotential2014)."""
    import torch

    pt, pa = mw14
    rng = np.random.default_rng(4)
    ngroup = 5
    args = np.tile(pa, (ngroup, 1))
    scale = rng.uniform(0.8, 1.2, (ngroup, 6))
    args[:, 6] *= scale[:, 0]  # MN a
    args[:, 7] *= scale[:, 1]  # MN b
    args[:, 9] *= scale[:, 2]  # NFW a
    args[:, 0] *= scale[:, 3]
    args[:, 5] *= scale[:, 4]
    args[:, 8] *= scale[:, 5]
    counts = rng.integers(10, 40, ngroup)
    group = np.repeat(np.arange(ngroup), counts).astype(np.int32)
    ics = seeded_ics(len(group), 5)
    t = np.linspace(0, 10, 21)
    comps, n = gb.compile_potential((pt, args.ravel()), ngroup=ngroup)
    dev = torch.device("cuda:0")
    out = torch.empty((6, 21, len(ics)), dtype=torch.float64, device=dev)
    e = torch.empty(len(ics), dtype=torch.int32, device=dev)
    ns = torch.empty(len(ics), dtype=torch.int64, device=dev)
    gb.integrate_device(torch.tensor(comps, device=dev), n,
                        torch.tensor(cyl_to_rect(ics).T.copy(), device=dev),
                        torch.tensor(t, device=dev), out, e, "dop853_cuda", nsteps=ns,
                        group=torch.tensor(group, device=dev), rtol=1e-9, atol=1e-9)
    got = rect_to_cyl(out.cpu().numpy().transpose(2, 1, 0))
    ns = ns.cpu().numpy()
    for g in range(ngroup):
        sel = group == g
        ref, _, nref, _ = oracle.integrate(ics[sel], t, pt, args[g], "dop853", rtol=1e-9,
                                           atol=1e-9)
        d = cyl_diff(ref, got[sel]).max(axis=(1, 2))
        same = ns[sel] == nref  # an accept/reject flip at err ~ 1 changes the steps
        assert same.mean() >= 0.9 and d[same].max() < 1e-8, (same.mean(), d.max())
        assert d.max() < 1e-6


def test_f32_force_variant(mw14):
    pt, pa = mw14
    ics = seeded_ics(512, 22)
    t = np.linspace(0, 10, 11)
    a, _ = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "symplec4_cuda", dt=0.01,
                                      progressbar=False)
    b, _ = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "symplec4_cuda", dt=0.01,
                                      progressbar=False, precision="f32force")
    d = cyl_diff(a, b)[..., :5].max()
    assert 0 < d < 1e-4, d


def test_edge_cases(mw14, oracle):
    pt, pa = mw14
    t = np.linspace(0, 5, 11)
    # no orbits
    out, err = gb.integrateFullOrbit_cuda((pt, pa), np.zeros((0, 6)), t, "dop853_cuda")
    assert out.shape == (0, 11, 6)
    # one orbit given as a 1-D array; yo overwritten with rectangular coords
    yo = seeded_ics(1, 30)[0].copy()
    yo0 = yo.copy()
    out, err = gb.integrateFullOrbit_cuda((pt, pa), yo, t, "symplec4_cuda")
    assert out.shape == (11, 6) and err == 0
    assert np.allclose(yo, cyl_to_rect(yo0[None])[0], rtol=0, atol=1e-15)
    assert cyl_diff(out[:1], yo0[None]).max() < 1e-15  # angle wraps to (-pi, pi] as in galpy
    # a single output time
    out, err = gb.integrateFullOrbit_cuda((pt, pa), seeded_ics(3, 31), t[:1], "rk4_cuda")
    assert out.shape == (3, 1, 6)
    # backward integration
    ics = seeded_ics(64, 32)
    tb = np.linspace(0, -10, 101)
    for m in METHODS:
        ref, _, _, _ = oracle.integrate(ics, tb, pt, pa, m)
        out, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), tb, cuda(m),
                                              progressbar=False)
        assert cyl_diff(ref, out).max() < 1e-10
    # non-finite initial condition: err 3, NaN rows, neighbours unaffected
    ics = seeded_ics(5, 33)
    ics[2, 0] = np.nan
    out, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "dop853_cuda",
                                          progressbar=False)
    assert err.tolist() == [0, 0, 3, 0, 0] and np.isnan(out[2, 1:]).all()
    # attempt budget
    out, err = gb.integrateFullOrbit_cuda((pt, pa), seeded_ics(4, 34), np.linspace(0, 100, 11),
                                          "dop853_cuda", max_attempts=30, progressbar=False)
    assert np.all(err == 2) and np.isnan(out[:, -1]).all()
    # dopr54 with a step too small to advance the time (t near 1e17): err 2
    out, err = gb.integrateFullOrbit_cuda((pt, pa), seeded_ics(3, 36),
                                          1e17 + np.array([0.0, 128.0, 256.0]), "dopr54_cuda",
                                          dt=1.0, progressbar=False)
    assert np.all(err == 2) and np.isnan(out[:, 1:]).all()
    # unsupported method and potential: typed errors
    with pytest.raises(ValueError):
        gb.integrateFullOrbit_cuda((pt, pa), seeded_ics(2, 35), t, "ias15_cuda")
    with pytest.raises(gb.PotentialNotSupported):
        gb.integrateFullOrbit_cuda(([11], [1.0, 1.0]), seeded_ics(2, 35), t, "dop853_cuda")


def test_progress_callback(mw14):
    pt, pa = mw14
    calls = []
    cb = _lib.CALLBACK(lambda: calls.append(1))
    ics = seeded_ics(300, 40)
    t = np.linspace(0, 10, 11)
    yo = np.ascontiguousarray(ics)
    res = np.empty((300, 11, 6))
    err = np.zeros(300, np.int32)
    pti = np.ascontiguousarray(pt, np.int32)
    pad = np.ascontiguousarray(pa, np.float64)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    rc = _lib.lib().integrateFullOrbit_cuda(
        300, yo.ctypes.data_as(dp), 11, t.ctypes.data_as(dp), 0, 3, pti.ctypes.data_as(ip),
        pad.ctypes.data_as(dp), None, -9999.99, -27.6, -27.6, res.ctypes.data_as(dp),
        err.ctypes.data_as(ip), 6, cb, None)
    assert rc == 0 and len(calls) == 300


def test_energy_conservation_gpu(oracle, mw14):
    """galpy's energy criterion (tests/test_orbit.py:111) on GPU output."""
    pt, pa = mw14
    ics = seeded_ics(64, 41)
    t = np.linspace(0, 14, 501)
    for m in METHODS:
        out, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, cuda(m), progressbar=False)
        E = oracle.energy_cyl(out, pt, pa)
        assert np.all((E.std(1) / E.mean(1)) ** 2 < 1e-10), m


def test_energy_kernel_vs_oracle(oracle, mw14):
    import torch

    pt, pa = mw14
    ics = seeded_ics(5000, 50, r_range=(0.05, 3.0), log_r=True)
    comps, n = gb.compile_potential((pt, pa))
    dev = torch.device("cuda:0")
    w = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    E = torch.empty(len(ics), dtype=torch.float64, device=dev)
    gb.energy_device(torch.tensor(comps, device=dev), n, w, E)
    torch.cuda.synchronize()
    ref = oracle.energy_cyl(ics[:, None, :], pt, pa)[:, 0]
    # absolute on the scale of the energies (some orbits have E close to 0)
    assert (np.abs(E.cpu().numpy() - ref) / np.abs(ref).max()).max() < 1e-14


@pytest.mark.parametrize("planar", [False, True])
def test_jacobi_kernel_vs_oracle(oracle, mw14, mw14_planar, planar):
    """galpy_cuda_jacobi_device: E - Omega . L (galpy's Orbit.Jacobi,
    Orbits.py:3298-3375) against the oracle's energies and the angular
    momentum from the same states, for a scalar pattern speed and a
    pattern-speed vector; Omega = 0 gives galpy_cuda_energy_device's E."""
    import torch

    from galpy_b200.orbit_quantities import jacobi_device

    pt, pa = mw14_planar if planar else mw14
    ics = seeded_ics(4000, 52, planar=planar)
    comps, n = gb.compile_potential((pt, pa), planar=planar)
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    w_np = cyl_to_rect(ics)
    w = torch.tensor(w_np.T.copy(), device=dev)
    if planar:
        x, y, vx, vy = w_np.T
        L = np.stack([np.zeros_like(x), np.zeros_like(x), x * vy - y * vx], 1)
        # the planar potential is the 3D one in the plane z = 0
        rows = np.insert(np.insert(ics, 3, 0.0, 1), 4, 0.0, 1)
        Eref = oracle.energy_cyl(rows[:, None], *mw14)[:, 0]
    else:
        L = np.cross(w_np[:, :3], w_np[:, 3:])
        Eref = oracle.energy_cyl(ics[:, None, :], pt, pa)[:, 0]
    E0 = torch.empty(len(ics), dtype=torch.float64, device=dev)
    if not planar:
        gb.energy_device(cd, n, w, E0)
    for omega in (0.0, 0.55, (0.1, -0.2, 0.7)):
        J = torch.empty(len(ics), dtype=torch.float64, device=dev)
        jacobi_device(cd, n, w, J, omega=omega, planar=planar)
        torch.cuda.synchronize()
        om = np.array([0.0, 0.0, omega]) if np.ndim(omega) == 0 else np.array(omega)
        if planar:
            om[:2] = 0.0  # planar states: only the z component acts
        ref = Eref - L @ om
        assert (np.abs(J.cpu().numpy() - ref) / np.abs(ref).max()).max() < 1e-14, omega
        if omega == 0.0 and not planar:
            assert torch.equal(J, E0)


@pytest.mark.parametrize("name", ["mw14", "hernquist", "loghalo", "logtri", "nfw", "mn", "pswc"]
                         + ADDED_POTS)
@pytest.mark.parametrize("planar", [False, True])
def test_device_accelerations(golden, harness, name, planar):
    """The kernels' force code on the device (branch-free FP64 helpers:
    hardware-seeded 1/sqrt and 1/x with a Newton correction, binade tables
    for the bulge power and the NFW log1p) against the same code built for
    the host with libm's 1/sqrt and division: a few ulp of the inputs, which
    the NFW force's cancellation at r << a amplifies (by 2a/r; 1e-12 is the
    tolerance of the host build against the reference's formulas too)."""
    import torch

    pt, pa = golden_pot(golden, name, planar)
    pa = np.array(pa, float)
    if planar and int(pt[0]) == 15:
        pa = pa[:3]
    if planar and name == "mw14":
        pt, pa = golden["mw14_planar_type"], np.array(golden["mw14_planar_args"], float)
    rng = np.random.default_rng(3)
    n = 4096
    R = np.exp(rng.uniform(np.log(0.01), np.log(50.0), n))
    phi = rng.uniform(0, 2 * np.pi, n)
    x, y, z = R * np.cos(phi), R * np.sin(phi), rng.normal(0, 0.3, n)
    acc_h, _, acc32_h = harness.forces(x, y, z, pt, pa, planar=planar)
    comps, nc = gb.compile_potential((pt, pa), planar=planar)
    dev = torch.device("cuda:0")
    pos = torch.tensor(np.stack([x, y, z]), device=dev)
    for sig in {0, gb.signature((pt, pa), planar=planar)}:
        for prec, ref, tol in (("fp64", acc_h, 1e-12), ("f32force", acc32_h, 1e-3)):
            acc = torch.empty((3, n), dtype=torch.float64, device=dev)
            gb.accel_device(torch.tensor(comps, device=dev), nc, pos, acc, planar=planar,
                            signature=sig, precision=prec)
            got = acc.cpu().numpy().T
            if planar:
                got, ref_ = got[:, :2], ref[:, :2]
            else:
                ref_ = ref
            if name == "null":
                assert not got.any()
                continue
            scale = np.linalg.norm(ref_, axis=1)
            err = np.abs(got - ref_).max(axis=1) / scale
            if name in ("pseudoiso", "burkert", "exptruncnfw"):
                # these forces cancel terms at r << a (1 - atan(x)/x;
                # 2 atan x - 2 ln(1+x) - ln(1+x^2) ~ -4x^3/3; ExpTruncNFW's
                # F(r) ~ r^2 / (2 a^2) from O(1) terms above its series
                # threshold), in the reference's formulas as here: compare
                # where x = r/a > 0.1 (0.5 in single precision)
                xr = np.sqrt(x**2 + y**2 + (0 if planar else z**2)) / float(pa[1])
                err = err[xr > (0.1 if prec == "fp64" else 0.5)]
            assert err.max() < tol, (sig, prec, err.max())
