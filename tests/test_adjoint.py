"""Reverse-mode gradients of DOP853 orbit integration, checked on the CPU by
running the engine's device code (galpy_b200/csrc/adjoint.cuh) as host C++
(tests/harness):

* analytic parameter derivatives of the forces against finite differences of
  the forces;
* the forward pass against the oracle's DOP853 (same step sequence as the
  reference's dop853_c);
* dL/dw0 and dL/dtheta against central finite differences (h = 1e-6) of the
  forward map with the step sizes frozen at the recorded ones (the map the
  discrete adjoint differentiates exactly);
* dL/dw0 against M^T dL/dy(T) with M from the reference's own variational
  DOP853 (integrate{Planar,Full}Orbit_dxdv, golden fixtures), which picks
  its own steps: agreement to the integration tolerance.
"""
import ctypes

import numpy as np
import pytest

from helpers import adj_param_index, central_fd, cyl_to_rect, seeded_ics

POTS = ["mw14", "hernquist", "loghalo", "logtri", "nfw", "mn", "pswc"]


@pytest.mark.parametrize("name", POTS)
@pytest.mark.parametrize("planar", [False, True])
def test_param_derivatives_match_force_differences(harness, golden, name, planar):
    pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
    if planar:  # planar PowerSphericalwCutoff carries 3 args, not 5
        _, pt2, pa2 = _planar_args(golden, name)
        pt, pa = pt2, pa2
    rng = np.random.default_rng(1)
    n = 32
    x, y = rng.uniform(-2, 2, n), rng.uniform(-2, 2, n)
    z = rng.normal(0, 0.3, n)
    lam = rng.normal(size=(n, 3))
    if planar:
        lam[:, 2] = 0.0
    g = harness.adj_param_vjp(x, y, z, lam, pt, pa, planar=planar)
    idx = adj_param_index(pt, planar)
    assert g.shape == (n, len(idx))

    def acc(p):
        return (harness.forces(x, y, z, pt, p, planar=planar)[0] * lam).sum(1)

    fd = central_fd(acc, np.array(pa, float), idx).T
    scale = np.abs(fd).max(0)
    assert np.all(np.abs(g - fd) <= 1e-7 * scale + 1e-12), np.abs(g - fd).max(0) / scale


def _planar_args(golden, name):
    """(npot, pot_type, pot_args) of the planar form of a golden potential."""
    if name == "mw14":
        return 3, golden["mw14_planar_type"], golden["mw14_planar_args"]
    pt, pa = golden[f"{name}_type"], golden[f"{name}_args"]
    if int(pt[0]) == 15:  # drop the two cache slots of the 3D argument list
        pa = pa[:3]
    return len(pt), pt, pa


def _case(golden, planar, n=4, seed=11):
    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    w0 = cyl_to_rect(seeded_ics(n, seed, planar=planar))
    return pt, np.array(pa, float), np.ascontiguousarray(w0)


@pytest.mark.parametrize("planar", [True, False])
def test_forward_matches_oracle_dop853(harness, oracle, golden, planar):
    pt, pa, w0 = _case(golden, planar)
    ics = seeded_ics(4, 11, planar=planar)
    T = 20.0
    yT, ns, err, _ = harness.adj_forward(w0, 0.0, T, pt, pa, planar=planar)
    assert not err.any() and (ns > 10).all()
    res, oerr, _, _ = oracle.integrate(ics, np.array([0.0, T]), pt, pa, "dop853", planar=planar,
                                       rtol=1e-10, atol=1e-10)
    assert not oerr.any()
    np.testing.assert_allclose(yT, cyl_to_rect(res[:, -1]), rtol=0, atol=1e-11)
    # the same map with the recorded steps frozen is bit-identical
    _, _, _, h = harness.adj_forward(w0, 0.0, T, pt, pa, planar=planar)
    assert np.array_equal(harness.adj_replay(w0, 0.0, T, pt, pa, h, ns, planar=planar), yT)


def test_zero_length_interval(harness, golden):
    pt, pa, w0 = _case(golden, True, n=2)
    yT, ns, err, _ = harness.adj_forward(w0, 3.0, 3.0, pt, pa, planar=True)
    assert np.array_equal(yT, w0) and not ns.any() and not err.any()
    g = np.ones_like(w0)
    gw, gth, err = harness.adj_gradient(w0, 3.0, 3.0, pt, pa, g, planar=True)
    assert np.array_equal(gw, g) and not gth.any()


@pytest.mark.parametrize("planar", [True, False])
@pytest.mark.parametrize("backward_in_time", [False, True])
def test_gradients_match_frozen_step_differences(harness, golden, planar, backward_in_time):
    pt, pa, w0 = _case(golden, planar)
    t0, T = (20.0, 0.0) if backward_in_time else (0.0, 20.0)
    yT, ns, err, h = harness.adj_forward(w0, t0, T, pt, pa, planar=planar)
    assert not err.any()
    tgt = np.random.default_rng(3).normal(size=yT.shape)

    def loss(w, p):
        y = harness.adj_replay(w, t0, T, pt, p, h, ns, planar=planar)
        return ((y - tgt) ** 2).sum(1)  # per orbit

    gw, gth, err = harness.adj_gradient(w0, t0, T, pt, pa, 2 * (yT - tgt), planar=planar)
    assert not err.any()
    nv = w0.shape[1]
    fdw = np.stack([central_fd(lambda v: loss(np.where(np.arange(nv) == c, v[:, None], w0), pa),
                               w0[:, c].copy(), range(len(w0)), floor=1.0).diagonal()
                    for c in range(nv)], 1)
    np.testing.assert_allclose(gw, fdw, rtol=1e-6, atol=1e-6 * np.abs(fdw).max())
    idx = adj_param_index(pt, planar)
    fdt = central_fd(lambda p: loss(w0, p), pa, idx).T
    np.testing.assert_allclose(gth, fdt, rtol=1e-6, atol=1e-6 * np.abs(fdt).max())


@pytest.mark.parametrize("name", ["hernquist", "logtri", "nfw"])
def test_gradients_other_potentials(harness, golden, name):
    pt, pa = golden[f"{name}_type"], np.array(golden[f"{name}_args"], float)
    w0 = cyl_to_rect(seeded_ics(3, 5))
    T = 10.0
    yT, ns, err, h = harness.adj_forward(w0, 0.0, T, pt, pa)
    assert not err.any()
    gw, gth, _ = harness.adj_gradient(w0, 0.0, T, pt, pa, np.ones_like(yT))

    def loss(p):
        return harness.adj_replay(w0, 0.0, T, pt, p, h, ns).sum(1)

    fdt = central_fd(loss, pa, adj_param_index(pt, False)).T
    np.testing.assert_allclose(gth, fdt, rtol=1e-6, atol=1e-6 * np.abs(fdt).max())


@pytest.mark.parametrize("name", ["plummer", "isochrone", "einasto", "flatpower", "dehnen",
                                  "ell_trihern", "ell_perfell", "ell_trigauss"])
def test_ic_gradients_added_potentials(harness, golden, name):
    """The potentials added behind the component template have no
    differentiable parameters; they enter the adjoint through the tidal
    tensor: dL/dw0 against frozen-step central differences.  The ellipsoidal
    ones are aligned: the reference's second derivatives, which the tidal
    tensor follows, ignore any rotation, so for a rotated ellipsoid they are
    not the derivative of its force."""
    pt, pa = golden[f"{name}_type"], np.array(golden[f"{name}_args"], float)
    w0 = cyl_to_rect(seeded_ics(3, 5))
    t0, T = 0.0, 10.0
    yT, ns, err, h = harness.adj_forward(w0, t0, T, pt, pa)
    assert not err.any()
    tgt = np.random.default_rng(4).normal(size=yT.shape)

    def loss(w):
        return ((harness.adj_replay(w, t0, T, pt, pa, h, ns) - tgt) ** 2).sum(1)

    gw, gth, err = harness.adj_gradient(w0, t0, T, pt, pa, 2 * (yT - tgt))
    assert not err.any() and not np.any(gth)
    nv = w0.shape[1]
    fdw = np.stack([central_fd(lambda v: loss(np.where(np.arange(nv) == c, v[:, None], w0)),
                               w0[:, c].copy(), range(len(w0)), floor=1.0).diagonal()
                    for c in range(nv)], 1)
    np.testing.assert_allclose(gw, fdw, rtol=1e-6, atol=1e-6 * np.abs(fdw).max())


@pytest.mark.parametrize("planar", [True, False])
def test_ic_gradient_matches_reference_variational(harness, golden, planar):
    key = "adj_planar" if planar else "adj_3d"
    w0, jac, yref = golden[f"{key}_w0"], golden[f"{key}_jac"], golden[f"{key}_yT"]
    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    yT, ns, err, _ = harness.adj_forward(w0, 0.0, 20.0, pt, pa, planar=planar)
    # the variational run picks its own steps (error norm over 2*nv values)
    np.testing.assert_allclose(yT, yref, rtol=0, atol=1e-7)
    tgt = np.random.default_rng(9).normal(size=yT.shape)
    gy = 2 * (yT - tgt)
    gw, _, err = harness.adj_gradient(w0, 0.0, 20.0, pt, pa, gy, planar=planar)
    assert not err.any()
    ref = np.einsum("nij,ni->nj", jac, gy)
    np.testing.assert_allclose(gw, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


def test_adjoint_params_abi_matches_layout(golden):
    """galpy_cuda_adjoint_params (host-only; no GPU needed)."""
    from galpy_b200 import _lib
    from galpy_b200.adjoint import adjoint_params

    for planar in (False, True):
        pt = golden["mw14_planar_type"] if planar else golden["mw14_type"]
        np.testing.assert_array_equal(adjoint_params(pt, planar), adj_param_index(pt, planar))
    lib = _lib.lib()
    bad = np.array([15, 99], np.int32)
    assert lib.galpy_cuda_adjoint_params(0, 2, bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                         None, None) == _lib.ERR_POTENTIAL
    # an ellipsoidal component ahead of a Miyamoto-Nagai disk: its argument
    # count comes from its arguments (none of its own are differentiable)
    pte, pae = golden["ell_trihern_type"], golden["ell_trihern_args"]
    pt = np.concatenate([pte, golden["mn_type"]]).astype(np.int32)
    pa = np.concatenate([pae, golden["mn_args"]])
    np.testing.assert_array_equal(adjoint_params(pt, False, pa), len(pae) + np.arange(3))
    with pytest.raises(_lib.PotentialNotSupported):
        adjoint_params(pt, False)
    # a rotated ellipsoid has no consistent second derivatives: refused
    with pytest.raises(_lib.PotentialNotSupported, match="rotated"):
        adjoint_params(golden["ell_trinfw_type"], False, golden["ell_trinfw_args"])


def test_adjoint_refuses_bar_and_scf():
    """The adjoint's forward pass evaluates static forces, and the device has
    no tidal tensor of an SCF expansion: both potentials are refused."""
    import timedep_pots as TP

    from galpy_b200 import _lib
    from galpy_b200.adjoint import adjoint_params

    for name in ("bar+mw14", "scf_axi+mn"):
        pt, pa = TP.potential(name, planar=True)
        with pytest.raises(_lib.PotentialNotSupported, match="time-dependent or SCF"):
            adjoint_params(pt, True, pa)
    for planar in (False, True):  # rotating spiral arms and needle bar
        for pt, pa in (TP.spiral_arms("spiral+mw14", planar), TP.needle_bar("needle+mw14", planar)):
            with pytest.raises(_lib.PotentialNotSupported, match="time-dependent or SCF"):
                adjoint_params(pt, planar, pa)
    pt, pa = TP.planar_perturbation("lopsided+mw14")
    with pytest.raises(_lib.PotentialNotSupported, match="time-dependent or SCF"):
        adjoint_params(pt, True, pa)
