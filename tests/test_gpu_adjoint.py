"""Reverse-mode gradients on a B200 through the C ABI and the autograd
wrapper: the CUDA kernels against the same algorithm compiled for the host
(tests/harness), against central finite differences (h = 1e-6) of the
frozen-step forward map, and against the variational (dxdv) integration.
Tolerance of every gradient check: 1e-6 relative."""
import numpy as np
import pytest
from helpers import (adj_param_index, central_fd, cyl_to_rect, differentiation_workload,
                     seeded_ics)

import galpy_b200 as gb
from galpy_b200 import _lib
from galpy_b200 import adjoint as adj

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "no CUDA device: GPU tests need a GPU"


def _pot(golden, planar):
    if planar:
        return golden["mw14_planar_type"], np.array(golden["mw14_planar_args"], float)
    return golden["mw14_type"], np.array(golden["mw14_args"], float)


def _dev(pt, pa, planar, generic=False):
    buf, n = gb.compile_potential((pt, pa), planar=planar)
    sig = 0 if generic else gb.signature((pt, pa), planar=planar)
    return torch.from_numpy(buf).cuda(), n, sig


def _soa(w):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(w).T)).cuda()


def _run(pt, pa, w0, T, planar, generic=False, gy=None, record=0, rtol=1e-10):
    comps, n, sig = _dev(pt, pa, planar, generic)
    w = _soa(w0)
    f = adj.adjoint_forward(comps, n, w, T, rtol=rtol, atol=rtol, planar=planar, signature=sig,
                            record_steps=record)
    out = {"fwd": f, "comps": comps, "n": n, "sig": sig, "w": w}
    if gy is not None:
        npar = len(adj.adjoint_params(pt, planar))
        gw, gp = adj.adjoint_backward(comps, n, f, _soa(gy), T, rtol=rtol, atol=rtol,
                                      planar=planar, signature=sig, nparam=npar)
        out["gw0"] = gw.cpu().numpy().T
        out["gparam"] = gp.cpu().numpy().T
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("planar", [True, False])
@pytest.mark.parametrize("generic", [False, True])
def test_gpu_adjoint_matches_host_build(harness, golden, planar, generic):
    """The same algorithm built for the host.  The step-size controller
    amplifies rounding (its error norm is a small difference of stage
    sums), so device and host choose step sizes that agree to ~1e-7; with
    the device's steps frozen into the host build, forward map and gradients
    agree to rounding."""
    pt, pa = _pot(golden, planar)
    w0 = cyl_to_rect(seeded_ics(256, 21, planar=planar))
    T = 20.0
    yh, nh, eh, hh = harness.adj_forward(w0, 0.0, T, pt, pa, planar=planar)
    gy = np.random.default_rng(2).normal(size=yh.shape)
    r = _run(pt, pa, w0, T, planar, generic, gy=gy, record=hh.shape[1] + 64)
    f = r["fwd"]
    assert not f["err"].any()
    ns = f["nsteps"].cpu().numpy()
    hd = np.ascontiguousarray(f["hrec"].cpu().numpy().T)
    yT = f["yT"].cpu().numpy().T
    # independent step choices: the same accepted-step counts, and step sizes
    # that differ no more than the host build's own step sizes move under a
    # one-ulp change of the initial conditions (the controller's error norm
    # is a small difference of stage sums: on this workload that response
    # alone is ~2e-8 median, ~6e-7 at the 90th percentile, measured on a
    # B200 together with the device's differences, which match it)
    assert (ns == nh).mean() >= 0.99, (ns == nh).mean()
    ulp = 1 + np.finfo(float).eps * np.random.default_rng(7).choice([-1, 1], w0.shape)
    _, nh1, _, hh1 = harness.adj_forward(w0 * ulp, 0.0, T, pt, pa, planar=planar)

    def step_rel_diff(a, b, n):
        k = min(a.shape[1], b.shape[1])
        used = np.arange(k)[None, :] < n[:, None]
        return np.where(used, np.abs(a[:, :k] - b[:, :k]) / np.abs(b[:, :k]).clip(1e-300),
                        0.0).max(axis=1)

    dev = step_rel_diff(hd, hh, nh)[ns == nh]
    resp = step_rel_diff(hh1, hh, nh)[nh1 == nh]
    for qtl in (0.5, 0.9):
        assert np.quantile(dev, qtl) <= 3 * np.quantile(resp, qtl) + 1e-12, (
            qtl, np.quantile(dev, qtl), np.quantile(resp, qtl))
    np.testing.assert_allclose(yT, yh, rtol=0, atol=1e-8)
    # the device's steps frozen into the host build
    np.testing.assert_allclose(harness.adj_replay(w0, 0.0, T, pt, pa, hd, ns, planar=planar),
                               yT, rtol=0, atol=1e-12)
    gwh, gth = harness.adj_backward_frozen(w0, 0.0, T, pt, pa, hd, ns, gy, planar=planar)
    for dev, host in ((r["gw0"], gwh), (r["gparam"], gth)):
        np.testing.assert_allclose(dev, host, rtol=1e-10, atol=1e-10 * np.abs(host).max())


@pytest.mark.parametrize("planar", [True, False])
def test_gpu_gradients_match_frozen_step_differences(golden, planar):
    pt, pa = _pot(golden, planar)
    w0 = cyl_to_rect(seeded_ics(256, 5, planar=planar))
    T = 20.0
    tgt = np.random.default_rng(4).normal(size=w0.shape)
    r0 = _run(pt, pa, w0, T, planar, record=8192)
    f = r0["fwd"]
    assert not f["err"].any()
    yT = f["yT"].cpu().numpy().T
    r = _run(pt, pa, w0, T, planar, gy=2 * (yT - tgt))
    hrec, ns = f["hrec"], f["nsteps"]

    def loss(w, p):  # per orbit, steps frozen at the recorded ones
        comps, n, sig = _dev(pt, p, planar)
        y = adj.adjoint_replay(comps, n, _soa(w), hrec, ns, T, planar=planar, signature=sig)
        return ((y.cpu().numpy().T - tgt) ** 2).sum(1)

    nv = w0.shape[1]
    h = 1e-6
    fdw = np.zeros_like(w0)
    for c in range(nv):  # orbits are independent: one perturbation per component
        wp, wm = w0.copy(), w0.copy()
        wp[:, c] += h
        wm[:, c] -= h
        fdw[:, c] = (loss(wp, pa) - loss(wm, pa)) / (2 * h)
    np.testing.assert_allclose(r["gw0"], fdw, rtol=1e-6, atol=1e-6 * np.abs(fdw).max())
    fdt = central_fd(lambda p: loss(w0, p).sum(), pa, adj_param_index(pt, planar))
    np.testing.assert_allclose(r["gparam"].sum(0), fdt, rtol=1e-6)


@pytest.mark.parametrize("planar", [True, False])
def test_gpu_ic_gradient_matches_variational(golden, planar):
    """dL/dw0 = M^T dL/dy(T) with M from the batched variational DOP853."""
    pt, pa = _pot(golden, planar)
    nv = 4 if planar else 6
    w0 = cyl_to_rect(seeded_ics(32, 6, planar=planar))
    T = 20.0
    w = np.zeros((len(w0) * nv, 2 * nv))
    for c in range(nv):
        w[c::nv, :nv] = w0
        w[c::nv, nv + c] = 1.0
    res, err = gb.integrate_dxdv_batch((pt, pa), w, np.array([0.0, T]), "dop853_cuda",
                                       planar=planar, rtol=1e-10, atol=1e-10)
    assert not err.any()
    M = res[:, -1, nv:].reshape(len(w0), nv, nv).transpose(0, 2, 1)  # M[i][row][col]
    tgt = np.random.default_rng(8).normal(size=w0.shape)
    r0 = _run(pt, pa, w0, T, planar)
    yT = r0["fwd"]["yT"].cpu().numpy().T
    gy = 2 * (yT - tgt)
    r = _run(pt, pa, w0, T, planar, gy=gy)
    ref = np.einsum("nij,ni->nj", M, gy)
    np.testing.assert_allclose(r["gw0"], ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max())


def test_autograd_final_state(golden):
    pt, pa = _pot(golden, True)
    w0, tgt = differentiation_workload(128)
    w = torch.tensor(w0, dtype=torch.float64, device="cuda", requires_grad=True)
    p = torch.tensor(pa, dtype=torch.float64, requires_grad=True)
    yT = adj.final_state(w, (pt, p), tend=20.0, rtol=1e-10, atol=1e-10, planar=True)
    loss = ((yT - torch.from_numpy(tgt).cuda()) ** 2).sum()
    loss.backward()
    gy = 2 * (yT.detach().cpu().numpy() - tgt)
    r = _run(pt, pa, w0, 20.0, True, gy=gy)
    np.testing.assert_allclose(w.grad.cpu().numpy(), r["gw0"], rtol=1e-12, atol=1e-14)
    idx = adj_param_index(pt, True)
    expect = np.zeros_like(pa)
    np.add.at(expect, idx, r["gparam"].sum(0))
    np.testing.assert_allclose(p.grad.numpy(), expect, rtol=1e-10, atol=0)
    assert p.grad.numpy()[np.setdiff1d(np.arange(len(pa)), idx)].tolist() == [0.0] * (
        len(pa) - len(idx))


def test_differentiation_workload_full_size(golden):
    """65,536 planar orbits, t in [0, 20], rtol = atol = 1e-10: the full
    gradient workload through the autograd wrapper; the parameter gradient
    of the total loss and the per-orbit initial-condition gradients against
    central differences of the frozen-step map over the whole batch."""
    pt, pa = _pot(golden, True)
    w0, tgt = differentiation_workload(65536)
    w = torch.tensor(w0, dtype=torch.float64, device="cuda", requires_grad=True)
    p = torch.tensor(pa, dtype=torch.float64, requires_grad=True)
    yT = adj.final_state(w, (pt, p), tend=20.0, rtol=1e-10, atol=1e-10, planar=True)
    ((yT - torch.from_numpy(tgt).cuda()) ** 2).sum().backward()
    gw = w.grad.cpu().numpy()
    assert np.isfinite(gw).all() and np.isfinite(p.grad.numpy()).all()
    r0 = _run(pt, pa, w0, 20.0, True, record=4096)
    f = r0["fwd"]
    assert not f["err"].any()
    hrec, ns = f["hrec"], f["nsteps"]

    def loss(w_, p_):
        comps, n, sig = _dev(pt, p_, True)
        y = adj.adjoint_replay(comps, n, _soa(w_), hrec, ns, 20.0, planar=True, signature=sig)
        return ((y.cpu().numpy().T - tgt) ** 2).sum(1)

    h = 1e-6
    for c in range(4):
        wp, wm = w0.copy(), w0.copy()
        wp[:, c] += h
        wm[:, c] -= h
        fd = (loss(wp, pa) - loss(wm, pa)) / (2 * h)
        np.testing.assert_allclose(gw[:, c], fd, rtol=1e-6, atol=1e-6 * np.abs(fd).max())
    idx = adj_param_index(pt, True)
    fdt = central_fd(lambda q: loss(w0, q).sum(), pa, idx)
    np.testing.assert_allclose(p.grad.numpy()[idx], fdt, rtol=1e-6)
