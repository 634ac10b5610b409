"""galpy_cuda_integrate_device_noalloc: the entry point for callers that must
not let a library allocate GPU memory while they integrate -- for example an
application that runs the integrator inside a loop where an allocation would
synchronise the device, or that has sized and locked its memory pool for its
own buffers.  It keeps its scratch (work counter, abort word, work queue) in a
fixed array compiled into the library instead of allocating it per call.

This file is collected last on purpose (test_zz_*): a failure here must not
hide the results of the other GPU tests.  It runs on its own in a fresh
process as well as after them."""
import ctypes

import numpy as np
import pytest

from galpy_b200 import _lib

pytestmark = pytest.mark.gpu

NOALLOC_MAX_ORBITS = 1 << 20


def _workload(n, seed=7):
    rng = np.random.default_rng(seed)
    R = np.exp(rng.uniform(np.log(0.05), np.log(3.0), n))
    phi = rng.uniform(0, 2 * np.pi, n)
    vR, vT = rng.normal(0, 0.1, n), 1 + rng.normal(0, 0.1, n)
    z, vz = rng.normal(0, 0.05, n), rng.normal(0, 0.05, n)
    c, s = np.cos(phi), np.sin(phi)
    w = np.stack([R * c, R * s, z, vR * c - vT * s, vR * s + vT * c, vz])
    tend = np.exp(rng.normal(np.log(5.0), 0.5, n))
    t = np.linspace(0, 1, 21)[None, :] * tend[:, None]
    return w, t


def _launch(comps, ncomp, w0, t, out, err, nsteps, signature, schedule):
    import torch

    L = _lib.GalpyCudaLaunch()
    L.planar, L.variational, L.odeint_type, L.precision = 0, 0, 6, _lib.FP64
    L.nobj, L.nt, L.indiv_t = err.shape[0], t.shape[-1], 1
    L.t, L.w0, L.in_layout = t.data_ptr(), w0.data_ptr(), _lib.IN_SOA
    L.out, L.out_layout, L.out_row0 = out.data_ptr(), _lib.OUT_SOA_RECT, 0
    L.err, L.nsteps = err.data_ptr(), nsteps.data_ptr()
    L.comps, L.ncomp, L.group = comps.data_ptr(), ncomp, None
    L.dt, L.rtol, L.atol = _lib.DT_SENTINEL, float(np.log(1e-10)), float(np.log(1e-10))
    L.max_attempts, L.abort_flag = 0, None
    L.stream = torch.cuda.current_stream().cuda_stream
    L.block_size = L.grid_size = 0
    L.signature, L.schedule, L.variant = signature, schedule, 0
    return L


@pytest.mark.parametrize("schedule", [1, 0])  # longest-first, in order
def test_noalloc_matches_allocating_entry_point(schedule):
    import torch

    import galpy_b200 as gb
    from galpy_b200 import build

    build.build()
    lib = _lib.lib()
    assert lib.galpy_cuda_device_count() > 0
    pot = gb.MWPotential2014()
    comps_np, ncomp = gb.compile_potential(pot)
    sig = gb.signature(pot)
    dev = torch.device("cuda:0")
    n = 20000
    w_np, t_np = _workload(n)
    comps = torch.tensor(comps_np, device=dev)
    w0 = torch.tensor(w_np, device=dev)
    t = torch.tensor(t_np, device=dev)

    def buffers():
        return (torch.full((6, 21, n), float("nan"), dtype=torch.float64, device=dev),
                torch.full((n,), -99, dtype=torch.int32, device=dev),
                torch.full((n,), -1, dtype=torch.int64, device=dev))

    ref_out, ref_err, ref_ns = buffers()
    L = _launch(comps, ncomp, w0, t, ref_out, ref_err, ref_ns, sig, schedule)
    assert lib.galpy_cuda_integrate_device(ctypes.byref(L)) == 0
    torch.cuda.synchronize()
    assert (ref_err == 0).all()

    for call in range(2):  # two calls in a row share the fixed scratch
        out, err, ns = buffers()
        L = _launch(comps, ncomp, w0, t, out, err, ns, sig, schedule)
        rc = lib.galpy_cuda_integrate_device_noalloc(ctypes.byref(L))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(err, ref_err), call
        assert torch.equal(ns, ref_ns), call
        # same kernel on the same inputs: the orbits are independent of the
        # order they were scheduled in, so the tolerance is the device-API one
        diff = (out - ref_out).abs().max().item()
        assert diff <= 1e-14, (call, diff)


@pytest.mark.parametrize("case", ["planar_aos", "variational_aos"])
def test_noalloc_other_layouts(case):
    """The bucketed work queue reads the initial positions of planar rows
    (4 values) and of variational rows (12 values) laid out as AoS: both
    calls must give the allocating entry point's results bit for bit."""
    import torch

    import galpy_b200 as gb
    from galpy_b200 import build

    build.build()
    lib = _lib.lib()
    planar = case == "planar_aos"
    var = case == "variational_aos"
    pot = gb.MWPotential2014()
    comps_np, ncomp = gb.compile_potential(pot, planar=planar)
    sig = gb.signature(pot, planar=planar)
    dev = torch.device("cuda:0")
    n = 6000
    w3, t_np = _workload(n, seed=11)
    if planar:
        w = np.stack([w3[0], w3[1], w3[3], w3[4]], 1)  # [n][4] rectangular
    else:
        w = np.zeros((n, 12))
        w[:, :6] = w3.T
        w[np.arange(n), 6 + np.arange(n) % 6] = 1.0  # one unit deviation per orbit
    nv = w.shape[1]
    comps = torch.tensor(comps_np, device=dev)
    w0 = torch.tensor(np.ascontiguousarray(w), device=dev)
    t = torch.tensor(t_np, device=dev)
    method = 3 if var else 6  # variational symplec4 (tangent kicks) / dop853

    def run(entry):
        out = torch.full((nv, 21, n), float("nan"), dtype=torch.float64, device=dev)
        err = torch.full((n,), -99, dtype=torch.int32, device=dev)
        ns = torch.full((n,), -1, dtype=torch.int64, device=dev)
        L = _launch(comps, ncomp, w0, t, out, err, ns, sig, 1)
        L.planar, L.variational, L.odeint_type = int(planar), int(var), method
        L.in_layout = _lib.IN_AOS
        if var:
            L.signature = 0
            L.dt = 0.01
        rc = entry(ctypes.byref(L))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        return out, err, ns

    ref_out, ref_err, ref_ns = run(lib.galpy_cuda_integrate_device)
    assert (ref_err == 0).all()
    for call in range(2):
        out, err, ns = run(lib.galpy_cuda_integrate_device_noalloc)
        assert torch.equal(err, ref_err) and torch.equal(ns, ref_ns), call
        diff = (out - ref_out).abs().max().item()
        assert diff <= 1e-14, (call, diff)


def test_noalloc_rejects_oversized_batch():
    import torch

    lib = _lib.lib()
    dev = torch.device("cuda:0")
    tiny = torch.zeros(16, dtype=torch.float64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    L = _lib.GalpyCudaLaunch()
    L.odeint_type, L.precision = 6, _lib.FP64
    L.nobj, L.nt = NOALLOC_MAX_ORBITS + 1, 2
    L.t = L.w0 = L.out = L.comps = tiny.data_ptr()
    L.err = err.data_ptr()
    L.ncomp = 1
    rc = lib.galpy_cuda_integrate_device_noalloc(ctypes.byref(L))
    assert rc == _lib.ERR_ARG
    assert "exceeds" in _lib.last_error()
