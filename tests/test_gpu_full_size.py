"""The benchmark workloads at their full sizes on a B200, through
size-independent properties (the oracle cannot integrate millions of
orbits in a test): every orbit finishes without error, energy is conserved
to the integrator's tolerance, the FP32-force form stays close to the FP64
form, parameter groups behave like single-potential launches, and the
work-queue order does not change any result."""
import numpy as np
import pytest

import bench
import galpy_b200 as gb
from galpy_b200 import _lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "no CUDA device: GPU tests need a GPU"


def _energy_drift(comps, nc, w0, wT, group=None):
    E0 = torch.empty(w0.shape[1], dtype=torch.float64, device=w0.device)
    E1 = torch.empty_like(E0)
    gb.energy_device(comps, nc, w0, E0, group=group)
    gb.energy_device(comps, nc, wT, E1, group=group)
    return torch.abs(E1 / E0 - 1).cpu().numpy()


def test_batching_workload_full_size():
    """1,048,576 orbits, DOP853 rtol = atol = 1e-10, ragged end times, 101
    snapshots; the longest-first and in-order queues give identical results."""
    pt, pa = bench.mw14_args()
    ics, t = bench.workload(bench.N_ORBITS, seed=1)
    comps, nc = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    w0 = torch.tensor(bench.cyl_to_rect(ics).T.copy(), device=dev)
    td = torch.tensor(t, device=dev)
    outs = {}
    for schedule in ("longest_first", "in_order"):
        out = torch.empty((6, 2, len(ics)), dtype=torch.float64, device=dev)
        err = torch.empty(len(ics), dtype=torch.int32, device=dev)
        ns = torch.empty(len(ics), dtype=torch.int64, device=dev)
        # rows 99 and 100 only (out_row0 = nt - 2) keep the buffers small
        gb.integrate_device(cd, nc, w0, td, out, err, "dop853_cuda", nsteps=ns,
                            out_row0=bench.NT - 2, rtol=1e-10, atol=1e-10, signature=sig,
                            comps_host=comps, schedule=schedule)
        torch.cuda.synchronize()
        assert not err.any()
        outs[schedule] = (out, ns)
    assert torch.equal(outs["longest_first"][0], outs["in_order"][0])
    assert torch.equal(outs["longest_first"][1], outs["in_order"][1])
    out, ns = outs["longest_first"]
    assert int(ns.sum()) > 1.2e9  # ~1.3e9 accepted steps
    drift = _energy_drift(cd, nc, w0, out[:, 1, :].contiguous())
    assert np.median(drift) < 1e-8 and np.quantile(drift, 0.99) < 1e-7, (
        np.median(drift), np.quantile(drift, 0.99))


def test_precision_workload_full_size():
    """4,194,304 orbits, symplec4 dt = 0.01, 20,000 steps: FP64 energy
    drift, and the FP32-force form against it."""
    pt, pa = bench.mw14_args()
    ics, t = bench.precision_workload(1 << 22)
    comps, nc = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    w0 = torch.tensor(bench.cyl_to_rect(ics).T.copy(), device=dev)
    td = torch.tensor(t, device=dev)
    res = {}
    for prec in ("fp64", "f32force"):
        out = torch.empty((6, 1, len(ics)), dtype=torch.float64, device=dev)
        err = torch.empty(len(ics), dtype=torch.int32, device=dev)
        gb.integrate_device(cd, nc, w0, td, out, err, "symplec4_cuda", dt=0.01, out_row0=1,
                            precision=prec, signature=sig, comps_host=comps)
        torch.cuda.synchronize()
        assert not err.any()
        res[prec] = out[:, 0, :].contiguous()
    d64 = _energy_drift(cd, nc, w0, res["fp64"])
    d32 = _energy_drift(cd, nc, w0, res["f32force"])
    assert np.median(d64) < 1e-10 and np.quantile(d64, 0.99) < 1e-8
    assert np.median(d32) < 1e-6 and np.quantile(d32, 0.99) < 1e-5
    rel = (torch.abs(res["f32force"] - res["fp64"]).max(dim=0).values
           / torch.abs(res["fp64"]).max(dim=0).values).cpu().numpy()
    assert np.median(rel) < 1e-4


def test_ragged_workload_full_size():
    """512 parameter groups (about 4.3 M orbits) in one launch: energy
    conservation per orbit, and a group's orbits integrated alone give the
    same result as inside the ragged launch."""
    pt, args, group, ics, t = bench.ragged_workload()
    comps, nc = gb.compile_potential((pt, args.ravel()), ngroup=len(args))
    sig = gb.signature((pt, args[0]))
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    w0 = torch.tensor(bench.cyl_to_rect(ics).T.copy(), device=dev)
    td = torch.tensor(t, device=dev)
    gd = torch.tensor(group, device=dev)
    out = torch.empty((6, 1, len(ics)), dtype=torch.float64, device=dev)
    err = torch.empty(len(ics), dtype=torch.int32, device=dev)
    gb.integrate_device(cd, nc, w0, td, out, err, "dop853_cuda", group=gd, out_row0=len(t) - 1,
                        rtol=1e-9, atol=1e-9, signature=sig)
    torch.cuda.synchronize()
    assert not err.any()
    drift = _energy_drift(cd, nc, w0, out[:, 0, :].contiguous(), group=gd)
    assert np.median(drift) < 1e-7 and np.quantile(drift, 0.99) < 1e-6
    for g in (0, 511):
        sel = torch.tensor(np.nonzero(group == g)[0], device=dev)
        c1, n1 = gb.compile_potential((pt, args[g]))
        o1 = torch.empty((6, 1, len(sel)), dtype=torch.float64, device=dev)
        e1 = torch.empty(len(sel), dtype=torch.int32, device=dev)
        gb.integrate_device(torch.tensor(c1, device=dev), n1, w0[:, sel].contiguous(), td, o1,
                            e1, "dop853_cuda", out_row0=len(t) - 1, rtol=1e-9, atol=1e-9,
                            signature=sig)
        torch.cuda.synchronize()
        assert torch.equal(o1[:, 0, :], out[:, 0, sel])
