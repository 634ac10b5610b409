"""Interrupting integrations on the GPU (galpy's SIGINT behaviour).

galpy's C integrators poll a process-global flag set by their SIGINT
handler, stop the orbit with err = -10, and the Python wrappers raise
KeyboardInterrupt when any err is -10 (galpy/util/bovy_symplecticode.c:38-54,
galpy/orbit/integrateFullOrbit.py:737-738); the reference tests this by
sending SIGINT to a child process running a long integration
(tests/test_orbit.py:12211-12420).  The engine forwards SIGINT to a device
abort word that the persistent kernel polls every 256 loop iterations.

Nothing here faults or hangs a GPU: the interruption is a host-written flag
(or a signal to a host process), and every kernel ends by itself.
"""
import os
import select
import signal
import subprocess
import sys
import time

import numpy as np
import pytest
from helpers import cyl_to_rect, seeded_ics

pytestmark = pytest.mark.gpu
CHILD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sigint_child.py")


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import _lib, build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "GPU tests need a GPU"


@pytest.mark.parametrize("method", ["dop853", "symplec4"])
def test_device_abort_word(oracle, mw14, method):
    """A set abort word stops every orbit with err -10: the rows an orbit
    wrote before it stopped are the oracle's, every later row is NaN, and
    orbits that had not started are all NaN."""
    import torch

    import galpy_b200 as gb

    pt, pa = mw14
    n = 4096
    ics = seeded_ics(n, 50)
    if method == "dop853":
        # early output times so that some rows are written before the kernel
        # first reads the flag, then a long stretch it never reaches
        t = np.concatenate([np.linspace(0.0, 0.02, 5), [2000.0]])
    else:
        # galpy's fixed-step integrators take evenly spaced output times
        # (the number of steps per output comes from the first interval)
        t = np.linspace(0.0, 2000.0, 6)
    comps, ncomp = gb.compile_potential((pt, pa))
    dev = torch.device("cuda", 0)
    d_comps = torch.from_numpy(comps).to(dev)
    w0 = torch.from_numpy(np.ascontiguousarray(cyl_to_rect(ics).T)).to(dev)
    d_t = torch.from_numpy(t).to(dev)
    out = torch.full((6, len(t), n), 7.0, dtype=torch.float64, device=dev)
    err = torch.zeros(n, dtype=torch.int32, device=dev)
    abort = torch.ones(1, dtype=torch.int32, device=dev)
    gb.integrate_device(d_comps, ncomp, w0, d_t, out, err, method, out_layout="soa_cyl",
                        dt=0.001 if method == "symplec4" else None, abort_flag=abort)
    torch.cuda.synchronize()
    e = err.cpu().numpy()
    rows = out.cpu().numpy().transpose(2, 1, 0)  # [n][nt][6]
    assert (e == -10).all(), np.unique(e)
    fin = np.isfinite(rows).all(axis=2)
    partial = np.isfinite(rows).any(axis=2) & ~fin
    assert not partial.any()  # a row is either written in full or all NaN
    assert not fin[:, -1].any()  # no orbit reached t = 2000
    # the finite rows form a prefix of each orbit ...
    nfin = fin.sum(axis=1)
    assert (fin == (np.arange(len(t))[None, :] < nfin[:, None])).all()
    assert (rows != 7.0).all()  # every row was written
    # ... equal to the oracle's rows (same step sequence up to the stop); the
    # oracle integrates only as far as the last row any orbit wrote (the
    # first row is the initial state)
    k = nfin > 0
    assert k.any()
    assert np.abs(rows[k, 0, :5] - ics[k, :5]).max() < 1e-15
    jmax = int(nfin.max()) - 1
    if jmax >= 1:
        sel_o = nfin > 1
        ref, _, _, _ = oracle.integrate(ics[sel_o], t[:jmax + 1], pt, pa, method,
                                        dt=0.001 if method == "symplec4" else None)
        for j in range(1, jmax + 1):
            sel = fin[sel_o, j]
            if sel.any():
                d = np.abs(rows[sel_o][sel, j, :5] - ref[sel, j, :5]).max()
                assert d < 1e-9, (j, d)


def _wait_line(p, prefix, timeout):
    deadline = time.time() + timeout
    buf = ""
    while time.time() < deadline:
        r, _, _ = select.select([p.stdout], [], [], 1.0)
        if r:
            line = p.stdout.readline()
            if not line:
                return False, buf
            buf += line
            if line.startswith(prefix):
                return True, buf
        if p.poll() is not None:
            return False, buf
    return False, buf


@pytest.mark.parametrize("method,kind,split", [
    ("dop853_cuda", "full", False), ("dop853_cuda", "planar", False),
    ("leapfrog_cuda", "full", False), ("leapfrog_cuda", "planar", False),
    ("dop853_cuda", "full", True)])
def test_sigint_interrupts_blocking_call(method, kind, split):
    """SIGINT during integrateFullOrbit_cuda / integratePlanarOrbit_cuda
    ends the call early with KeyboardInterrupt, as galpy's C integrators do
    -- also when the call spreads its orbits over several ranges, each run
    by its own thread."""
    argv = [sys.executable, CHILD, method, kind] + (["split"] if split else [])
    p = subprocess.Popen(argv, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        ok, log = _wait_line(p, "Starting long integration", 300)
        assert ok, log + (p.stderr.read() if p.poll() is not None else "")
        time.sleep(2.0)
        sent = time.time()
        p.send_signal(signal.SIGINT)
        out, errtxt = p.communicate(timeout=120)
        took = time.time() - sent
    finally:
        if p.poll() is None:
            p.kill()
            p.wait()
    assert p.returncode == 0, (p.returncode, out, errtxt)
    assert "KeyboardInterrupt after" in out, out
    assert took < 30.0, took
