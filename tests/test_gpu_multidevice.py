"""One blocking call spread over several devices (galpy_cuda_opts.ndevices).

The call cuts its orbits into contiguous ranges of equal estimated cost and
integrates each range on its own thread and device, writing straight into
the caller's arrays.  With one GPU the ranges go to the same device
(devices=[0, 0, ...]: repeated ordinals run concurrently there), which runs
every part of the split path -- the cut, the per-range slices of states,
times and result rows, the per-range threads, progress, elapsed time and
error collection -- and must give the one-device result bit for bit.  The
results of an orbit do not depend on which launch integrates it."""
import numpy as np
import pytest
from helpers import seeded_ics

import galpy_b200 as gb
from galpy_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "GPU tests need a GPU"


def _sorted_ics(n, seed, planar=False):
    ics = seeded_ics(n, seed, planar=planar, r_range=(0.05, 20.0), log_r=True)
    return ics[np.argsort(ics[:, 0])]


@pytest.mark.parametrize("method", ["dop853_cuda", "symplec4_cuda", "rk6_cuda"])
@pytest.mark.parametrize("planar", [False, True])
def test_split_equals_one_device(golden, method, planar):
    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    n = 5003
    ics = _sorted_ics(n, 70, planar=planar)
    rng = np.random.default_rng(70)
    if method == "dop853_cuda":
        t = np.linspace(0, 1, 21)[None, :] * np.exp(rng.normal(np.log(20.0), 0.5, n))[:, None]
    else:
        t = np.linspace(0, 20, 21)
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    o1, e1, n1 = fn((pt, pa), ics.copy(), t, method, progressbar=False, return_nsteps=True,
                    rtol=1e-10, atol=1e-10)
    o3, e3, n3 = fn((pt, pa), ics.copy(), t, method, progressbar=False, return_nsteps=True,
                    rtol=1e-10, atol=1e-10, devices=[0, 0, 0])
    assert not e1.any()
    assert np.array_equal(e1, e3) and np.array_equal(n1, n3)
    assert np.array_equal(o1, o3)


def test_split_progress_elapsed_and_streaming(golden):
    """The progress callback sees every orbit once; elapsed_ms is the
    slowest range's; streamed rows (each range streams its own) land in the
    right rows of the caller's array."""
    import ctypes

    pt = np.ascontiguousarray(golden["mw14_type"], np.int32)
    pa = np.ascontiguousarray(golden["mw14_args"], np.float64)
    n = 3 * 4096 + 77
    ics = _sorted_ics(n, 71)
    t = np.ascontiguousarray(np.linspace(0, 5, 31))
    ref, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "dop853_cuda",
                                          progressbar=False)
    calls = [0]

    def tick():
        calls[0] += 1

    cb = _lib.CALLBACK(tick)
    res = np.full((n, len(t), 6), np.nan)
    yo = np.ascontiguousarray(ics.copy())
    er = np.zeros(n, np.int32)
    ms = ctypes.c_double(-1.0)
    opts = _lib.make_opts(elapsed=ms, stream_rows=1, devices=[0, 0])
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lr, la = gb.parse_tol(None, None)  # the wrapper's default tolerances
    rc = _lib.lib().integrateFullOrbit_cuda(
        n, yo.ctypes.data_as(dp), len(t), t.ctypes.data_as(dp), 0, len(pt),
        pt.ctypes.data_as(ip), pa.ctypes.data_as(dp), None, -9999.99, lr, la,
        res.ctypes.data_as(dp), er.ctypes.data_as(ip), 6, cb, ctypes.byref(opts))
    assert rc == 0 and not er.any()
    assert calls[0] == n
    assert ms.value > 0.0
    assert np.array_equal(res, ref)


def test_split_sos_and_variational(golden):
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    ics = _sorted_ics(1001, 72)
    psi = np.linspace(0, 20 * np.pi, 11)
    s1, e1 = gb.integrateFullOrbit_sos_cuda((pt, pa), ics, psi, 0.0, "dop853_cuda",
                                            progressbar=False)
    s2, e2 = gb.integrateFullOrbit_sos_cuda((pt, pa), ics, psi, 0.0, "dop853_cuda",
                                            progressbar=False, devices=[0, 0])
    assert np.array_equal(e1, e2) and np.array_equal(s1, s2, equal_nan=True)
    from helpers import cyl_to_rect

    w = np.concatenate([cyl_to_rect(ics[:300]), np.tile(np.eye(6)[0], (300, 1))], 1)
    t = np.linspace(0, 10, 6)
    v1, f1 = gb.integrate_dxdv_batch((pt, pa), w, t, "dop853_cuda")
    v2, f2 = gb.integrate_dxdv_batch((pt, pa), w, t, "dop853_cuda", devices=[0, 0, 0, 0])
    assert np.array_equal(f1, f2) and np.array_equal(v1, v2)


def test_every_visible_device_and_bad_ordinals(golden):
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    ics = _sorted_ics(300, 73)
    t = np.linspace(0, 3, 4)
    o1, _ = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "rk4_cuda", progressbar=False)
    o2, _ = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "rk4_cuda", progressbar=False,
                                       devices=-1)
    assert np.array_equal(o1, o2)
    count = _lib.lib().galpy_cuda_device_count()
    with pytest.raises(_lib.CudaError, match="out of range"):
        gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "rk4_cuda", progressbar=False,
                                   devices=[0, count])
    # fewer orbits than ranges: one device
    o3, _ = gb.integrateFullOrbit_cuda((pt, pa), ics[:2].copy(), t, "rk4_cuda",
                                       progressbar=False, devices=[0, 0, 0])
    assert np.array_equal(o3, o1[:2])
