"""The blocking entry points' result streaming on a B200.

For large results integrateFullOrbit_cuda / integratePlanarOrbit_cuda copy
the rows of finished orbits to the host while the kernel runs (staging in
completion order, chunked copies, host-side scatter into galpy's result
array).  Streamed and one-copy transfers must give the same result arrays
bit for bit -- through the queued DOP853 dense output (whose last rows are
written by other lanes than the orbit's own), the plain loop (symplec4),
planar orbits, pageable and pinned result arrays, and orbits stopped
early."""
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


def _both(fn, pot, ics, t, method, **kw):
    res = []
    for stream in (0, 1):
        out, err, ns = fn(pot, ics.copy(), t, method, progressbar=False, return_nsteps=True,
                          stream_rows=stream, **kw)
        res.append((out, err, ns))
    return res


@pytest.mark.parametrize("method", ["dop853_cuda", "symplec4_cuda"])
@pytest.mark.parametrize("planar", [False, True])
def test_streamed_rows_equal_one_copy(golden, method, planar):
    pt, pa = ((golden["mw14_planar_type"], golden["mw14_planar_args"]) if planar
              else (golden["mw14_type"], golden["mw14_args"]))
    n = 3 * 4096 + 517  # several chunks and a partial one
    ics = seeded_ics(n, 60, planar=planar, r_range=(0.05, 3.0), log_r=True)
    rng = np.random.default_rng(60)
    tend = np.exp(rng.normal(np.log(10.0), 0.7, n))
    if method == "dop853_cuda":  # ragged per-orbit grids
        t = np.linspace(0, 1, 51)[None, :] * tend[:, None]
    else:
        t = np.linspace(0, 10, 51)
    fn = gb.integratePlanarOrbit_cuda if planar else gb.integrateFullOrbit_cuda
    (o0, e0, n0), (o1, e1, n1) = _both(fn, (pt, pa), ics, t, method, rtol=1e-10, atol=1e-10)
    assert not e0.any()
    assert np.array_equal(e0, e1) and np.array_equal(n0, n1)
    assert np.array_equal(o0, o1)


def test_streamed_rows_into_pinned_memory(golden):
    import torch

    pt, pa = golden["mw14_type"], golden["mw14_args"]
    n = 2 * 4096 + 3
    ics = seeded_ics(n, 61)
    t = np.linspace(0, 5, 41)
    ref, err = gb.integrateFullOrbit_cuda((pt, pa), ics.copy(), t, "dop853_cuda",
                                          progressbar=False, stream_rows=0)
    import ctypes

    lib = _lib.lib()
    res = torch.empty((n, len(t), 6), dtype=torch.float64, pin_memory=True).numpy()
    res[:] = np.nan
    yo = np.ascontiguousarray(ics)
    er = np.zeros(n, np.int32)
    pti = np.ascontiguousarray(pt, np.int32)
    pad = np.ascontiguousarray(pa, np.float64)
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    opts = _lib.make_opts(stream_rows=1)
    tt = np.ascontiguousarray(t)
    # the wrapper's default tolerances (-12 ln 10, one ulp away from ln 1e-12)
    lr, la = gb.parse_tol(None, None)
    rc = lib.integrateFullOrbit_cuda(n, yo.ctypes.data_as(dp), len(t), tt.ctypes.data_as(dp), 0,
                                     3, pti.ctypes.data_as(ip), pad.ctypes.data_as(dp), None,
                                     -9999.99, lr, la, res.ctypes.data_as(dp),
                                     er.ctypes.data_as(ip), 6, _lib.CALLBACK(),
                                     ctypes.byref(opts))
    assert rc == 0 and not er.any()
    assert np.array_equal(res, ref)


def test_streamed_rows_of_stopped_orbits(golden):
    """Orbits stopped early (here by the attempt budget, err 2) are
    delivered like finished ones: their rows up to the stop, then NaN."""
    pt, pa = golden["mw14_type"], golden["mw14_args"]
    n = 2 * 4096 + 11
    ics = seeded_ics(n, 62)
    t = np.linspace(0, 1e5, 5)
    (o0, e0, _), (o1, e1, _) = _both(gb.integrateFullOrbit_cuda, (pt, pa), ics, t,
                                     "dop853_cuda", max_attempts=400)
    assert (e0 == 2).all() and np.array_equal(e0, e1)
    assert np.array_equal(o0, o1, equal_nan=True)
    assert np.isnan(o1[:, -1]).all() and np.isfinite(o1[:, 0]).all()
