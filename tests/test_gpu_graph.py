"""CUDA-graph capture of a device-resident integration and the launch-shape
autotuner, on a B200."""
import numpy as np
import pytest
from helpers import cyl_to_rect, seeded_ics

import galpy_b200 as gb
from galpy_b200 import _lib, autotune
from galpy_b200.graph import IntegrationGraph

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "no CUDA device: GPU tests need a GPU"


def _batch(mw14, n=4096, seed=12):
    pt, pa = mw14
    comps, ncomp = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    ics = seeded_ics(n, seed)
    tend = np.random.default_rng(seed).uniform(5, 15, n)
    t = np.linspace(0, 1, 11)[None, :] * tend[:, None]
    dev = torch.device("cuda")
    return dict(comps=torch.tensor(comps, device=dev), ncomp=ncomp, sig=sig, comps_host=comps,
                w0=torch.tensor(cyl_to_rect(ics).T.copy(), device=dev),
                t=torch.tensor(t, device=dev),
                out=torch.empty((6, 11, n), dtype=torch.float64, device=dev),
                err=torch.empty(n, dtype=torch.int32, device=dev),
                ns=torch.empty(n, dtype=torch.int64, device=dev))


def _direct(b, method="dop853_cuda", **kw):
    out = torch.empty_like(b["out"])
    err = torch.empty_like(b["err"])
    ns = torch.empty_like(b["ns"])
    gb.integrate_device(b["comps"], b["ncomp"], b["w0"], b["t"], out, err, method, nsteps=ns,
                        rtol=1e-10, atol=1e-10, signature=b["sig"], comps_host=b["comps_host"],
                        **kw)
    torch.cuda.synchronize()
    return out, err, ns


@pytest.mark.parametrize("method", ["dop853_cuda", "symplec4_cuda"])
def test_graph_replay_matches_direct_call(mw14, method):
    b = _batch(mw14)
    ref_out, ref_err, ref_ns = _direct(b, method)
    g = IntegrationGraph(b["comps"], b["ncomp"], b["w0"], b["t"], b["out"], b["err"], method,
                         nsteps=b["ns"], rtol=1e-10, atol=1e-10, signature=b["sig"],
                         comps_host=b["comps_host"])
    for _ in range(2):
        b["out"].zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(b["out"], ref_out) and torch.equal(b["err"], ref_err)
        assert torch.equal(b["ns"], ref_ns)
    # new contents of the bound input buffer are picked up by the next replay
    b["w0"][3] *= 1.01  # vx of every orbit
    new_out, _, _ = _direct(b, method)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(b["out"], new_out) and not torch.equal(new_out, ref_out)


def test_autotune_picks_a_candidate_and_caches(mw14, tmp_path, monkeypatch):
    monkeypatch.setenv("GALPY_B200_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    b = _batch(mw14, n=2048)
    cfg = autotune.tune(b["comps"], b["ncomp"], b["w0"], b["t"], b["out"], b["err"],
                        "dop853_cuda", rtol=1e-10, atol=1e-10, signature=b["sig"],
                        comps_host=b["comps_host"], sample=1024)
    shapes = autotune.candidates("dop853_cuda")
    assert {k: cfg[k] for k in shapes[0]} in shapes and cfg["ms"] > 0 and cfg["sample"] == 1024
    assert (tmp_path / "tune.json").exists()
    again = autotune.tune(b["comps"], b["ncomp"], b["w0"], b["t"], b["out"], b["err"],
                          "dop853_cuda", rtol=1e-10, atol=1e-10, signature=b["sig"])
    assert again == cfg
    # every candidate shape gives the same result (the shape changes only scheduling)
    ref = _direct(b)
    for shape in shapes:
        out, err, ns = _direct(b, **autotune.launch_kwargs(shape))
        assert torch.equal(out, ref[0]) and torch.equal(ns, ref[2])
