"""The precision forms on a B200 (include/galpy_cuda.h): float64, float32
force / float64 state (f32force), float64 force with float32 tails of its
table polynomials (f64tail32), that with the bulge term in float32
(f32bulge), and float32 force with a double-float state (f32force_df).

Bounds: the forces of the mixed forms against the float64 force (1e-11 and
3e-6 relative, the host build's figures in tests/test_harness.py); on the
precision workload's symplec4 (dt = 0.01), the relative energy drift of
every form and its final distance from the float64 kernel; DOP853 in the
f64tail32 form keeps the float64 accepted-step sequence (its force error is
far below the tolerance the step controller resolves)."""
import numpy as np
import pytest
from helpers import cyl_to_rect, seeded_ics

import galpy_b200 as gb
from galpy_b200 import _lib

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def engine():
    from galpy_b200 import build

    build.build()
    assert _lib.lib().galpy_cuda_device_count() > 0, "GPU tests need a GPU"


def _mw14(golden, planar=False):
    if planar:
        return golden["mw14_planar_type"], golden["mw14_planar_args"]
    return golden["mw14_type"], golden["mw14_args"]


@pytest.mark.parametrize("planar", [False, True])
def test_mixed_forces_on_device(golden, planar):
    pt, pa = _mw14(golden, planar)
    comps, n = gb.compile_potential((pt, pa), planar=planar)
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    rng = np.random.default_rng(31)
    m = 50000
    r = np.exp(rng.uniform(np.log(0.01), np.log(30.0), m))
    th = np.full(m, np.pi / 2) if planar else np.arccos(rng.uniform(-1, 1, m))
    ph = rng.uniform(0, 2 * np.pi, m)
    pos = torch.tensor(np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph),
                                 r * np.cos(th)]), device=dev)
    acc = {}
    for prec in ("fp64", "f64tail32", "f32bulge"):
        a = torch.empty_like(pos)
        gb.accel_device(cd, n, pos, a, planar=planar, signature=1, precision=prec)
        acc[prec] = a
    torch.cuda.synchronize()
    ref = acc["fp64"].cpu().numpy()
    scale = np.abs(ref).max(axis=0)
    for prec, tol in (("f64tail32", 1e-11), ("f32bulge", 3e-6)):
        rel = (np.abs(acc[prec].cpu().numpy() - ref).max(axis=0) / scale).max()
        assert 0 < rel < tol, (prec, rel)


def test_precision_forms_symplec4(golden):
    """The precision workload's integration (symplec4, dt = 0.01, 20,000
    steps) on 4,096 orbits in every form."""
    pt, pa = _mw14(golden)
    comps, n = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    ics = seeded_ics(4096, 2)
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    t = torch.tensor([0.0, 200.0], dtype=torch.float64, device=dev)
    E0 = torch.empty(len(ics), dtype=torch.float64, device=dev)
    gb.energy_device(cd, n, w0, E0)
    fin, drift = {}, {}
    for prec in ("fp64", "f32force", "f64tail32", "f32bulge", "f32force_df"):
        out = torch.empty((6, 1, len(ics)), dtype=torch.float64, device=dev)
        err = torch.empty(len(ics), dtype=torch.int32, device=dev)
        gb.integrate_device(cd, n, w0, t, out, err, "symplec4_cuda", dt=0.01, out_row0=1,
                            precision=prec, signature=sig, comps_host=comps)
        E1 = torch.empty_like(E0)
        gb.energy_device(cd, n, out[:, 0, :], E1)
        torch.cuda.synchronize()
        assert (err == 0).all(), prec
        fin[prec] = out[:, 0, :].cpu().numpy()
        drift[prec] = np.median(torch.abs(E1 / E0 - 1).cpu().numpy())
    scale = np.abs(fin["fp64"]).max(axis=0)
    dist = {p: np.median(np.abs(fin[p] - fin["fp64"]).max(axis=0) / scale) for p in fin}
    # float64 force (tails in float32): the float64 kernel's trajectory and drift
    assert dist["f64tail32"] < 1e-8 and drift["f64tail32"] < 1e-10, (dist, drift)
    # float32 bulge: its rounding noise random-walks the energy, a fraction
    # of the all-float32 force's
    assert drift["f32bulge"] < drift["f32force"] and drift["f32bulge"] < 1e-7, drift
    # float32 force: noise-limited drift, double-float state no better or
    # worse than float64 state
    assert drift["f32force"] < 1e-6 and drift["f32force_df"] < 1e-6, drift
    assert 0.2 < drift["f32force_df"] / drift["f32force"] < 5, drift


def test_dop853_f64tail32_keeps_step_sequence(golden):
    """The batching configuration's DOP853 (rtol = atol = 1e-10) on 2,048
    of its orbits: f64tail32 takes the float64 accepted-step counts and
    agrees with it inside the tolerance."""
    pt, pa = _mw14(golden)
    comps, n = gb.compile_potential((pt, pa))
    sig = gb.signature((pt, pa))
    dev = torch.device("cuda:0")
    cd = torch.tensor(comps, device=dev)
    ics = seeded_ics(2048, 1, r_range=(0.05, 3.0), log_r=True)
    rng = np.random.default_rng(1)
    tend = np.exp(rng.normal(np.log(50), 0.7, len(ics)))
    t = torch.tensor(np.linspace(0, 1, 101)[None, :] * tend[:, None], device=dev)
    w0 = torch.tensor(cyl_to_rect(ics).T.copy(), device=dev)
    res = {}
    for prec in ("fp64", "f64tail32"):
        out = torch.empty((6, 101, len(ics)), dtype=torch.float64, device=dev)
        err = torch.empty(len(ics), dtype=torch.int32, device=dev)
        ns = torch.empty(len(ics), dtype=torch.int64, device=dev)
        gb.integrate_device(cd, n, w0, t, out, err, "dop853_cuda", nsteps=ns, rtol=1e-10,
                            atol=1e-10, precision=prec, signature=sig, comps_host=comps)
        torch.cuda.synchronize()
        assert (err == 0).all()
        res[prec] = (out.cpu().numpy(), ns.cpu().numpy())
    same = res["fp64"][1] == res["f64tail32"][1]
    assert same.mean() >= 0.95, same.mean()
    d = np.abs(res["fp64"][0] - res["f64tail32"][0]).max(axis=(0, 1))
    scale = np.maximum(np.abs(res["fp64"][0]).max(axis=(0, 1)), 1.0)
    # force differences of ~1e-11 stay near the tolerance on most orbits;
    # over tens of dynamical times the chaotic ones amplify them
    rel = (d / scale)[same]
    q50, q99 = np.quantile(rel, [0.5, 0.99])
    assert q50 < 1e-10 and q99 < 1e-7 and rel.max() < 1e-6, (q50, q99, rel.max())


def test_mixed_forms_refuse_other_potentials(golden):
    """The mixed forms exist for MWPotential2014 only: other potentials (and
    variational runs) return GALPY_CUDA_ERR_METHOD, not a silent float64."""
    pt, pa = golden["hernquist_type"], golden["hernquist_args"]
    for prec in ("f64tail32", "f32bulge", "f32force_df"):
        with pytest.raises(gb.MethodNotSupported):
            gb.integrateFullOrbit_cuda((pt, pa), seeded_ics(4, 3), np.linspace(0, 1, 3),
                                       "symplec4_cuda", precision=prec, progressbar=False)
