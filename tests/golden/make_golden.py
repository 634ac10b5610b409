"""Generate the golden fixtures in tests/golden/ (run in a container that has
the reference tree and its C build, oracle/_ref/libgalpy_ref.so):

    make -C oracle ref && python tests/golden/make_golden.py

Two kinds of vectors are written to golden.npz:

* from galpy's own Python (imported from the reference tree): the
  MWPotential2014 argument vector galpy passes to C (_parse_pot), and the
  Python-side forces, second derivatives and potential values of
  MWPotential2014 / Hernquist / LogarithmicHalo (axisymmetric and
  triaxial) / NFW / MiyamotoNagai / PowerSphericalwCutoff and of the
  spherical PowerSpherical, Kepler, Jaffe, Isochrone, Plummer,
  PseudoIsothermal, Burkert, DehnenCoreSpherical, DehnenSpherical,
  HomogeneousSphere, Null, Einasto and ExpTruncNFW potentials, the
  axisymmetric FlattenedPower, KuzminKutuzovStaeckel and KuzminDisk, the
  planar HenonHeiles and the ellipsoidal family at fixed points, plus
  galpy's pure-Python DOP853 orbits (galpy/util/leung_dop853.py) in
  MWPotential2014;
* from the reference's own C integrators (integrateFullOrbit /
  integratePlanarOrbit / *_dxdv built from its sources into oracle/_ref):
  small seeded batches for every implemented method, 3D, planar and
  variational, runs in each of the spherical potentials, and surface-of-
  section runs (integrateFullOrbit_sos).

The CPU oracle is checked against these in tests/test_oracle.py, so it stays
pinned on machines that have neither the reference tree nor oracle/_ref.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from galpy_stub import import_galpy  # noqa: E402

from oracle import oracle as O  # noqa: E402


def seeded_ics(n, seed, planar=False):
    rng = np.random.default_rng(seed)
    R = rng.uniform(0.5, 2.0, n)
    vR = rng.normal(0, 0.1, n)
    vT = 1 + rng.normal(0, 0.1, n)
    z = rng.normal(0, 0.05, n)
    vz = rng.normal(0, 0.05, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    if planar:
        return np.stack([R, vR, vT, phi], 1)
    return np.stack([R, vR, vT, z, vz, phi], 1)


def cyl_to_rect(v):
    if v.shape[-1] == 4:
        R, vR, vT, phi = v.T
        return np.stack([R * np.cos(phi), R * np.sin(phi), vR * np.cos(phi) - vT * np.sin(phi),
                         vR * np.sin(phi) + vT * np.cos(phi)], 1)
    R, vR, vT, z, vz, phi = v.T
    return np.stack([R * np.cos(phi), R * np.sin(phi), z, vR * np.cos(phi) - vT * np.sin(phi),
                     vR * np.sin(phi) + vT * np.cos(phi), vz], 1)


def main():
    galpy = import_galpy()
    if galpy is None or not O.ref_available():
        raise SystemExit("needs the reference tree and oracle/_ref (make -C oracle ref)")
    from galpy import potential as gp
    from galpy.orbit import Orbit
    from galpy.orbit.integrateFullOrbit import _parse_pot as parse3
    from galpy.orbit.integratePlanarOrbit import _parse_pot as parse2

    out = {}
    mw = gp.MWPotential2014
    _, pt, pa, _ = parse3(mw)
    out["mw14_type"] = np.asarray(pt, np.int32)
    out["mw14_args"] = np.asarray(pa)
    _, pt2, pa2, _ = parse2(gp.toPlanarPotential(mw))
    out["mw14_planar_type"] = np.asarray(pt2, np.int32)
    out["mw14_planar_args"] = np.asarray(pa2)

    # galpy Python forces at fixed points
    rng = np.random.default_rng(7)
    R = rng.uniform(0.05, 3.0, 64)
    z = rng.normal(0, 0.4, 64)
    phi = rng.uniform(0, 2 * np.pi, 64)
    out["pts_R"], out["pts_z"], out["pts_phi"] = R, z, phi
    pots = {
        "mw14": mw,
        "hernquist": [gp.HernquistPotential(amp=1.3, a=0.7)],
        "loghalo": [gp.LogarithmicHaloPotential(normalize=1.0, q=0.9, core=0.2)],
        "logtri": [gp.LogarithmicHaloPotential(normalize=1.0, q=0.9, core=0.2, b=0.8)],
        "nfw": [gp.NFWPotential(a=3.0, normalize=0.5)],
        "mn": [gp.MiyamotoNagaiPotential(a=0.5, b=0.1, normalize=0.7)],
        "pswc": [gp.PowerSphericalPotentialwCutoff(alpha=1.2, rc=0.5, normalize=0.2)],
    }
    # the spherical potentials added behind the same component template
    sph = {
        "power": [gp.PowerSphericalPotential(amp=1.0, alpha=1.8)],
        "kepler": [gp.KeplerPotential(amp=0.9)],
        "jaffe": [gp.JaffePotential(amp=1.2, a=0.8)],
        "isochrone": [gp.IsochronePotential(amp=1.1, b=0.6)],
        "plummer": [gp.PlummerPotential(amp=1.0, b=0.5)],
        "pseudoiso": [gp.PseudoIsothermalPotential(amp=0.9, a=0.7)],
        "burkert": [gp.BurkertPotential(amp=1.3, a=0.9)],
        "dehnencore": [gp.DehnenCoreSphericalPotential(amp=2.5, a=0.7)],
        "dehnen": [gp.DehnenSphericalPotential(amp=2.2, a=0.6, alpha=1.2)],
        "homsphere": [gp.HomogeneousSpherePotential(amp=0.4, R=1.5)],
        # galpy drops NullPotentials from combined lists before parsing, so
        # type 40 reaches C only on its own; its Python value is the
        # constant amp, which C never evaluates
        "null": [gp.NullPotential()],
        "einasto": [gp.EinastoPotential(amp=1.5, h=1.2, n=1.8)],
        "exptruncnfw": [gp.ExpTruncNFWPotential(amp=2.0, a=1.5, rc=6.0)],
        # axisymmetric (the same tests)
        "flatpower": [gp.FlattenedPowerPotential(amp=1.1, alpha=0.5, q=0.8, core=0.3)],
        "flatlog": [gp.FlattenedPowerPotential(amp=0.9, alpha=0.0, q=0.7, core=0.2)],
        "kks": [gp.KuzminKutuzovStaeckelPotential(amp=1.0, ac=5.0, Delta=0.8)],
        "kuzmindisk": [gp.KuzminDiskPotential(amp=1.3, a=0.7)],
    }
    pots.update(sph)
    for name, p in pots.items():
        _, t_, a_, _ = parse3(p)
        out[f"{name}_type"] = np.asarray(t_, np.int32)
        out[f"{name}_args"] = np.asarray(a_)
        fns = (gp.evaluateRforces, gp.evaluatezforces, gp.evaluatephitorques,
               gp.evaluateR2derivs, gp.evaluatez2derivs, gp.evaluateRzderivs,
               gp.evaluatePotentials)
        vals = np.stack([np.broadcast_to(np.asarray(f(p, R, z, phi=phi), float), R.shape)
                         for f in fns], 1)
        out[f"{name}_pyforces"] = vals

    # galpy pure-Python DOP853 orbits (galpy/util/leung_dop853.py)
    ics = seeded_ics(3, 11)
    ts = np.linspace(0.0, 10.0, 101)
    o = Orbit(ics)
    o.integrate(ts, mw, method="dop853")
    out["pydop_ics"] = ics
    out["pydop_t"] = ts
    out["pydop_orbit"] = np.stack([o.R(ts), o.vR(ts), o.vT(ts), o.z(ts), o.vz(ts), o.phi(ts)],
                                  -1)

    # the reference's own C integrators in the spherical potentials:
    # dop853 in 3D, symplec4 in the plane, dop853 variational in 3D
    ics = seeded_ics(8, 0)
    ics2 = seeded_ics(8, 1, planar=True)
    t = np.linspace(0, 5, 51)
    w = np.zeros((2, 12))
    w[:, :6] = cyl_to_rect(ics[:2])
    w[0, 6] = w[1, 10] = 1.0
    for name, p in sph.items():
        _, ptn, pan, _ = parse3(p)
        _, ptn2, pan2, _ = parse2(gp.toPlanarPotential(p))
        out[f"{name}_planar_type"] = np.asarray(ptn2, np.int32)
        out[f"{name}_planar_args"] = np.asarray(pan2)
        res, _, _, _ = O.integrate(ics, t, ptn, pan, "dop853", impl="ref")
        out[f"sph_{name}_3d"] = res
        res, _, _, _ = O.integrate(ics2, t, ptn2, pan2, "symplec4", planar=True, impl="ref")
        out[f"sph_{name}_planar"] = res
        res, _, _ = O.integrate_dxdv(w, t, ptn, pan, "dop853", impl="ref")
        out[f"sph_{name}_dxdv3"] = res
    out["sph_dxdv_w3"] = w

    # the reference's own C integrators
    ics = seeded_ics(8, 0)
    ics2 = seeded_ics(8, 1, planar=True)
    out["c_ics"], out["c_ics_planar"] = ics, ics2
    for m in ("leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"):
        t = np.linspace(0, 5, 51)
        res, err, _, _ = O.integrate(ics, t, pt, pa, m, impl="ref")
        out[f"c_{m}_3d"] = res
        res, err, _, _ = O.integrate(ics2, t, pt2, pa2, m, planar=True, impl="ref")
        out[f"c_{m}_planar"] = res
    # per-orbit time grids, dop853, looser tolerance
    tend = np.linspace(3.0, 9.0, 8)
    tt = np.linspace(0, 1, 21)[None, :] * tend[:, None]
    out["c_indiv_t"] = tt
    res, _, _, _ = O.integrate(ics, tt, pt, pa, "dop853", rtol=1e-10, atol=1e-10, impl="ref")
    out["c_dop853_indiv"] = res
    res, _, _, _ = O.integrate(ics, tt, pt, pa, "dopr54", rtol=1e-10, atol=1e-10, impl="ref")
    out["c_dopr54_indiv"] = res
    # dopr54's forced steps: one output interval of 50 started with an
    # explicit step of 50 at an unreachable tolerance, so every orbit ends up
    # at the smallest allowed step (interval's first step / 10000), err = 1
    res, err, _, _ = O.integrate(ics, np.array([0.0, 50.0]), pt, pa, "dopr54", dt=50.0,
                                 rtol=1e-20, atol=1e-20, impl="ref")
    out["c_dopr54_forced"], out["c_dopr54_forced_err"] = res, err
    # variational
    w = np.zeros((6, 12))
    w[:, :6] = cyl_to_rect(ics[:6])
    w[np.arange(6), 6 + np.arange(6)] = 1.0
    w2 = np.zeros((4, 8))
    w2[:, :4] = cyl_to_rect(ics2[:4])
    w2[np.arange(4), 4 + np.arange(4)] = 1.0
    out["c_dxdv_w3"], out["c_dxdv_w2"] = w, w2
    t = np.linspace(0, 3, 31)
    for m in ("leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"):
        res, _, _ = O.integrate_dxdv(w, t, pt, pa, m, impl="ref")
        out[f"c_{m}_dxdv3"] = res
        res, _, _ = O.integrate_dxdv(w2, t, pt2, pa2, m, planar=True, impl="ref")
        out[f"c_{m}_dxdv2"] = res
    # surface of section (integrateFullOrbit_sos): 8 orbits in MWPotential2014,
    # ten crossings of psi = 0 (mod 2 pi), every RK-type method; per-orbit
    # increments with dop853
    yo7 = np.concatenate([seeded_ics(8, 5), np.linspace(0.0, 1.0, 8)[:, None]], 1)
    psi = np.linspace(0.0, 20.0 * np.pi, 11)
    out["sos_yo"], out["sos_psi"] = yo7, psi
    for m in ("rk4", "rk6", "dopr54", "dop853"):
        res, err, _ = O.integrate_sos(yo7, psi, pt, pa, m, rtol=1e-10, atol=1e-10, impl="ref")
        assert not err.any()
        out[f"sos_{m}"] = res
    # planar (integratePlanarOrbit_sos), surfaces x = 0 and y = 0
    yo5 = np.concatenate([seeded_ics(8, 6, planar=True), np.linspace(0.0, 1.0, 8)[:, None]], 1)
    out["sos_planar_yo"] = yo5
    for surface in (0, 1):
        for m in ("rk4", "rk6", "dopr54", "dop853"):
            res, err, _ = O.integrate_sos(yo5, psi, pt2, pa2, m, rtol=1e-10, atol=1e-10,
                                          planar=True, surface=surface, impl="ref")
            assert not err.any()
            out[f"sos_planar{surface}_{m}"] = res
    psi_i = np.linspace(0.0, 1.0, 6)[None, :] * np.linspace(6.0, 30.0, 8)[:, None]
    out["sos_psi_indiv"] = psi_i
    res, _, _ = O.integrate_sos(yo7, psi_i, pt, pa, "dop853", rtol=1e-10, atol=1e-10, impl="ref")
    out["sos_dop853_indiv"] = res

    # the planar Henon-Heiles potential (type 29, a planarPotential only):
    # galpy's Python forces at the planar points, and the reference's C
    # orbits (every method), variational orbits and surface of section
    # x = 0 for bound orbits (E < 1/6 for amp = 1)
    hh = gp.HenonHeilesPotential(amp=1.2)
    _, pth, pah, _ = parse2([hh])
    out["hh_type"], out["hh_args"] = np.asarray(pth, np.int32), np.asarray(pah)
    out["hh_pyforces"] = np.stack(
        [np.asarray([f(r, phi=q) for r, q in zip(R, phi)], float)
         for f in (hh.Rforce, hh.phitorque, hh.R2deriv, hh.phi2deriv, hh.Rphideriv, hh)], 1)
    hics = np.stack([np.full(8, 0.3), np.linspace(-0.2, 0.2, 8), np.full(8, 0.22),
                     np.linspace(0.0, 6.0, 8)], 1)
    out["hh_ics"] = hics
    t = np.linspace(0, 30, 61)
    for m in ("leapfrog", "rk4", "rk6", "symplec4", "symplec6", "dopr54", "dop853"):
        res, err, _, _ = O.integrate(hics, t, pth, pah, m, planar=True, rtol=1e-10, atol=1e-10,
                                     impl="ref")
        assert not err.any()
        out[f"hh_{m}"] = res
    w2 = np.zeros((4, 8))
    w2[:, :4] = cyl_to_rect(hics[:4])
    w2[np.arange(4), 4 + np.arange(4)] = 1.0
    out["hh_dxdv_w2"] = w2
    res, _, _ = O.integrate_dxdv(w2, np.linspace(0, 10, 21), pth, pah, "dop853", planar=True,
                                 impl="ref")
    out["hh_dop853_dxdv2"] = res
    hyo = np.concatenate([hics, np.zeros((8, 1))], 1)
    for m in ("rk6", "dop853"):
        res, err, _ = O.integrate_sos(hyo, psi, pth, pah, m, rtol=1e-10, atol=1e-10,
                                      planar=True, surface=0, impl="ref")
        assert not err.any()
        out[f"hh_sos0_{m}"] = res

    # the EllipsoidalPotential family (aligned and rotated): galpy's Python
    # forces (second derivatives where galpy implements them: aligned only;
    # NaN elsewhere), and the reference's C orbits (dop853 3D, symplec4
    # planar, dop853 variational 3D)
    ell = {
        "trihern": gp.TriaxialHernquistPotential(amp=1.5, a=0.8, b=0.8, c=0.6),
        "trinfw": gp.TriaxialNFWPotential(amp=2.0, a=2.0, b=0.9, c=0.7, zvec=[0.1, 0.2, 1.0],
                                          pa=0.3),
        "trijaffe": gp.TriaxialJaffePotential(amp=1.2, a=0.9, b=0.85, c=0.75, pa=0.4),
        "perfell": gp.PerfectEllipsoidPotential(amp=1.1, a=1.2, b=0.9, c=0.8),
        "trigauss": gp.TriaxialGaussianPotential(amp=1.3, sigma=1.5, b=0.8, c=0.7),
        "powertri": gp.PowerTriaxialPotential(amp=1.0, alpha=1.6, b=0.85, c=0.75, pa=0.2),
        "twopowtri": gp.TwoPowerTriaxialPotential(amp=1.4, a=1.1, alpha=1.2, beta=3.6, b=0.9,
                                                  c=0.8),
    }
    ics = seeded_ics(8, 0)
    ics2 = seeded_ics(8, 1, planar=True)
    t = np.linspace(0, 5, 51)
    w = np.zeros((2, 12))
    w[:, :6] = cyl_to_rect(ics[:2])
    w[0, 6] = w[1, 10] = 1.0
    for name, p in ell.items():
        _, pte, pae, _ = parse3([p])
        _, pte2, pae2, _ = parse2(gp.toPlanarPotential([p]))
        out[f"ell_{name}_type"] = np.asarray(pte, np.int32)
        out[f"ell_{name}_args"] = np.asarray(pae)
        out[f"ell_{name}_planar_type"] = np.asarray(pte2, np.int32)
        out[f"ell_{name}_planar_args"] = np.asarray(pae2)
        cols = [np.asarray(f(p, R, z, phi=phi), float)
                for f in (gp.evaluateRforces, gp.evaluatezforces, gp.evaluatephitorques)]
        for fn in ("R2deriv", "z2deriv", "Rzderiv", "phi2deriv", "Rphideriv", "phizderiv"):
            try:
                cols.append(np.array([getattr(p, fn)(r, zz, phi=q) for r, zz, q in zip(R, z, phi)]))
            except NotImplementedError:
                cols.append(np.full(len(R), np.nan))
        cols.append(np.asarray(gp.evaluatePotentials(p, R, z, phi=phi), float))
        out[f"ell_{name}_pyforces"] = np.stack(cols, 1)
        res, err, _, _ = O.integrate(ics, t, pte, pae, "dop853", impl="ref")
        assert not err.any()
        out[f"ell_{name}_3d"] = res
        res, err, _, _ = O.integrate(ics2, t, pte2, pae2, "symplec4", planar=True, impl="ref")
        out[f"ell_{name}_planar"] = res
        res, _, _ = O.integrate_dxdv(w, t, pte, pae, "dop853", impl="ref")
        out[f"ell_{name}_dxdv3"] = res

    # galpy's pure-Python DOP853 (an implementation apart from its C) in the
    # planar HenonHeiles and the 3D TriaxialHernquist potentials
    ts = np.linspace(0.0, 10.0, 51)
    o = Orbit(hics[:3])
    o.integrate(ts, hh, method="dop853")
    out["pydop_hh_orbit"] = np.stack([o.R(ts), o.vR(ts), o.vT(ts), o.phi(ts)], -1)
    pics = seeded_ics(3, 12)
    o = Orbit(pics)
    o.integrate(ts, ell["trihern"], method="dop853")
    out["pydop_trihern_ics"] = pics
    out["pydop_trihern_orbit"] = np.stack([o.R(ts), o.vR(ts), o.vT(ts), o.z(ts), o.vz(ts),
                                           o.phi(ts)], -1)

    # gradient oracle of the adjoint: Jacobians d y(T) / d y(0) from the
    # reference's variational DOP853 (integrate{Planar,Full}Orbit_dxdv), one
    # unit deviation column per run, t in [0, 20], rtol = atol = 1e-10
    for planar, n, seed in ((True, 6, 3), (False, 4, 4)):
        ics = cyl_to_rect(seeded_ics(n, seed, planar=planar))
        nv = ics.shape[1]
        ptp, pap = (pt2, pa2) if planar else (pt, pa)
        jac = np.zeros((n, nv, nv))
        yT = np.zeros((n, nv))
        for c in range(nv):
            w = np.zeros((n, 2 * nv))
            w[:, :nv] = ics
            w[:, nv + c] = 1.0
            res, err, _ = O.integrate_dxdv(w, np.array([0.0, 20.0]), ptp, pap, "dop853",
                                           planar=planar, rtol=1e-10, atol=1e-10, impl="ref")
            assert not err.any()
            jac[:, :, c] = res[:, -1, nv:]
            yT = res[:, -1, :nv]
        key = "adj_planar" if planar else "adj_3d"
        out[f"{key}_w0"], out[f"{key}_jac"], out[f"{key}_yT"] = ics, jac, yT
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
