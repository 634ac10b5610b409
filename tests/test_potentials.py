"""Host-side potential construction against galpy's own argument vectors."""
import numpy as np

import galpy_b200 as gb


def test_mwpotential2014_args_match_galpy(golden):
    n, pt, pa = gb.parse_pot(gb.MWPotential2014())
    assert n == 3 and pt.tolist() == golden["mw14_type"].tolist()
    np.testing.assert_allclose(pa, golden["mw14_args"], rtol=1e-13, atol=0)
    n, pt, pa = gb.parse_pot(gb.MWPotential2014(), planar=True)
    assert pt.tolist() == golden["mw14_planar_type"].tolist()
    np.testing.assert_allclose(pa, golden["mw14_planar_args"], rtol=1e-13, atol=0)


def test_single_potentials_match_galpy(golden):
    cases = {
        "hernquist": gb.HernquistPotential(amp=1.3, a=0.7),
        "loghalo": gb.LogarithmicHaloPotential(normalize=1.0, q=0.9, core=0.2),
        "logtri": gb.LogarithmicHaloPotential(normalize=1.0, q=0.9, core=0.2, b=0.8),
        "nfw": gb.NFWPotential(a=3.0, normalize=0.5),
        "mn": gb.MiyamotoNagaiPotential(a=0.5, b=0.1, normalize=0.7),
        "pswc": gb.PowerSphericalPotentialwCutoff(alpha=1.2, rc=0.5, normalize=0.2),
    }
    for name, p in cases.items():
        n, pt, pa = gb.parse_pot(p)
        assert pt.tolist() == golden[f"{name}_type"].tolist(), name
        np.testing.assert_allclose(pa, golden[f"{name}_args"], rtol=1e-13, atol=0, err_msg=name)


def test_raw_pair_passthrough():
    n, pt, pa = gb.parse_pot(([8], [1.0, 2.0]))
    assert n == 1 and pt.dtype == np.int32 and pa.tolist() == [1.0, 2.0]
