"""Device Psi4 extraction (granite_ccz4_psi4_modes*) against the oracle's
restatement of Psi4Extractor::extract (postprocess.cpp:245-314, pinned bit for
bit to the compiled reference in test_oracle_pin.py): the golden vector, blocks
and radii fully inside, partly inside and outside, l_max 2..6, the resident,
host and device-pointer forms, and the inside-point counts exactly.

Tolerance: the device's sin, cos and pow are CUDA's and its sums run in a tree,
so modes agree to rounding: |d| <= 1e-12 max |modes| of the radius."""
import os

import numpy as np
import pytest

import oracle
from oracle import Geom

from test_parity_gpu import block_of

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def close(got, want):
    for r in range(want.shape[0]):
        s = np.abs(want[r]).max()
        assert np.abs(got[r] - want[r]).max() <= TOL * max(s, 1e-300), f"radius {r}"


def host_modes(gb, g, u, radii, nth, nph, l_max):
    from granite_b200.gw import GWExtractionParams, Psi4Extractor
    ev = gb.CCZ4Evolution(gb.CCZ4Params())
    ex = Psi4Extractor(GWExtractionParams(extraction_radii=list(radii), l_max=l_max, n_theta=nth, n_phi=nph))
    ex.extract_block(ev, block_of(g, u), 0.0)
    from granite_b200.gw import mode_list
    keys = mode_list(l_max)
    out = np.array([[ex.getMode(l, m, r) for (l, m) in keys] for r in radii])
    return out, ex


def test_psi4_golden(gb):
    z = np.load(os.path.join(GOLD, "psi4_modes.npz"))
    g = Geom(tuple(int(x) for x in z["n"]), tuple(float(x) for x in z["lo"]), tuple(float(x) for x in z["hi"]))
    u = oracle.seeded_state(g, int(z["seed"]))
    got, ex = host_modes(gb, g, u, z["radii"], int(z["n_theta"]), int(z["n_phi"]), int(z["l_max"]))
    close(got, z["modes"])
    assert float(z["radii"][-1]) not in ex.data  # no point of the outer radius inside: nothing recorded


@pytest.mark.parametrize("n,l_max,nth,nph", [((32, 28, 24), 4, 40, 80), ((17, 23, 19), 2, 9, 13),
                                             ((24, 24, 24), 6, 64, 128)])
def test_psi4_resident_vs_oracle(gb, oracle_lib, n, l_max, nth, nph):
    g = Geom(n, (-8.0, -7.0, -6.0), (8.0, 7.5, 6.5))
    u = oracle.seeded_state(g, 21)
    radii = [2.0, 5.5, 6.8, 7.4, 30.0]
    want, npts = oracle_lib.psi4_modes(g, u, radii, nth, nph, l_max, counts=True)
    ev = gb.Evolver(gb.CCZ4Params())
    ev.add_block(block_of(g, u))
    ev.commit()
    ev.upload()
    import ctypes as C
    nm = (l_max + 1) ** 2 - 4
    out = np.zeros((len(radii), nm, 2))
    cnt = (C.c_int * len(radii))()
    r = np.array(radii)
    ev.ctx.check(ev.ctx.lib.granite_ccz4_psi4_modes(ev.ctx.h, 0, r.ctypes.data_as(C.POINTER(C.c_double)), len(radii),
                                                    nth, nph, l_max, out.ctypes.data_as(C.POINTER(C.c_double)), cnt))
    close(out[..., 0] + 1j * out[..., 1], want)
    assert list(cnt) == npts
    ev.close()


def test_psi4_time_series_and_errors(gb, oracle_lib):
    from granite_b200.gw import GWExtractionParams, Psi4Extractor
    g = Geom((20, 20, 20), (-5.0, -5.0, -5.0), (5.0, 5.0, 5.0))
    ev = gb.Evolver(gb.CCZ4Params())
    ev.add_block(block_of(g, oracle.seeded_state(g, 3)))
    ev.commit()
    ev.upload()
    ex = Psi4Extractor(GWExtractionParams(extraction_radii=[2.0, 3.0], l_max=3, n_theta=12, n_phi=24))
    for t in (0.0, 0.1, 0.1, 0.2):
        ex.extract(ev, 0, t)
    s = ex.getTimeSeries(2, 2, 2.0)
    assert [p[0] for p in s] == [0.0, 0.1, 0.2] and s[1][1] == 2 * s[0][1]
    with pytest.raises(gb.GraniteError):
        Psi4Extractor(GWExtractionParams(extraction_radii=[2.0], l_max=17)).extract(ev, 0, 0.0)
    with pytest.raises(gb.GraniteError):
        Psi4Extractor(GWExtractionParams(extraction_radii=[2.0], n_theta=0)).extract(ev, 0, 0.0)
    ev.close()
