"""Apparent-horizon finder on the GPU against the reference.

The flow of ApparentHorizonFinder::findHorizon (horizon_finder.cpp:310-449) is
computed on the device with the reference's operations in its order, so the
converged iteration, the surface, and the area / mass / spin / circumferences
equal the reference's bit for bit (golden vectors from the compiled
horizon_finder.cpp; the oracle, pinned to it in test_oracle_pin.py, for a flow
that does not converge). findAllHorizons' candidate scan and the results per
candidate likewise.
"""
import os

import numpy as np
import pytest

import oracle
from oracle import Geom

from test_parity_gpu import block_of

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    g = Geom(tuple(int(x) for x in z["n"]), tuple(float(x) for x in z["lo"]), tuple(float(x) for x in z["hi"]))
    return g, z


def resident(gb, g, u):
    ev = gb.Evolver(gb.CCZ4Params())
    ev.add_block(block_of(g, u))
    ev.commit()
    ev.upload()
    return ev


def params(z):
    from granite_b200.horizon import HorizonParams
    return HorizonParams(int(z["max_iterations"]), float(z["tolerance"]), int(z["angular_resolution"]),
                         float(z["initial_guess_radius"]))


def test_find_horizon_golden(gb, oracle_lib):
    from granite_b200.horizon import ApparentHorizonFinder
    g, z = load("horizon_flow")
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]]) + 1e-9 * oracle.hash_noise(g.shape, int(z["seed"]))
    it, _, _ = oracle_lib.find_horizon(g, u, (0.0, 0.0, 0.0), int(z["max_iterations"]), float(z["tolerance"]),
                                       int(z["angular_resolution"]), float(z["initial_guess_radius"]))
    ev = resident(gb, g, u)
    f = ApparentHorizonFinder(params(z))
    for hd in (f.findHorizon((ev, 0), (0.0, 0.0, 0.0)), f.findHorizon((ev, block_of(g, u)), (0.0, 0.0, 0.0))):
        assert hd is not None and hd.iterations == it
        got = [hd.area, hd.irreducible_mass, hd.spin, hd.circumference_equatorial, hd.circumference_polar]
        assert got == list(z["res"])
        assert np.array_equal(np.array(hd.surface_points), z["surface"])
    ev.close()


@pytest.mark.parametrize("center", [(0.05, -0.03, 0.02), (0.1, 0.2, -0.15)])
def test_flow_that_does_not_converge(gb, oracle_lib, center):
    from granite_b200.horizon import ApparentHorizonFinder, HorizonParams
    g = Geom((32, 30, 28), (-1.6, -1.5, -1.4), (1.6, 1.5, 1.4))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]]) + 1e-7 * oracle.hash_noise(g.shape, 9)
    it, h, _ = oracle_lib.find_horizon(g, u, center, 150, 1e-12, 10, 0.8)
    assert it == -1
    ev = resident(gb, g, u)
    f = ApparentHorizonFinder(HorizonParams(150, 1e-12, 10, 0.8))
    radii, iters, found = f.flowRadii((ev, 0), center)
    assert not found and iters == 150
    assert np.array_equal(radii, h)
    assert f.findHorizon((ev, 0), center) is None
    ev.close()


def test_find_all_horizons_golden(gb, oracle_lib):
    from granite_b200.horizon import ApparentHorizonFinder
    g, z = load("horizon_all")
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]])
    ev = resident(gb, g, u)
    f = ApparentHorizonFinder(params(z))
    hs = f.findAllHorizons((ev, 0))
    rows = [list(h.centroid) + [h.area, h.irreducible_mass, h.spin] for h in hs]
    assert np.array_equal(np.array(rows).reshape(-1, 6), z["rows"])
    assert [h.id for h in hs] == list(range(len(hs))) and len(hs) == 1
    assert f.findCommonHorizon((ev, 0), hs) is None  # needs two
    assert 0.0 <= f.computeSpin(hs[0]) <= 1.0
    ev.close()


def test_find_all_horizons_binary_golden(gb, oracle_lib):
    """Two punctures on cell centres: two lapse minima, both horizons found, in
    the reference's order, values bit for bit."""
    from granite_b200.horizon import ApparentHorizonFinder
    g, z = load("horizon_all_binary")
    u = oracle_lib.init_brill_lindquist(g, list(z["masses"]), z["positions"].tolist())
    ev = resident(gb, g, u)
    hs = ApparentHorizonFinder(params(z)).findAllHorizons((ev, 0))
    rows = [list(h.centroid) + [h.area, h.irreducible_mass, h.spin] for h in hs]
    assert len(hs) == 2 and np.array_equal(np.array(rows), z["rows"])
    ev.close()


def test_find_horizon_rejects_bad_params(gb, oracle_lib):
    from granite_b200.horizon import ApparentHorizonFinder, HorizonParams
    g = Geom((16, 16, 16), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    ev = resident(gb, g, oracle.seeded_state(g, 2))
    with pytest.raises(gb.GraniteError):
        ApparentHorizonFinder(HorizonParams(angular_resolution=0)).findHorizon((ev, 0), (0.0, 0.0, 0.0))
    ev.close()
