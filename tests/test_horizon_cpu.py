"""Host logic of the horizon finder against the compiled reference, on the CPU.

``findCommonHorizon`` (horizon_finder.cpp:510-551) is a guess (the
irreducible-mass-weighted centroid of the horizons and an enclosing radius)
followed by ``findHorizon`` from it; ``computeSpin`` (:553-582) maps the
circumference ratio to a spin. Both guesses and spins are host arithmetic
here (``granite_b200.horizon``). The reference's own findCommonHorizon is
compared with the reference's findHorizon started from this package's guess:
equal surfaces and integrals, bit for bit, pin the guess without a GPU.
"""
import math

import numpy as np
import pytest

from oracle import Geom
from granite_b200.horizon import ApparentHorizonFinder, HorizonData, common_horizon_guess, surface_points

PI = 3.14159265358979323846


def hd(i, centroid, m_irr, c_eq, c_pol=0.0):
    return HorizonData(i, tuple(centroid), 0.0, m_irr, 0.0, (0.0, 0.0, 1.0), c_eq, c_pol)


@pytest.fixture(scope="module")
def binary():
    g = Geom((41, 33, 33), (-2.05, -1.65, -1.65), (2.05, 1.65, 1.65))
    return g


@pytest.mark.parametrize("horizons,tol", [
    # the two horizons the reference finds about the BL punctures m = 0.6, 0.4 at x = -+1
    ([((-1.0, 0.0, 0.0), 0.766165062, 0.3), ((1.0, 0.0, 0.0), 0.293438394, 0.4)], 0.3),
    ([((-1.0, 0.0, 0.0), 0.766165062, 0.3), ((1.0, 0.0, 0.0), 0.293438394, 0.4)], 1.0),
    # off-axis centroids, three horizons, one of them massless
    ([((-0.6, 0.2, -0.1), 0.5, 1.1), ((0.7, -0.15, 0.25), 0.25, 0.6), ((0.1, 0.3, 0.0), 0.0, 2.0)], 0.3),
])
def test_common_horizon_guess_matches_reference(reference_lib, binary, horizons, tol):
    g = binary
    u = reference_lib.init_brill_lindquist(g, [0.6, 0.4], [[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    hs = [hd(i, c, m, ce) for i, (c, m, ce) in enumerate(horizons)]
    cc, radius = common_horizon_guess(hs)
    found, res, surf, (cen, hid) = reference_lib.find_common_horizon(
        g, u, [h.centroid for h in hs], [h.irreducible_mass for h in hs],
        [h.circumference_equatorial for h in hs], 400, tol, 6, 0.4)
    f2, res2, surf2 = reference_lib.find_horizon(g, u, cc, 400, tol, 6, radius)
    assert found and f2
    assert cen == tuple(cc) and hid == len(hs)
    assert np.array_equal(surf, surf2) and np.array_equal(res, res2)


def test_common_horizon_guess_edge_cases():
    """Fewer than two horizons, or a total irreducible mass below 1e-14: no search."""
    assert common_horizon_guess([]) is None
    assert common_horizon_guess([hd(0, (0, 0, 0), 1.0, 1.0)]) is None
    assert common_horizon_guess([hd(0, (0, 0, 0), 0.0, 1.0), hd(1, (1, 0, 0), 5e-15, 1.0)]) is None
    f = ApparentHorizonFinder()
    assert f.findCommonHorizon(None, [hd(0, (0, 0, 0), 1.0, 1.0)]) is None  # returns before any device call
    cc, r = common_horizon_guess([hd(0, (-1, 0, 0), 1.0, 2 * PI), hd(1, (1, 0, 0), 1.0, 0.0)])
    assert cc == [0.0, 0.0, 0.0] and r == pytest.approx(1.2 * 2.0, abs=0)


@pytest.mark.parametrize("c_eq,c_pol", [
    (0.0, 1.0), (1e-13, 1.0), (-1.0, 2.0), (2.0, 1.5), (2.0, 2.0), (2.0, 2.0000001), (2.0, 2.5),
    (2.0, 3.0), (2.0, PI), (2.0, 3.2), (10.0, 15.7), (1.0, float("inf")), (float("inf"), 1.0),
])
def test_compute_spin_matches_reference(reference_lib, c_eq, c_pol):
    got = ApparentHorizonFinder().computeSpin(hd(0, (0, 0, 0), 1.0, c_eq, c_pol))
    want = reference_lib.compute_spin(c_eq, c_pol)
    assert got == want or (math.isnan(got) and math.isnan(want))


def test_surface_points_layout():
    """Point (i, j) at index i * 2n + j: theta = pi (i + 1/2) / n, phi = 2 pi j / (2n)."""
    n = 4
    radii = np.arange(n * 2 * n, dtype=float).reshape(n, 2 * n) * 0.01 + 1.0
    pts = surface_points((0.5, -0.25, 2.0), radii)
    assert len(pts) == n * 2 * n
    for i in range(n):
        th = PI * (i + 0.5) / n
        for j in range(2 * n):
            ph = 2.0 * PI * j / (2 * n)
            r = radii[i, j]
            assert pts[i * 2 * n + j] == (0.5 + r * math.sin(th) * math.cos(ph),
                                          -0.25 + r * math.sin(th) * math.sin(ph), 2.0 + r * math.cos(th))
