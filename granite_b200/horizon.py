"""Apparent horizons with the reference's ApparentHorizonFinder interface.

``findHorizon`` and ``findAllHorizons`` (horizon_finder.cpp:310-507) run on the
GPU through ``granite_ccz4_find_horizon*`` / ``granite_ccz4_find_all_horizons``;
``findCommonHorizon`` and ``computeSpin`` (:510-582) are host logic over the
found horizons and stay here, restated.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import GridBlock, _dp, _f64, _Horizon, _HorizonParams

PI = 3.14159265358979323846  # constants::PI


@dataclass
class HorizonParams:
    """horizon_finder.hpp:17-23 (find_every is the caller's schedule, unused here)."""
    max_iterations: int = 200
    tolerance: float = 1.0e-10
    angular_resolution: int = 50
    initial_guess_radius: float = 1.0
    find_every: int = 10

    def _c(self):
        return _HorizonParams(self.max_iterations, self.tolerance, self.angular_resolution,
                              self.initial_guess_radius)


@dataclass
class HorizonData:
    """horizon_finder.hpp:28-40."""
    id: int
    centroid: tuple
    area: float
    irreducible_mass: float
    spin: float
    spin_axis: tuple
    circumference_equatorial: float
    circumference_polar: float
    surface_points: list = field(default_factory=list)
    iterations: int = 0


def surface_points(center, radii):
    """center + r (sin t cos p, sin t sin p, cos t) on the finder's angular grid
    (horizon_finder.cpp:292-300, 384-395), with the host libm as the reference."""
    nth, nph = radii.shape
    pts = []
    for i in range(nth):
        th = PI * (i + 0.5) / nth
        sth, cth = math.sin(th), math.cos(th)
        for j in range(nph):
            ph = 2.0 * PI * j / nph
            r = float(radii[i, j])
            pts.append((center[0] + r * sth * math.cos(ph), center[1] + r * sth * math.sin(ph), center[2] + r * cth))
    return pts


def _data(h: _Horizon, radii=None):
    c = tuple(h.centroid)
    return HorizonData(h.id, c, h.area, h.irreducible_mass, h.spin, (0.0, 0.0, 1.0), h.circumference_equatorial,
                       h.circumference_polar, surface_points(c, radii) if radii is not None else [], h.iterations)


def common_horizon_guess(horizons):
    """Centre and initial radius of the common-horizon search, or None
    (horizon_finder.cpp:513-543): the irreducible-mass-weighted centroid of the
    horizons, and 1.2 times the largest centroid distance plus equatorial
    radius C_eq / (2 pi)."""
    if len(horizons) < 2:
        return None
    total = 0.0
    cc = [0.0, 0.0, 0.0]
    for h in horizons:
        for d in range(3):
            cc[d] += h.irreducible_mass * h.centroid[d]
        total += h.irreducible_mass
    if total < 1.0e-14:
        return None
    cc = [x / total for x in cc]
    max_r = 0.0
    for h in horizons:
        dist = 0.0
        for d in range(3):
            dd = h.centroid[d] - cc[d]
            dist += dd * dd
        max_r = max(max_r, math.sqrt(dist) + h.circumference_equatorial / (2.0 * PI))
    return cc, 1.2 * max_r


class ApparentHorizonFinder:
    """horizon_finder.hpp:43-87. ``source``: (Evolver, block index) for a resident
    block, or (runner, GridBlock) for a host block (runner: any object of this
    package with a context)."""

    def __init__(self, params: HorizonParams | None = None):
        self.params = params or HorizonParams()

    def _find(self, source, center, params):
        obj, blk = source
        ctx = obj.ctx
        n = params.angular_resolution
        radii = np.zeros((n, 2 * n))
        out = _Horizon()
        cen = np.ascontiguousarray(center, dtype=np.float64)
        p = params._c()
        if isinstance(blk, GridBlock):
            ctx.check(ctx.lib.granite_ccz4_find_horizon_host(ctx.h, C.byref(blk.desc()), _dp(_f64(blk.array)),
                                                             C.byref(p), _dp(cen), C.byref(out), _dp(radii)))
        else:
            ctx.check(ctx.lib.granite_ccz4_find_horizon(ctx.h, int(blk), C.byref(p), _dp(cen), C.byref(out),
                                                        _dp(radii)))
        return out, radii

    def findHorizon(self, source, center):
        """The converged surface about ``center``, or None (horizon_finder.cpp:310-449)."""
        out, radii = self._find(source, center, self.params)
        return _data(out, radii) if out.found else None

    def flowRadii(self, source, center):
        """The surface radii after the flow (converged or not) and the iterations run."""
        out, radii = self._find(source, center, self.params)
        return radii, out.iterations, bool(out.found)

    def findAllHorizons(self, source):
        """Horizons about the lapse minima of a resident block (horizon_finder.cpp:452-507)."""
        obj, blk = source
        ctx = obj.ctx
        cap = 64
        out = (_Horizon * cap)()
        n = C.c_int()
        p = self.params._c()
        ctx.check(ctx.lib.granite_ccz4_find_all_horizons(ctx.h, int(blk), C.byref(p), out, cap, C.byref(n)))
        return [_data(out[i]) for i in range(min(n.value, cap))]

    def findCommonHorizon(self, source, horizons):
        """A horizon about the mass-weighted centroid enclosing all (horizon_finder.cpp:510-551)."""
        guess = common_horizon_guess(horizons)
        if guess is None:
            return None
        cc, radius = guess
        p = HorizonParams(self.params.max_iterations, self.params.tolerance, self.params.angular_resolution,
                          radius)
        out, radii = self._find(source, cc, p)
        if not out.found:
            return None
        r = _data(out, radii)
        r.id = len(horizons)
        return r

    def computeSpin(self, horizon: HorizonData) -> float:
        """Spin from the polar / equatorial circumference ratio (horizon_finder.cpp:553-582)."""
        if horizon.circumference_equatorial < 1.0e-12:
            return 0.0
        ratio = horizon.circumference_polar / horizon.circumference_equatorial
        if ratio <= 1.0:
            return 0.0
        if ratio >= PI / 2.0:
            return 1.0
        return (ratio - 1.0) / (PI / 2.0 - 1.0)
