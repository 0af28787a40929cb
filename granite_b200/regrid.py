"""Host side of the reference regrid (AMRHierarchy::regrid, amr.cpp:80-301).

The reference refines around tracking spheres: for every sphere whose
``min_level`` reaches the new level it proposes one box with the base grid's
cell count at half the parent spacing, centred on the sphere and snapped to
the parent grid, merges boxes that overlap or touch, and adds one block per
merged box that no block of the new level already covers. The new blocks are
prolongated from the parent level. Blocks are never removed.

``RegridPlanner`` decides the boxes on the host, with the reference's
floating-point steps in the reference's order, so the new blocks get the
reference's corners and cell counts exactly; ``Evolver.regrid`` in this
package sends them to the device (``granite_ccz4_regrid_add``), which
prolongates their data there, and asks the device tagger
(``granite_ccz4_tag_count``) whether a gradient tagger fires when no sphere
requires the level.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

CHI = 0     # SpacetimeVar::CHI
LAPSE = 18  # SpacetimeVar::LAPSE


def tagger_fires(tagger, count) -> bool:
    """Whether ``tagger`` tags any interior cell of a level (the early-out of
    amr.cpp:124-133). ``tagger``: None (never tags), ``(var, threshold)`` for
    gradientChiTagger (var CHI) or gradientLapseTagger (var LAPSE), or a list of
    taggers for compositeTagger (amr.cpp:723-731: a cell is tagged when any of
    them tags it, so the level is when any of them tags a cell of it).
    ``count(var, threshold)`` is the number of interior cells one tagger tags."""
    if tagger is None:
        return False
    if isinstance(tagger, tuple):
        var, threshold = tagger
        return count(var, threshold) > 0
    return any(tagger_fires(t, count) for t in tagger)


@dataclass
class TrackingSphere:
    """amr.hpp:33-37."""
    center: tuple
    radius: float
    min_level: int


@dataclass
class Box:
    """A planned block: its level, interior cells, corners and reference block id."""
    level: int
    ncells: tuple
    lo: tuple
    hi: tuple
    id: int

    def dx(self, d: int) -> float:
        return (self.hi[d] - self.lo[d]) / self.ncells[d]  # grid.cpp:20-22


def _round_half_away(x: float) -> int:
    """std::round: halves away from zero (Python's round() rounds halves to even)."""
    r = math.trunc(x)
    if abs(x - r) >= 0.5:
        r += 1 if x > 0 else -1
    return int(r)


class RegridPlanner:
    """The tracking spheres and regrid parameters of an AMRHierarchy (amr.hpp:22-37).

    ``base_ncells``, ``domain_lo`` and ``domain_hi`` are the level-0 grid
    (SimulationParams::ncells, domain_lo, domain_hi); every child box carries
    ``base_ncells`` cells before merging, as in the reference.
    """

    def __init__(self, base_ncells, domain_lo, domain_hi, max_levels: int = 15, refinement_ratio: int = 2):
        self.base_ncells = tuple(int(n) for n in base_ncells)
        self.domain_lo = tuple(float(x) for x in domain_lo)
        self.domain_hi = tuple(float(x) for x in domain_hi)
        self.max_levels = int(max_levels)
        self.ratio = int(refinement_ratio)
        self.spheres: list[TrackingSphere] = []

    def add_tracking_sphere(self, center, radius: float, min_level: int):
        """AMRHierarchy::addTrackingSphere (amr.cpp:628-630)."""
        self.spheres.append(TrackingSphere(tuple(float(c) for c in center), float(radius), int(min_level)))

    def update_tracking_spheres(self, new_centers):
        """AMRHierarchy::updateTrackingSpheres (amr.cpp:632-636): the first
        min(len(spheres), len(new_centers)) spheres move."""
        for s, c in zip(self.spheres, new_centers):
            s.center = tuple(float(x) for x in c)

    def deepest_required(self) -> int:
        """The level initialize() cascades down to (amr.cpp:68-71)."""
        d = max([s.min_level for s in self.spheres], default=0)
        return min(d, self.max_levels - 1)

    def spheres_require(self, next_level: int) -> bool:
        return any(next_level <= s.min_level for s in self.spheres)

    def plan(self, level: int, blocks) -> list[Box]:
        """New blocks on level + 1 when the reference regrids ``level`` with
        refinement active (a sphere requires level + 1, or the tagger fired).

        ``blocks`` is the hierarchy's block list (objects with ``level``,
        ``ncells``, ``lo``, ``hi`` and ``dx(d)``), each level in creation order.
        Returns the boxes in the order the reference creates them, with the
        reference's block ids.
        """
        parents = [b for b in blocks if b.level == level]
        next_level = level + 1
        if not parents or self.max_levels <= 1 or next_level >= self.max_levels:
            return []
        parent_dx = [parents[0].dx(d) for d in range(3)]
        child_dx = [parent_dx[d] / float(self.ratio) for d in range(3)]
        half_width = [0.5 * float(self.base_ncells[d]) * child_dx[d] for d in range(3)]
        lo_dom, hi_dom = self.domain_lo, self.domain_hi

        # one candidate per sphere that requires the new level (amr.cpp:160-191)
        cands = []
        for s in self.spheres:
            if next_level > s.min_level:
                continue
            lo, hi = [0.0] * 3, [0.0] * 3
            for d in range(3):
                ext = float(self.base_ncells[d]) * child_dx[d]
                ideal = s.center[d] - half_width[d]
                lo[d] = math.floor((ideal - lo_dom[d]) / parent_dx[d]) * parent_dx[d] + lo_dom[d]
                hi[d] = lo[d] + ext
                if lo[d] < lo_dom[d]:
                    lo[d] = lo_dom[d]
                    hi[d] = lo[d] + ext
                if hi[d] > hi_dom[d]:
                    hi[d] = hi_dom[d]
                    lo[d] = hi[d] - ext
                    if lo[d] < lo_dom[d]:
                        lo[d] = lo_dom[d]
            cands.append([lo, hi])
        if not cands:
            return []

        # merge boxes that overlap or touch within one fine cell, restarting the
        # scan after every merge; the merged-away box is replaced by the last one
        # (amr.cpp:200-235)
        tol = child_dx[0]
        merged = True
        while merged:
            merged = False
            for a in range(len(cands)):
                for b in range(a + 1, len(cands)):
                    A, B = cands[a], cands[b]
                    if any(A[0][d] > B[1][d] + tol or B[0][d] > A[1][d] + tol for d in range(3)):
                        continue
                    for d in range(3):
                        A[0][d] = max(min(A[0][d], B[0][d]), lo_dom[d])
                        A[1][d] = min(max(A[1][d], B[1][d]), hi_dom[d])
                    cands[b] = cands[-1]
                    cands.pop()
                    merged = True
                    break
                if merged:
                    break

        # one block per merged box that no block of the new level duplicates,
        # blocks created earlier in this pass included (same spacing and first
        # cell centre within 0.1 cells; amr.cpp:243-268)
        existing = [(tuple(b.dx(d) for d in range(3)), tuple(b.lo)) for b in blocks if b.level == next_level]
        id_base = 1000 * next_level + len(existing)
        out = []
        for bi, (lo, hi) in enumerate(cands):
            n = tuple(max(_round_half_away((hi[d] - lo[d]) / child_dx[d]), 1) for d in range(3))
            dup = any(all(abs(edx[d] - child_dx[d]) <= 1e-10 * child_dx[d]
                          and abs((elo[d] + 0.5 * edx[d]) - (lo[d] + 0.5 * child_dx[d])) <= 0.1 * child_dx[d]
                          for d in range(3))
                      for edx, elo in existing)
            if dup:
                continue
            box = Box(next_level, n, tuple(lo), tuple(hi), id_base + bi)
            out.append(box)
            existing.append((tuple(box.dx(d) for d in range(3)), box.lo))
        return out

    def initial_layout(self) -> list[Box]:
        """The blocks AMRHierarchy::initialize builds (amr.cpp:34-78): one level-0
        block over the domain, then a regrid of levels 0, 1, ... down to the
        deepest level a sphere requires, stopping at the first level that gets
        no block."""
        blocks = [Box(0, self.base_ncells, self.domain_lo, self.domain_hi, 0)]
        for lev in range(self.deepest_required()):
            new = self.plan(lev, blocks) if self.spheres_require(lev + 1) else []
            blocks += new
            if not any(b.level == lev + 1 for b in blocks):
                break
        return blocks
