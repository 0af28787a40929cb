"""Seeded, static Berger-Oliger block hierarchies for the hierarchy workloads.

The reference builds one block per tracking sphere and level (amr.cpp:80-301).
The hierarchy workloads instead need many uneven blocks per level, so this
module lays them out itself: level L covers a cube centred on the origin whose
edge halves with every level (ratio-2 refinement, amr.cpp:389-398) while its
cell count stays the same, and that cube is tiled by non-overlapping blocks
whose edge lengths are drawn, per axis, from a size set (a tensor product of
three random compositions of the level's cell count), with the block count per
level drawn into a requested range. Levels nest with a margin of at least two
coarse cells, every block corner lies on its level's cell grid, and blocks
follow level order. These workload layouts are static (the benchmarks do not
regrid); the reference's tracking-sphere regrid is in regrid.py.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class BlockSpec:
    level: int
    ncells: tuple
    lo: tuple
    hi: tuple


@dataclass
class Hierarchy:
    blocks: list = field(default_factory=list)
    level_box: list = field(default_factory=list)     # (lo[3], hi[3]) per level
    level_dx: list = field(default_factory=list)      # cell spacing per level
    level_cells: list = field(default_factory=list)   # cells per axis per level
    masses: list = field(default_factory=list)
    positions: list = field(default_factory=list)

    @property
    def num_levels(self) -> int:
        return len(self.level_box)

    def interior_points(self, level=None) -> int:
        return int(sum(np.prod(b.ncells) for b in self.blocks if level is None or b.level == level))

    def point_updates_per_coarse_step(self) -> int:
        """Sum over levels of interior points x the 2^L substeps of that level."""
        return int(sum(self.interior_points(L) * 2 ** L for L in range(self.num_levels)))

    def cells_with_ghosts(self, ng: int = 4) -> int:
        return int(sum(np.prod([n + 2 * ng for n in b.ncells]) for b in self.blocks))


def _composition(total: int, sizes, rng, max_tries: int = 1000):
    """Random ordered composition of `total` into parts from `sizes`."""
    sizes = sorted(sizes)
    smin = sizes[0]
    for _ in range(max_tries):
        parts, rem = [], total
        while rem > 0:
            ok = [s for s in sizes if s == rem or (s < rem and rem - s >= smin)]
            if not ok:
                break
            s = int(rng.choice(ok))
            parts.append(s)
            rem -= s
        if rem == 0:
            return parts
    raise ValueError(f"cannot compose {total} from {sizes}")


def make_hierarchy(seed: int, levels: int, coarse_n: int, extent: float, sizes, blocks_per_level,
                   masses=(), positions=()) -> Hierarchy:
    """Nested cubes [-extent/2^L, extent/2^L]^3 of coarse_n^3 cells each, tiled by
    blocks with edges from `sizes`, block count per level in blocks_per_level."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo_n, hi_n = blocks_per_level
    h = Hierarchy(masses=list(masses), positions=[list(p) for p in positions])
    for L in range(levels):
        half = extent / 2 ** L
        dx = 2.0 * half / coarse_n
        for _ in range(10000):
            comps = [_composition(coarse_n, sizes, rng) for _ in range(3)]
            count = len(comps[0]) * len(comps[1]) * len(comps[2])
            if lo_n <= count <= hi_n:
                break
        else:
            raise ValueError("no tiling with the requested block count")
        edges = [np.concatenate([[0], np.cumsum(c)]) for c in comps]
        for k in range(len(comps[2])):
            for j in range(len(comps[1])):
                for i in range(len(comps[0])):
                    idx = (i, j, k)
                    lo = tuple(-half + edges[d][idx[d]] * dx for d in range(3))
                    hi = tuple(-half + edges[d][idx[d] + 1] * dx for d in range(3))
                    n = tuple(int(comps[d][idx[d]]) for d in range(3))
                    h.blocks.append(BlockSpec(L, n, lo, hi))
        h.level_box.append(((-half,) * 3, (half,) * 3))
        h.level_dx.append(dx)
        h.level_cells.append((coarse_n,) * 3)
    return h


def make_binary_hierarchy(seed: int = 2024, levels: int = 4, coarse_n: int = 128, extent: float = 64.0,
                          sizes=(16, 24, 32, 48, 64), blocks_per_level=(80, 400)) -> Hierarchy:
    """Binary Brill-Lindquist punctures (m = 0.5 at x = +-3) on the 4-level
    workload: coarse dx = 1 on [-64, 64]^3, 80-400 blocks per level with edges
    from {16, 24, 32, 48, 64}."""
    return make_hierarchy(seed, levels, coarse_n, extent, sizes, blocks_per_level,
                          masses=(0.5, 0.5), positions=((3.0, 0.0, 0.0), (-3.0, 0.0, 0.0)))


def make_triple_hierarchy(seed: int = 7, levels: int = 6, coarse_n: int = 216, extent: float = 256.0,
                          sizes=(16, 24, 32, 40, 48, 56, 64, 72, 80, 88, 96),
                          blocks_per_level=(250, 420)) -> Hierarchy:
    """Three Brill-Lindquist punctures (0.4 / 0.35 / 0.25 at seeded positions with
    r < 6) on 6 levels of 216^3 cells (~60M interior points, ~2000 blocks)."""
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    pos = []
    while len(pos) < 3:
        p = rng.uniform(-6.0, 6.0, size=3)
        if np.linalg.norm(p) < 6.0:
            pos.append(tuple(float(x) for x in p))
    return make_hierarchy(seed, levels, coarse_n, extent, sizes, blocks_per_level,
                          masses=(0.4, 0.35, 0.25), positions=pos)


def block_states(h: Hierarchy, noise: float = 0.0, seed: int = 12345, r_floor_cells: float = 0.5):
    """GridBlocks of the hierarchy with Brill-Lindquist data of its punctures
    (r floored at r_floor_cells x the block's dx) and optional U(-a, a) noise."""
    from . import GridBlock
    from .initial_data import add_noise, brill_lindquist
    out = []
    for i, b in enumerate(h.blocks):
        g = GridBlock(i, b.level, b.ncells, b.lo, b.hi)
        brill_lindquist(g, h.masses, h.positions, r_floor=r_floor_cells * g.dx(0))
        if noise > 0.0:
            add_noise(g, noise, seed + i)
        out.append(g)
    return out
