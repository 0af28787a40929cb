"""Hierarchy oracle pins (CPU).

The restated Berger-Oliger step (oracle/hierarchy.py, "reference" mode) is
checked bit for bit against the compiled reference's own AMRHierarchy
(tracking spheres, subcycle; amr.cpp:34-350) stepped with the same RK3
evolve_func. The seeded block-hierarchy generator of the product is checked for
the properties the transfer lists rely on.
"""
import numpy as np

import oracle
from oracle import Params
from oracle.hierarchy import HierarchyOracle, RefHierarchy

BL_M = [0.5, 0.5]
BL_X = [[1.5, 0.0, 0.0], [-1.5, 0.0, 0.0]]


def _ref_hier(reference_lib):
    return RefHierarchy(reference_lib, (16, 16, 16), (-8.0, -8.0, -8.0), (8.0, 8.0, 8.0),
                        [((1.5, 0.0, 0.0), 2.0, 2), ((-1.5, 0.0, 0.0), 2.0, 2)])


def test_reference_hierarchy_has_levels(reference_lib):
    rh = _ref_hier(reference_lib)
    assert max(rh.levels) == 2
    assert rh.levels[0] == 0


def test_oracle_reference_mode_equals_compiled_hierarchy(oracle_lib, reference_lib):
    rh = _ref_hier(reference_lib)
    ho = HierarchyOracle(rh.geoms, rh.levels, oracle_lib)
    for i, g in enumerate(rh.geoms):
        u = oracle_lib.init_brill_lindquist(g, BL_M, BL_X)
        u = u + 1e-8 * oracle.hash_noise(g.shape, 100 + i)
        rh.set(i, u)
        ho.u[i][...] = u
    dt = 0.25 * rh.geoms[0].dx[0]
    rh.step(Params(), dt, 2)
    ho.step(Params(), dt, "reference", 2)
    for i in range(len(rh.geoms)):
        assert np.array_equal(ho.u[i], rh.get(i)), f"block {i} (level {rh.levels[i]})"


def test_generator_properties():
    from granite_b200.hierarchy import make_binary_hierarchy
    h = make_binary_hierarchy(seed=7, levels=3, coarse_n=64, sizes=(8, 16, 24, 32),
                              blocks_per_level=(20, 80), extent=16.0)
    assert h.num_levels == 3
    for L in range(3):
        blocks = [b for b in h.blocks if b.level == L]
        assert 20 <= len(blocks) <= 80
        # non-overlapping, tiling the level's region
        vol = sum(np.prod(b.ncells) for b in blocks)
        assert vol == np.prod(h.level_cells[L])
        for b in blocks:
            assert all(n in (8, 16, 24, 32) for n in b.ncells)
    # nesting: every fine region lies inside the coarse region with a 2-cell margin
    for L in range(1, 3):
        lo_f, hi_f = h.level_box[L]
        lo_c, hi_c = h.level_box[L - 1]
        dxc = h.level_dx[L - 1]
        assert all(lo_f[d] >= lo_c[d] + 2 * dxc - 1e-12 and hi_f[d] <= hi_c[d] - 2 * dxc + 1e-12
                   for d in range(3))


def test_ghosts_plan_covers_every_fine_ghost_cell(oracle_lib):
    from granite_b200.hierarchy import make_binary_hierarchy
    h = make_binary_hierarchy(seed=3, levels=2, coarse_n=32, sizes=(8, 16), blocks_per_level=(8, 64),
                              extent=8.0)
    geoms = [oracle.Geom(b.ncells, b.lo, b.hi) for b in h.blocks]
    ho = HierarchyOracle(geoms, [b.level for b in h.blocks], oracle_lib)
    ho._plan()
    plan, rest = ho._ghost_plan
    for b, g in enumerate(geoms):
        if ho.levels[b] == 0:
            continue
        covered = np.zeros(g.shape[1:], dtype=bool)
        for _, m in plan[b][0]:
            assert not (covered & m.astype(bool)).any()
            covered |= m.astype(bool)
        ghost = np.ones(g.shape[1:], bool)
        ghost[g.interior()[1:]] = False
        assert np.array_equal(covered, ghost), f"fine block {b}: ghost cells without a coarse source"
    assert len(rest) > 0
