"""Device regrid against the reference regrid and the oracle.

* ``granite_ccz4_tag_count`` against the oracle's gradient taggers
  (amr.cpp:653-731), summed over a level's blocks: equal counts.
* ``Evolver.regrid`` (host planning + ``granite_ccz4_regrid_add``) against the
  compiled reference's AMRHierarchy::regrid (amr.cpp:80-301) on the same state:
  the same blocks, every cell (ghosts included) bit for bit; and against the
  oracle's prolongation (amr.cpp:484-564) of the coarse level's last block.
* The regridded hierarchy keeps stepping: two coarse steps after a regrid
  against the hierarchy oracle on the new layout, with the per-point bound of
  test_parity_gpu.py.
* The in-step regrid of subcycle (amr.cpp:343-349) through
  ``granite_ccz4_hierarchy_step_regrid``: blocks created between substeps,
  against the oracle's restated subcycle with the same hook (itself pinned bit
  for bit to the compiled AMRHierarchy in test_regrid_cpu.py), and the level
  times.
"""
import numpy as np
import pytest

import oracle
from oracle import Geom, Params
from oracle.hierarchy import HierarchyOracle
from oracle.hierarchy import tag_count as oracle_tag_count

from test_parity_gpu import VARIANTS, parity

pytestmark = pytest.mark.gpu

BL_M = [0.5, 0.5]
BL_X = [[1.5, 0.0, 0.0], [-1.5, 0.0, 0.0]]
N, LO, HI = (16, 16, 16), (-8.0, -8.0, -8.0), (8.0, 8.0, 8.0)
SPHERES = [((1.5, 0.0, 0.0), 2.0, 2), ((-1.5, 0.0, 0.0), 2.0, 2)]
MOVED = [(2.5, 0.5, 0.0), (-2.5, -0.5, 0.0)]


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def geom(b):
    return Geom(tuple(b.ncells), tuple(b.lo), tuple(b.hi))


def state(g, i):
    u = oracle.Oracle().init_brill_lindquist(g, BL_M, BL_X, r_floor=0.5 * g.dx[0])
    return u + 1e-8 * oracle.hash_noise(g.shape, 300 + i)


def setup(gb, variant=None):
    from granite_b200.regrid import RegridPlanner
    planner = RegridPlanner(N, LO, HI)
    for c, r, m in SPHERES:
        planner.add_tracking_sphere(c, r, m)
    ev = gb.Evolver(gb.CCZ4Params(), variant)
    for bx in planner.initial_layout():
        b = gb.GridBlock(bx.id, bx.level, bx.ncells, bx.lo, bx.hi)
        b.array[...] = state(geom(b), len(ev.blocks))
        ev.add_block(b)
    ev.commit()
    ev.upload()
    return planner, ev


def level_order(blocks):
    return sorted(range(len(blocks)), key=lambda i: (blocks[i].level, i))


@pytest.mark.parametrize("var", [0, 18])
def test_tag_count_matches_oracle(gb, var):
    _, ev = setup(gb)
    for level in range(3):
        for t in (0.02, 0.3, 1.5, 6.0):
            want = sum(oracle_tag_count(geom(b), b.array, var, t) for b in ev.blocks if b.level == level)
            assert ev.tag_count(level, var, t) == want, (level, t)
    ev.close()


def test_tag_count_rejects_other_fields(gb):
    _, ev = setup(gb)
    with pytest.raises(gb.GraniteError):
        ev.tag_count(0, 5, 0.1)
    ev.close()


@pytest.mark.parametrize("variant", [0, 4])
def test_regrid_matches_reference(gb, variant):
    planner, ev = setup(gb, variant)
    rh = None
    if oracle.reference_available("strict"):
        from oracle.hierarchy import RefHierarchy
        rh = RefHierarchy(oracle.Reference("strict"), N, LO, HI, SPHERES)
        order = level_order(ev.blocks)
        assert [(ev.blocks[i].level, tuple(ev.blocks[i].ncells)) for i in order] == \
            [(lv, tuple(g.n)) for g, lv in zip(rh.geoms, rh.levels)]
        for r, i in enumerate(order):
            rh.set(r, ev.blocks[i].array)
    planner.update_tracking_spheres(MOVED)
    if rh is not None:
        rh.update_spheres(MOVED)
    o = oracle.Oracle()
    total_new = 0
    for level in (1, 0, 1):
        coarse = [b for b in ev.blocks if b.level == level]
        new = ev.regrid(planner, level)
        total_new += len(new)
        ev.download()
        # every new block is the prolongation of the coarse level's last block
        # as it stood before this regrid (new coarse blocks come from earlier calls)
        for b in new:
            want = o.prolongate(geom(coarse[-1]), coarse[-1].array, geom(b), np.zeros(b.array.shape))
            assert np.array_equal(b.array, want), f"new block {b.id} vs oracle prolongation"
        if rh is not None:
            rh.regrid(level)
            order = level_order(ev.blocks)
            assert len(order) == len(rh.geoms)
            for r, i in enumerate(order):
                b = ev.blocks[i]
                assert (b.level, tuple(b.ncells), tuple(b.lo), tuple(b.hi)) == \
                    (rh.levels[r], tuple(rh.geoms[r].n), tuple(rh.geoms[r].lo), tuple(rh.geoms[r].hi))
                assert np.array_equal(b.array, rh.get(r)), f"block {b.id} after regrid({level})"
    assert total_new == 3
    ev.close()


def test_regrid_without_sphere_or_tag_adds_nothing(gb):
    planner, ev = setup(gb)
    n = len(ev.blocks)
    assert ev.regrid(planner, 2) == []                       # no sphere requires level 3
    assert ev.regrid(planner, 2, tagger=(0, 0.02)) == []     # tagged, but no box to place
    assert ev.tag_count(2, 0, 0.02) > 0
    assert len(ev.blocks) == n
    ev.close()


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("mode", ["reference", "ghosts"])
def test_step_after_regrid_matches_oracle(gb, oracle_lib, variant, mode):
    planner, ev = setup(gb, variant)
    amr = gb.AMR_REFERENCE if mode == "reference" else gb.AMR_GHOSTS
    dt = 0.25 * (HI[0] - LO[0]) / N[0]
    ev.hierarchy_step(dt, gb.PRECISION_FP64, amr)
    planner.update_tracking_spheres(MOVED)
    ev.regrid(planner, 1)
    ev.regrid(planner, 0)
    ev.download()
    geoms = [geom(b) for b in ev.blocks]
    levels = [b.level for b in ev.blocks]
    ho = HierarchyOracle(geoms, levels, oracle_lib)
    for i, b in enumerate(ev.blocks):
        ho.u[i][...] = b.array
    ho.step(Params(), dt, mode, 2)
    for _ in range(2):
        ev.hierarchy_step(dt, gb.PRECISION_FP64, amr)
    ev.download()
    for i, b in enumerate(ev.blocks):
        parity(b.array, ho.u[i], rtol=1e-10, what=f"{mode} block {i} level {levels[i]} after regrid")
    ev.close()


@pytest.mark.parametrize("interval", [1, 2])
@pytest.mark.parametrize("mode", ["reference", "ghosts"])
def test_in_step_regrid_matches_oracle(gb, oracle_lib, interval, mode):
    """Two coarse steps of subcycle with its in-step regrid after the spheres
    moved (new level-2 blocks appear between level-1 steps, a new level-1 block
    at the end of the coarse step): the device hierarchy against the oracle's
    restated subcycle with the same regrid hook, block for block."""
    from test_regrid_cpu import oracle_regrid_hook
    planner, ev = setup(gb)
    ho = HierarchyOracle([geom(b) for b in ev.blocks], [b.level for b in ev.blocks], oracle_lib)
    for i, b in enumerate(ev.blocks):
        ho.u[i][...] = b.array
    planner.update_tracking_spheres(MOVED)
    ho.regrid_interval = interval
    ho.regrid_hook = oracle_regrid_hook(planner)
    n0 = len(ev.blocks)
    dt = 0.25 * (HI[0] - LO[0]) / N[0]
    ho.step(Params(), dt, mode, 2)
    amr = gb.AMR_REFERENCE if mode == "reference" else gb.AMR_GHOSTS
    for _ in range(2):
        ev.hierarchy_step_regrid(dt, planner, interval, amr_mode=amr)
    assert len(ev.blocks) > n0
    assert [(b.level, geom(b)) for b in ev.blocks] == list(zip(ho.levels, ho.geoms))
    ev.download()
    for i, b in enumerate(ev.blocks):
        parity(b.array, ho.u[i], rtol=1e-10, what=f"{mode} block {i} level {b.level} (in-step regrid)")
    assert [ev.level_time(L) for L in range(ho.nlev)] == ho.time
    ev.close()


def test_level_times_and_callback_errors(gb):
    planner, ev = setup(gb)
    dt = 0.125
    ev.hierarchy_step(dt, gb.PRECISION_FP64, gb.AMR_GHOSTS)
    ev.hierarchy_step(dt, gb.PRECISION_FP64, gb.AMR_GHOSTS)
    want = []
    for L in range(3):
        t, h = 0.0, dt / 2 ** L
        for _ in range(2 * 2 ** L):
            t += h
        want.append(t)
    assert [ev.level_time(L) for L in range(3)] == want
    with pytest.raises(AttributeError):  # the callback's own exception comes back
        ev.hierarchy_step_regrid(dt, None, 1, amr_mode=gb.AMR_GHOSTS)
    ev.close()
