"""Checkpoint / restart of the resident state on the GPU.

A hierarchy stepped k coarse steps, checkpointed, and stepped further equals,
bit for bit, a fresh context restored from the checkpoint and stepped the same
way: state of every block (ghosts included), level times, resident matter
sources, blocks added by a regrid. Mismatching contexts are refused.
"""
import numpy as np
import pytest

import oracle
from oracle import Geom

pytestmark = pytest.mark.gpu

BL_M = [0.5, 0.5]
BL_X = [[1.5, 0.0, 0.0], [-1.5, 0.0, 0.0]]
N, LO, HI = (16, 16, 16), (-8.0, -8.0, -8.0), (8.0, 8.0, 8.0)
SPHERES = [((1.5, 0.0, 0.0), 2.0, 2), ((-1.5, 0.0, 0.0), 2.0, 2)]


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def build(gb, matter=False, variant=None):
    from granite_b200.regrid import RegridPlanner
    planner = RegridPlanner(N, LO, HI)
    for c, r, m in SPHERES:
        planner.add_tracking_sphere(c, r, m)
    ev = gb.Evolver(gb.CCZ4Params(), variant)
    if matter:
        ev.enable_matter()
    o = oracle.Oracle()
    for i, bx in enumerate(planner.initial_layout()):
        b = gb.GridBlock(bx.id, bx.level, bx.ncells, bx.lo, bx.hi)
        g = Geom(bx.ncells, bx.lo, bx.hi)
        b.array[...] = o.init_brill_lindquist(g, BL_M, BL_X, r_floor=0.5 * g.dx[0]) + \
            1e-8 * oracle.hash_noise(g.shape, 600 + i)
        ev.add_block(b)
    ev.commit()
    ev.upload()
    if matter:
        for i, b in enumerate(ev.blocks):
            g = Geom(b.ncells, b.lo, b.hi)
            prim = oracle.seeded_primitives(g, 30 + i)
            prim[0] *= 1e-3
            prim[4] *= 1e-4
            prim[5:8] *= 1e-2
            ev.upload_primitives(i, prim)
    return planner, ev


def states(ev):
    ev.download()
    return [b.array.copy() for b in ev.blocks]


@pytest.mark.parametrize("mode", ["ghosts", "reference"])
@pytest.mark.parametrize("matter", [False, True])
def test_restart_continues_bit_for_bit(gb, tmp_path, mode, matter):
    amr = gb.AMR_GHOSTS if mode == "ghosts" else gb.AMR_REFERENCE
    planner, ev = build(gb, matter)
    dt = 0.125
    for _ in range(2):
        ev.hierarchy_step(dt, gb.PRECISION_FP64, amr)
    planner.update_tracking_spheres([(2.5, 0.5, 0.0), (-2.5, -0.5, 0.0)])
    ev.regrid(planner, 1)
    ev.regrid(planner, 0)
    path = str(tmp_path / "ck.bin")
    ev.checkpoint_write(path, step=2, time=2 * dt)
    for _ in range(2):
        ev.hierarchy_step(dt, gb.PRECISION_MIXED, amr)
    want = states(ev)
    times = [ev.level_time(L) for L in range(3)]

    ev2, step, t = gb.Evolver.from_checkpoint(path)
    assert (step, t) == (2, 2 * dt)
    assert [(b.level, b.ncells, b.lo, b.hi) for b in ev2.blocks] == \
        [(b.level, b.ncells, b.lo, b.hi) for b in ev.blocks]
    for _ in range(2):
        ev2.hierarchy_step(dt, gb.PRECISION_MIXED, amr)
    got = states(ev2)
    for i, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"block {i}"
    assert [ev2.level_time(L) for L in range(3)] == times
    ev.close()
    ev2.close()


def test_restart_refuses_other_layouts(gb, tmp_path):
    _, ev = build(gb)
    path = str(tmp_path / "ck.bin")
    ev.checkpoint_write(path)
    other = gb.Evolver(gb.CCZ4Params())
    for b in ev.blocks[:-1]:
        other.add_block(gb.GridBlock(b.id, b.level, b.ncells, b.lo, b.hi))
    other.commit()
    with pytest.raises(gb.GraniteError):  # one block fewer
        other.checkpoint_read(path)
    _, ev_m = build(gb, matter=True)
    with pytest.raises(gb.GraniteError):  # matter in the context, not in the file
        ev_m.checkpoint_read(path)
    for e in (ev, other, ev_m):
        e.close()
