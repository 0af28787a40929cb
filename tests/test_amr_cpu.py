"""granite_b200.amr.AMRHierarchy on the CPU: the layout against the compiled
reference AMRHierarchy, and the host logic around the device (dt per level,
when the state moves between host and device, which entry point a step takes,
the errors) with a stand-in for the device Evolver that records its calls."""
import numpy as np
import pytest

from oracle.hierarchy import RefHierarchy
from granite_b200 import (AMR_GHOSTS, AMR_REFERENCE, PRECISION_FP64, PRECISION_MIXED, Evolver, GraniteError,
                          GridBlock)
from granite_b200.amr import (AMRHierarchy, AMRParams, SimulationParams, compositeTagger, gradientChiTagger,
                              gradientLapseTagger)
from granite_b200.regrid import CHI, LAPSE

SIM = SimulationParams(ncells=(16, 16, 16), domain_lo=(-8.0, -8.0, -8.0), domain_hi=(8.0, 8.0, 8.0))


class FakeEvolver:
    """Records the Evolver calls AMRHierarchy makes; ``grow`` adds one block on a
    new level at the next in-step regrid, as a regrid creating a level would."""

    def __init__(self, grow=False):
        self.blocks, self.calls, self.grow, self.closed = [], [], grow, False

    def add_block(self, b):
        self.calls.append(("add", b.id))
        self.blocks.append(b)

    def commit(self):
        self.calls.append(("commit",))

    def upload(self):
        self.calls.append(("upload", len(self.blocks)))

    def download(self):
        self.calls.append(("download", len(self.blocks)))
        for b in self.blocks:
            b.array[:] = 7.0

    def hierarchy_step(self, dt, precision, mode):
        self.calls.append(("step", dt, precision, mode))

    def hierarchy_step_regrid(self, dt, planner, interval, tagger, precision, mode):
        self.calls.append(("step_regrid", dt, interval, tagger, precision, mode))
        if not self.grow:
            return []
        top = max(b.level for b in self.blocks)
        p = [b for b in self.blocks if b.level == top][0]
        c = [0.5 * (p.lo[d] + p.hi[d]) for d in range(3)]
        w = [0.25 * (p.hi[d] - p.lo[d]) for d in range(3)]
        nb = GridBlock(1000 * (top + 1), top + 1, p.ncells, [c[d] - w[d] for d in range(3)],
                       [c[d] + w[d] for d in range(3)])
        self.blocks.append(nb)
        return [nb]

    def level_time(self, level):
        return 0.5 * level

    # the real Evolver.regrid host logic over stand-in device calls
    def tag_count(self, level, var, threshold):
        self.calls.append(("tag_count", level, var, threshold))
        return 0

    def regrid_add(self, blocks):
        self.calls.append(("regrid_add", [b.id for b in blocks]))
        self.blocks.extend(blocks)

    def regrid(self, planner, level, tagger=None):
        return Evolver.regrid(self, planner, level, tagger)

    def close(self):
        self.closed = True


def make(sphere=((1.0, -0.5, 0.25), 2.0, 2), interval=0, grow=False, **kw):
    fakes = []

    def factory():
        fakes.append(FakeEvolver(grow))
        return fakes[-1]

    h = AMRHierarchy(AMRParams(max_levels=4, regrid_interval=interval), SIM, evolver_factory=factory, **kw)
    if sphere:
        h.addTrackingSphere(*sphere)
    h.initialize(gradientChiTagger(0.1))
    return h, fakes


@pytest.mark.parametrize("spheres,max_levels", [([((1.0, -0.5, 0.25), 2.0, 2)], 4),
                                                ([((3.0, 3.0, 0.0), 1.0, 3), ((-3.0, 2.0, 1.0), 1.5, 1)], 5),
                                                ([((0.0, 0.0, 0.0), 1.0, 6)], 3), ([], 4)])
def test_initialize_matches_the_compiled_hierarchy(reference_lib, spheres, max_levels):
    h = AMRHierarchy(AMRParams(max_levels=max_levels), SIM, evolver_factory=FakeEvolver)
    for s in spheres:
        h.addTrackingSphere(*s)
    h.initialize()
    ref = RefHierarchy(reference_lib, SIM.ncells, SIM.domain_lo, SIM.domain_hi, spheres, max_levels)
    got = [(b.level, b.ncells, b.lo, b.hi) for b in h.getAllBlocks()]
    assert got == [(lv, g.n, g.lo, g.hi) for g, lv in zip(ref.geoms, ref.levels)]
    assert h.numBlocks() == len(ref.levels) and h.numLevels() == max(ref.levels) + 1
    assert h.effectiveResolution((0.0, 0.0, 0.0)) == 1.0
    for lv in range(h.numLevels()):
        assert [b.level for b in h.getLevel(lv)] == [lv] * ref.levels.count(lv)


def test_set_level_dt_halves_per_level():
    h, _ = make()
    assert h.numLevels() == 3
    h.setLevelDt(0, 0.4)
    assert [h.levelDt(lv) for lv in range(3)] == [0.4, 0.2, 0.1]
    h.setLevelDt(5, 1.0)  # no such level: ignored, as amr.cpp:389-391
    h.setLevelDt(1, 0.3)
    assert [h.levelDt(lv) for lv in range(3)] == [0.4, 0.3, 0.15]
    with pytest.raises(GraniteError):  # the device needs dt(0) / 2^L
        h.subcycle(0)


def test_state_moves_once_each_way_per_access():
    h, fakes = make(precision=PRECISION_MIXED, amr_mode=AMR_GHOSTS)
    h.setLevelDt(0, 0.25)
    blocks0 = h.getAllBlocks()
    for b in blocks0:
        b.array[:] = 1.0  # initial data written on the host
    assert h.subcycle(0) == []
    ev = fakes[0]
    assert [c[0] for c in ev.calls] == ["add"] * 3 + ["commit", "upload", "step"]
    assert [c[1] for c in ev.calls[:3]] == [b.id for b in blocks0]  # level order
    assert ev.calls[-1] == ("step", 0.25, PRECISION_MIXED, AMR_GHOSTS)
    h.subcycle(0)  # nothing handed out since: no transfer
    assert [c[0] for c in ev.calls[6:]] == ["step"]
    blocks = h.getLevel(1)  # stale host: one download, then the blocks are handed out
    assert [c[0] for c in ev.calls[7:]] == ["download"] and np.all(blocks[0].array == 7.0)
    h.getLevel(0)  # already current
    h.subcycle(0)  # handed-out blocks go back before the step
    assert [c[0] for c in ev.calls[8:]] == ["upload", "step"]
    assert h.currentTime(2) == 1.0 and len(fakes) == 1


def test_in_step_regrid_path_and_new_levels():
    h, fakes = make(interval=2, grow=True)
    h.setLevelDt(0, 0.5)
    tg = compositeTagger([gradientChiTagger(0.1), gradientLapseTagger(0.2)])
    assert tg == [(CHI, 0.1), (LAPSE, 0.2)]
    added = h.subcycle(0, None, tg)
    assert [b.level for b in added] == [3] and h.numLevels() == 4 and h.numBlocks() == 4
    assert fakes[0].calls[-1] == ("step_regrid", 0.5, 2, tg, PRECISION_FP64, AMR_REFERENCE)
    assert [h.levelDt(lv) for lv in range(4)] == [0.5, 0.25, 0.125, 0.0625]  # amr.cpp:137-143
    assert h.getLevel(3)[0] is added[0]


def test_errors_and_reinitialize():
    h, fakes = make()
    with pytest.raises(GraniteError):
        h.subcycle(1)
    with pytest.raises(GraniteError):
        h.subcycle(0, lambda blocks, dt: None)
    h.setLevelDt(0, 0.1)
    h.subcycle(0)
    h.initialize()  # a new layout drops the device hierarchy
    assert fakes[0].closed
    h.setLevelDt(0, 0.1)
    h.subcycle(0)
    assert len(fakes) == 2
    empty = AMRHierarchy(AMRParams(), SIM, evolver_factory=FakeEvolver)
    with pytest.raises(GraniteError):
        empty.subcycle(0)
    with pytest.raises(GraniteError):
        AMRHierarchy(AMRParams(refinement_ratio=4), SIM)
    with pytest.raises(GraniteError):
        AMRHierarchy(AMRParams(), SimulationParams(ghost_cells=3))


def test_reference_amr_smoke_tests():
    """tests/amr/test_amr_basic.cpp:85-205 of GRANITE (T1 construction, T2 one
    level without spheres, T5 a regrid with nothing tagged keeps the level count)
    on this AMRHierarchy; T3 / T4 (constant-field prolongation / restriction)
    are device transfers, pinned through the oracle's known answers."""
    params = AMRParams(max_levels=3, refinement_ratio=2, regrid_interval=4)
    sim = SimulationParams(ncells=(8, 8, 8), domain_lo=(-1.0, -1.0, -1.0), domain_hi=(1.0, 1.0, 1.0),
                           ghost_cells=4)
    AMRHierarchy(params, sim, evolver_factory=FakeEvolver)
    h = AMRHierarchy(params, sim, evolver_factory=FakeEvolver)
    h.initialize()
    assert h.numLevels() >= 1
    fakes = []
    h = AMRHierarchy(params, sim, evolver_factory=lambda: fakes.append(FakeEvolver()) or fakes[-1])
    h.addTrackingSphere((0.0, 0.0, 0.0), 1.0, 2)
    h.initialize()
    h.getLevel(0)[0].array[:] = 0.0
    before = h.numLevels()
    assert h.regrid(0, None) == [] and h.numLevels() == before == 3
    assert not any(c[0] == "tag_count" or (c[0] == "regrid_add" and c[1]) for c in fakes[0].calls)
    assert h.regrid(2, gradientChiTagger(0.1)) == []  # level 3 is beyond max_levels
    h2 = AMRHierarchy(params, sim, evolver_factory=lambda: fakes.append(FakeEvolver()) or fakes[-1])
    h2.initialize()
    assert h2.regrid(0, gradientChiTagger(0.1)) == [] and h2.numLevels() == 1
    assert ("tag_count", 0, CHI, 0.1) in fakes[1].calls  # no sphere: the tagger is asked
