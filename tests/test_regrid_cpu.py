"""Regrid planning and the gradient taggers on the CPU.

* ``RegridPlanner`` (granite_b200/regrid.py) against the block layouts the
  compiled reference's AMRHierarchy produces (amr.cpp:34-301): after
  initialize() and after every tracking-sphere update and regrid of each
  scenario, corners and cell counts equal, block for block (golden file
  tests/golden/regrid_layouts.json, and the live reference where it is built).
  The scenarios cover merged and separate spheres, clamping at the domain
  faces and corners, unequal cell spacings per axis, spheres that moved (new
  blocks beside the old ones), duplicates that are skipped, and the
  max_levels cap.
* The oracle's numpy restatement of gradientChiTagger / gradientLapseTagger
  (amr.cpp:653-731) against the reference's own taggers.
"""
import json
import os

import numpy as np
import pytest

import oracle
from oracle import Geom
from oracle.hierarchy import tag_count as oracle_tag_count

from granite_b200.regrid import CHI, LAPSE, RegridPlanner

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "regrid_layouts.json")

SCENARIOS = [
    # two spheres merged at every level, then moved apart, then to the x faces
    dict(n=(16, 16, 16), lo=(-8.0, -8.0, -8.0), hi=(8.0, 8.0, 8.0), max_levels=15,
         spheres=[((1.5, 0.0, 0.0), 2.0, 2), ((-1.5, 0.0, 0.0), 2.0, 2)],
         ops=[("update", [(2.5, 0.5, 0.0), (-2.5, -0.5, 0.0)]), ("regrid", 1), ("regrid", 0), ("regrid", 1),
              ("regrid", 1), ("update", [(6.9, 0.0, 0.0), (-6.9, 0.0, 0.0)]), ("regrid", 0), ("regrid", 1),
              ("regrid", 2)]),
    # three spheres, unequal depths, max_levels cap, a sphere at the z face
    dict(n=(24, 20, 16), lo=(-12.0, -10.0, -8.0), hi=(12.0, 10.0, 8.0), max_levels=4,
         spheres=[((3.3, -1.7, 0.2), 1.5, 3), ((-4.1, 2.2, -0.6), 1.5, 2), ((0.0, 0.0, 7.9), 1.0, 1)],
         ops=[("update", [(3.9, -1.1, 0.4), (-4.6, 2.9, -1.3)]), ("regrid", 0), ("regrid", 1), ("regrid", 2),
              ("regrid", 3), ("update", [(3.3, -1.7, 0.2), (-4.1, 2.2, -0.6), (0.0, 0.0, -7.9)]),
              ("regrid", 0), ("regrid", 2), ("regrid", 1)]),
    # unequal spacings per axis (dx = 1, 2, 2), a sphere in a domain corner
    dict(n=(16, 12, 8), lo=(0.0, 0.0, -4.0), hi=(16.0, 24.0, 12.0), max_levels=15,
         spheres=[((8.0, 12.0, 4.0), 1.0, 2), ((1.0, 1.0, -3.0), 1.0, 1)],
         ops=[("update", [(8.7, 13.1, 4.9), (15.2, 23.0, 11.5)]), ("regrid", 0), ("regrid", 1),
              ("update", [(8.7, 13.1, 4.9)]), ("regrid", 0), ("regrid", 1)]),
]

BL_M = [0.5, 0.5]
BL_X = [[1.5, 0.0, 0.0], [-1.5, 0.0, 0.0]]
TAG_CASES = [dict(var=v, threshold=t, geom=gi) for gi in range(2) for v in (CHI, LAPSE)
             for t in (0.05, 0.3, 1.0, 4.0)]
TAG_GEOMS = [Geom((20, 16, 12), (-5.0, -4.0, -3.0), (5.0, 4.0, 3.0)),
             Geom((12, 12, 12), (0.25, -3.0, -3.0), (6.25, 3.0, 3.0))]


def tag_case_state(case):
    g = TAG_GEOMS[case["geom"]]
    u = oracle.Oracle().init_brill_lindquist(g, BL_M, BL_X, r_floor=0.5 * g.dx[0])
    return g, u + 1e-6 * oracle.hash_noise(g.shape, 77 + case["geom"])


def planner_layouts(sc):
    p = RegridPlanner(sc["n"], sc["lo"], sc["hi"], sc["max_levels"])
    for c, r, m in sc["spheres"]:
        p.add_tracking_sphere(c, r, m)
    blocks = p.initial_layout()

    def layout():
        # the reference lists blocks level by level, each level in creation order
        return [[b.level, list(b.ncells), list(b.lo), list(b.hi)]
                for lv in range(max(b.level for b in blocks) + 1) for b in blocks if b.level == lv]

    steps = [layout()]
    for op, arg in sc["ops"]:
        if op == "update":
            p.update_tracking_spheres(arg)
        elif p.spheres_require(arg + 1):
            blocks += p.plan(arg, blocks)
        steps.append(layout())
    return steps


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.mark.parametrize("si", range(len(SCENARIOS)))
def test_planner_matches_reference_layouts(si):
    got = planner_layouts(SCENARIOS[si])
    want = golden()["scenarios"][si]
    assert len(got) == len(want)
    for step, (g, w) in enumerate(zip(got, want)):
        assert g == w, f"scenario {si}, after op {step}: {g} != {w}"


def test_scenarios_exercise_merging_and_moves():
    """The golden layouts contain merged boxes (more than the base cell count),
    blocks added by moved spheres beside old ones, and regrids that add nothing."""
    sc = golden()["scenarios"]
    merged = any(n != list(SCENARIOS[i]["n"]) for i, steps in enumerate(sc) for lv, n, lo, hi in steps[-1] if lv > 0)
    grew = [len(b) - len(a) for steps in sc for a, b in zip(steps, steps[1:])]
    assert merged and max(grew) >= 1 and grew.count(0) >= 3


@pytest.mark.skipif(not oracle.reference_available("strict"), reason="reference library not built")
@pytest.mark.parametrize("si", range(len(SCENARIOS)))
def test_planner_matches_live_reference(si):
    from oracle.hierarchy import RefHierarchy
    sc = SCENARIOS[si]
    rh = RefHierarchy(oracle.Reference("strict"), sc["n"], sc["lo"], sc["hi"], sc["spheres"], sc["max_levels"])
    got = planner_layouts(sc)

    def layout():
        return [[lv, list(g.n), list(g.lo), list(g.hi)] for g, lv in zip(rh.geoms, rh.levels)]

    assert got[0] == layout()
    for step, (op, arg) in enumerate(sc["ops"], start=1):
        if op == "update":
            rh.update_spheres(arg)
        else:
            rh.regrid(arg)
        assert got[step] == layout(), f"after op {step}"


@pytest.mark.parametrize("ci", range(len(TAG_CASES)))
def test_oracle_tagger_golden(ci):
    case = TAG_CASES[ci]
    g, u = tag_case_state(case)
    assert oracle_tag_count(g, u, case["var"], case["threshold"]) == golden()["tags"][ci]


def test_tagger_cases_are_nontrivial():
    n = golden()["tags"]
    cells = [int(np.prod(TAG_GEOMS[c["geom"]].n)) for c in TAG_CASES]
    assert any(0 < t < c for t, c in zip(n, cells))
    assert len(set(n)) > len(TAG_GEOMS) * 2


@pytest.mark.skipif(not oracle.reference_available("strict"), reason="reference library not built")
@pytest.mark.parametrize("var", [CHI, LAPSE])
def test_oracle_tagger_matches_reference(var):
    ref = oracle.Reference("strict")
    for gi, g in enumerate(TAG_GEOMS):
        _, u = tag_case_state(dict(geom=gi))
        for t in (0.01, 0.2, 0.7, 2.5, 10.0):
            assert oracle_tag_count(g, u, var, t) == ref.tag_count(g, u, var, t)


def oracle_regrid_hook(planner, tagger=None):
    """The regrid of AMRHierarchy::regrid (amr.cpp:80-301) for HierarchyOracle's
    in-step hook: boxes from the planner, data by the oracle's prolongation."""
    from granite_b200.regrid import Box

    def hook(ho, level):
        if not planner.spheres_require(level + 1):
            return  # a tagger may fire here, but only spheres place boxes
        blocks = [Box(lv, g.n, g.lo, g.hi, 0) for g, lv in zip(ho.geoms, ho.levels)]
        boxes = planner.plan(level, blocks)
        ho.add_blocks([Geom(b.ncells, b.lo, b.hi) for b in boxes], [b.level for b in boxes])

    return hook


@pytest.mark.parametrize("interval", [1, 2, 3])
def test_oracle_in_step_regrid_equals_compiled_hierarchy(oracle_lib, reference_lib, interval):
    """Moving spheres, then two coarse steps with the reference's in-step regrid:
    the oracle (restated subcycle + planner + oracle prolongation) and the
    compiled AMRHierarchy end with the same blocks, bit for bit."""
    from oracle import Params
    from oracle.hierarchy import HierarchyOracle, RefHierarchy
    sc = SCENARIOS[0]
    rh = RefHierarchy(reference_lib, sc["n"], sc["lo"], sc["hi"], sc["spheres"], sc["max_levels"],
                      regrid_interval=interval)
    ho = HierarchyOracle(rh.geoms, rh.levels, oracle_lib)
    for i, g in enumerate(rh.geoms):
        u = oracle_lib.init_brill_lindquist(g, BL_M, BL_X) + 1e-8 * oracle.hash_noise(g.shape, 500 + i)
        rh.set(i, u)
        ho.u[i][...] = u
    planner = RegridPlanner(sc["n"], sc["lo"], sc["hi"], sc["max_levels"])
    for c, r, m in sc["spheres"]:
        planner.add_tracking_sphere(c, r, m)
    moved = [(2.5, 0.5, 0.0), (-2.5, -0.5, 0.0)]
    rh.update_spheres(moved)
    planner.update_tracking_spheres(moved)
    ho.regrid_interval = interval
    ho.regrid_hook = oracle_regrid_hook(planner)
    n0 = len(rh.geoms)
    dt = 0.25 * rh.geoms[0].dx[0]
    rh.step(Params(), dt, 2)
    ho.step(Params(), dt, "reference", 2)
    assert len(rh.geoms) > n0
    order = sorted(range(len(ho.geoms)), key=lambda i: (ho.levels[i], i))
    assert [(ho.levels[i], ho.geoms[i]) for i in order] == list(zip(rh.levels, rh.geoms))
    for r, i in enumerate(order):
        assert np.array_equal(ho.u[i], rh.get(r)), f"block {r} (level {rh.levels[r]})"


def test_planner_edge_cases():
    """Nothing to place without a parent level, beyond max_levels, or when no
    sphere reaches the level; a sphere wider than the domain is clamped to it;
    an initial layout without spheres is the single level-0 block."""
    from granite_b200.regrid import Box
    p = RegridPlanner((8, 8, 8), (0.0, 0.0, 0.0), (8.0, 8.0, 8.0), max_levels=2)
    base = p.initial_layout()
    assert [(b.level, b.ncells) for b in base] == [(0, (8, 8, 8))]
    p.add_tracking_sphere((4.0, 4.0, 4.0), 1.0, 5)
    assert p.plan(1, base) == []                        # no block on level 1
    lay = p.initial_layout()
    assert [b.level for b in lay] == [0, 1]             # capped at max_levels - 1
    assert p.plan(1, lay) == []                         # level 2 would exceed max_levels
    q = RegridPlanner((8, 8, 8), (0.0, 0.0, 0.0), (8.0, 8.0, 8.0), max_levels=4)
    q.add_tracking_sphere((0.1, 7.9, 4.0), 1.0, 1)
    lv1 = [b for b in q.initial_layout() if b.level == 1]
    assert len(lv1) == 1
    b = lv1[0]
    assert b.lo[0] == 0.0 and b.hi[1] == 8.0 and b.ncells == (8, 8, 8)  # clamped to the domain faces
    assert q.plan(1, [Box(0, (8, 8, 8), (0.0,) * 3, (8.0,) * 3, 0), b]) == []  # min_level 1: nothing finer


@pytest.mark.skipif(not oracle.reference_available("strict"), reason="reference library not built")
@pytest.mark.parametrize("sphere,max_levels", [(((0.1, 7.9, 4.0), 1.0, 1), 4), (((4.0, 4.0, 4.0), 1.0, 5), 2),
                                              (((7.5, 0.5, 7.5), 3.0, 3), 15)])
def test_planner_edge_layouts_match_reference(sphere, max_levels):
    from oracle.hierarchy import RefHierarchy
    rh = RefHierarchy(oracle.Reference("strict"), (8, 8, 8), (0.0,) * 3, (8.0,) * 3, [sphere], max_levels)
    p = RegridPlanner((8, 8, 8), (0.0,) * 3, (8.0,) * 3, max_levels=max_levels)
    p.add_tracking_sphere(*sphere)
    got = sorted(((b.level, b.ncells, b.lo, b.hi) for b in p.initial_layout()), key=lambda t: t[0])
    assert got == [(lv, g.n, g.lo, g.hi) for g, lv in zip(rh.geoms, rh.levels)]


def test_tagger_fires_is_the_composite_early_out(reference_lib):
    """regrid's tagger test (amr.cpp:124-133) for None, one gradient tagger, or a
    compositeTagger list (amr.cpp:723-731), from per-tagger counts: equal to the
    compiled compositeTagger tagging any cell, on a puncture block."""
    from oracle import Geom
    from granite_b200.regrid import CHI, LAPSE, tagger_fires
    calls = []

    def fake(var, threshold):
        calls.append((var, threshold))
        return {(CHI, 1.0): 0, (LAPSE, 0.5): 3}.get((var, threshold), 0)

    assert not tagger_fires(None, fake) and calls == []
    assert not tagger_fires((CHI, 1.0), fake)
    assert tagger_fires([(CHI, 1.0), (LAPSE, 0.5), (CHI, 9.0)], fake)
    assert calls[-1] == (LAPSE, 0.5)  # stops at the first tagger that fires
    assert not tagger_fires([], fake)
    g = Geom((12, 12, 12), (-3.0, -3.0, -3.0), (3.0, 3.0, 3.0))
    u = reference_lib.init_brill_lindquist(g, [1.0], [[0.1, 0.0, 0.0]])

    def count(var, threshold):
        return reference_lib.tag_count(g, u, var, threshold)

    for taggers in ([(CHI, 5.0)], [(CHI, 2.0)], [(CHI, 5.0), (LAPSE, 2.0)], [(CHI, 5.0), (LAPSE, 1.0)],
                    [(LAPSE, 0.5), (CHI, 0.5)]):
        assert tagger_fires(taggers, count) == (reference_lib.composite_tag_count(g, u, taggers) > 0)
        if len(taggers) == 1:
            assert tagger_fires(taggers[0], count) == (count(*taggers[0]) > 0)
