"""Every configuration of the TMA stage kernel (the autotuner's candidates) and
the per-class configuration table.

Configuration 5 runs the mixed form warp-specialized (stencil warps feed
algebra warps through shared memory): its derivatives are the same FP32
values, its algebra the same code, so it is held to the same bounds.

The configurations differ in tile depth, ring depth, resident CTAs per SM and
where intermediate values live (shared memory or registers / local memory),
never in arithmetic: in FP64 every configuration must give the results of
configuration 0 bit for bit, and those equal the oracle (the restatement of
ccz4.cpp:251-935 and main.cpp:306-689, pinned to the compiled reference) with
the multi-step parity bound. Mixed precision is compared with FP64 at the mixed
tolerance. A hierarchy whose block-size classes use different configurations
(several launches per level and stage) must equal the single-configuration run
bit for bit.
"""
import numpy as np
import pytest

import oracle
from oracle import Geom, Params

from test_parity_gpu import parity

pytestmark = pytest.mark.gpu

CONFIGS = list(range(18))


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


@pytest.fixture(scope="module")
def case(oracle_lib):
    # partial tiles in x (40 = 16 + 16 + 8: configuration 11 covers the last 8 columns with 8 x 4 x 4
    # remainder tiles), y (22) and z (18 = 4 x 4 + 2 / 9 x 2)
    g = Geom((40, 22, 18), (-5.0, -2.75, -2.25), (5.0, 2.75, 2.25))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.12, -0.1, 0.05]], r_floor=0.5 * g.dx[0])
    u = oracle.add_noise(u, 1e-10, 99)
    u[19] += 0.05 * oracle.hash_noise(g.shape[1:], 5)  # shift of both signs (upwind sides)
    dt = 0.25 * g.dx[0]
    ref = oracle_lib.rk3_steps(Params(), g, u, dt, 4)
    return g, u, dt, ref


def _steps(gb, g, u, dt, n, precision, cfg, fp64_chi=0.0):
    ev = gb.Evolver(gb.CCZ4Params(device=0), gb.VARIANT_TMA)
    ev.force_stage_config(cfg)
    b = gb.GridBlock(0, 0, g.n, g.lo, g.hi)
    b.array[...] = u
    ev.add_block(b)
    ev.commit()
    ev.upload()
    if fp64_chi > 0.0:
        ev.set_fp64_chi_threshold(fp64_chi)
    for _ in range(n):
        ev.rk3_step(0, dt, precision, gb.BC_REFERENCE)
    ev.download()
    ev.close()
    return b.array.copy()


@pytest.mark.parametrize("cfg", CONFIGS)
def test_config_fp64_matches_oracle_and_config0(gb, case, cfg):
    g, u, dt, ref = case
    out = _steps(gb, g, u, dt, 4, gb.PRECISION_FP64, cfg)
    parity(out, ref, rtol=1e-10, what=f"config {cfg}, 4 FP64 steps")
    if cfg:
        base = _steps(gb, g, u, dt, 4, gb.PRECISION_FP64, 0)
        assert np.array_equal(out, base), f"config {cfg} differs from config 0 in FP64"


@pytest.mark.parametrize("fp64_chi", [0.0, 0.5])
@pytest.mark.parametrize("cfg", CONFIGS)
def test_config_mixed_close_to_fp64(gb, case, cfg, fp64_chi):
    # FP32 algebra everywhere, or per-tile FP64 where chi < 0.5 (both passes of
    # the per-tile precision run in this configuration)
    g, u, dt, ref = case
    out = _steps(gb, g, u, dt, 4, gb.PRECISION_MIXED, cfg, fp64_chi)
    parity(out, ref, rtol=2e-5, what=f"config {cfg}, 4 mixed steps, fp64_chi {fp64_chi}")
    base = _steps(gb, g, u, dt, 4, gb.PRECISION_MIXED, 0, fp64_chi)
    parity(out, base, rtol=1e-6, what=f"config {cfg} vs config 0, mixed")


def test_per_class_table_on_a_hierarchy(gb, oracle_lib):
    # blocks of three size classes on two levels; each class gets another
    # configuration, so a level stage runs as several launches
    geoms = [Geom((16, 16, 16), (-4.0, -4.0, -4.0), (0.0, 0.0, 0.0)),
             Geom((40, 32, 16), (0.0, -4.0, -4.0), (10.0, 4.0, 0.0)),
             Geom((16, 16, 16), (-4.0, 0.0, -4.0), (0.0, 4.0, 0.0)),
             Geom((48, 48, 48), (-3.0, -3.0, -3.0), (3.0, 3.0, 3.0))]
    levels = [0, 0, 0, 1]
    states = []
    for i, g in enumerate(geoms):
        v = oracle_lib.init_brill_lindquist(g, [0.5], [[0.3, 0.2, -0.1]], r_floor=0.5 * g.dx[0])
        states.append(oracle.add_noise(v, 1e-10, 40 + i))
    dt = 0.25 * geoms[0].dx[0]

    def run(table, precision):
        ev = gb.Evolver(gb.CCZ4Params(device=0), gb.VARIANT_TMA)
        if table is None:
            ev.force_stage_config(0)
        else:
            ev.apply_stage_table(table)
        blocks = []
        for i, (g, L) in enumerate(zip(geoms, levels)):
            b = gb.GridBlock(i, L, g.n, g.lo, g.hi)
            b.array[...] = states[i]
            ev.add_block(b)
            blocks.append(b)
        ev.commit()
        ev.upload()
        for _ in range(2):
            ev.hierarchy_step(dt, precision, gb.AMR_GHOSTS)
        ev.download()
        ev.close()
        return [b.array.copy() for b in blocks]

    classes = [gb.block_stage_class(g.n) for g in geoms]
    assert len(set(classes)) == 3
    mixed_table = [6, 11, 3, 5, 1, 2]  # the 40-wide block (class 1) gets x-remainder tiles
    table = {"fp64": mixed_table, "mixed": mixed_table}
    a = run(None, gb.PRECISION_FP64)
    b = run(table, gb.PRECISION_FP64)
    for i in range(len(geoms)):
        assert np.array_equal(a[i], b[i]), f"block {i}: per-class table differs from configuration 0"
    am = run(None, gb.PRECISION_MIXED)
    bm = run(table, gb.PRECISION_MIXED)
    for i in range(len(geoms)):
        parity(bm[i], am[i], rtol=1e-6, what=f"mixed block {i}")

