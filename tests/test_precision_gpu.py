"""Per-tile precision of MIXED steps (granite_ccz4_set_fp64_chi_threshold).

Tiles whose stage input has a point with chi below the threshold run the FP64
algebra (with pair-difference FP64 stencils), the others the FP32 algebra. A
threshold above every chi must reproduce FP64 steps to rounding (the parity
bound of the FP64 path), a positive threshold below every chi pure MIXED steps
bit for bit, and a threshold in between must bring the near-puncture points
closer to the FP64 run than pure MIXED does.
"""
import numpy as np
import pytest

import oracle
from oracle import Geom

from test_hierarchy_gpu import gpu_hierarchy, small_hierarchy
from test_parity_gpu import parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def puncture_block(oracle_lib, n=32, half=4.0):
    g = Geom((n, n, n), (-half,) * 3, (half,) * 3)
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.1, -0.05, 0.02]], r_floor=0.5 * g.dx[0])
    return g, oracle.add_noise(u, 1e-10, 77)


def run_block(gb, g, u, precision, steps, chi_fp64=None, variant=None):
    ev = gb.Evolver(gb.CCZ4Params(), variant)
    if chi_fp64 is not None:
        ev.set_fp64_chi_threshold(chi_fp64)
        assert ev.fp64_chi_threshold() == chi_fp64
    b = gb.GridBlock(0, 0, g.n, g.lo, g.hi)
    b.array[...] = u
    ev.add_block(b)
    ev.commit()
    ev.upload()
    dt = 0.25 * g.dx[0]
    for _ in range(steps):
        ev.rk3_step(0, dt, precision, gb.BC_REFERENCE)
    ev.download()
    ev.close()
    return b.array.copy()


@pytest.mark.parametrize("variant", [0, 4])
def test_threshold_above_all_chi_is_fp64(gb, oracle_lib, variant):
    g, u = puncture_block(oracle_lib)
    ref = run_block(gb, g, u, gb.PRECISION_FP64, 2, variant=variant)
    out = run_block(gb, g, u, gb.PRECISION_MIXED, 2, chi_fp64=1e30, variant=variant)
    parity(out, ref, rtol=1e-10, what="all tiles FP64 vs FP64 steps")  # multi-step bound


@pytest.mark.parametrize("variant", [0, 4])
def test_threshold_below_all_chi_is_mixed(gb, oracle_lib, variant):
    g, u = puncture_block(oracle_lib)
    ref = run_block(gb, g, u, gb.PRECISION_MIXED, 2, variant=variant)
    out = run_block(gb, g, u, gb.PRECISION_MIXED, 2, chi_fp64=1e-300, variant=variant)
    assert np.array_equal(out, ref)


def test_threshold_tightens_near_puncture(gb, oracle_lib):
    g, u = puncture_block(oracle_lib, n=48, half=6.0)
    steps = 4
    f64 = run_block(gb, g, u, gb.PRECISION_FP64, steps)
    mix = run_block(gb, g, u, gb.PRECISION_MIXED, steps)
    hyb = run_block(gb, g, u, gb.PRECISION_MIXED, steps, chi_fp64=0.5)
    it = g.interior()
    chi = f64[0][it[1:]]
    near = chi < 0.3
    assert near.sum() > 100
    d_mix = np.abs(mix[it] - f64[it])[:, near].max()
    d_hyb = np.abs(hyb[it] - f64[it])[:, near].max()
    # the split is real: neither all-FP64 nor all-FP32
    assert not np.array_equal(hyb, f64) and not np.array_equal(hyb, mix)
    assert d_hyb < 0.1 * d_mix, (d_hyb, d_mix)


def test_hierarchy_threshold_above_all_chi_is_fp64(gb, oracle_lib):
    h, geoms, levels = small_hierarchy(seed=17, levels=2)
    states = [oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]) for g in geoms]
    dt = 0.25 * geoms[0].dx[0]
    outs = []
    for prec, thr in ((gb.PRECISION_FP64, None), (gb.PRECISION_MIXED, 1e30)):
        ev, blocks = gpu_hierarchy(gb, geoms, levels, states)
        if thr is not None:
            ev.set_fp64_chi_threshold(thr)
        for _ in range(2):
            ev.hierarchy_step(dt, prec, gb.AMR_GHOSTS)
        ev.download()
        outs.append([b.array.copy() for b in blocks])
        ev.close()
    for a, b in zip(*outs):
        parity(b, a, rtol=1e-10, what="hierarchy, all tiles FP64 vs FP64 steps")  # multi-step bound


def test_threshold_rejects_bad_values(gb):
    ev = gb.Evolver(gb.CCZ4Params())
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(gb.GraniteError):
            ev.set_fp64_chi_threshold(bad)
    ev.close()
