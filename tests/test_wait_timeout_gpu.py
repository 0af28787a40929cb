"""The TMA stage kernel's bounded waits, exercised on the GPU without a fault.

Every mbarrier wait of the stage kernel gives up after its wait limit (2 s),
records the failure in the context's error flag, and the CTA then waits (again
bounded) for the copies it still has in flight before it exits. The reference
has no device waits; its failure detection is the NaN scan of main.cpp:525-568.

The test switch granite_ccz4_test_withhold_tile_load makes the first persistent
CTA of the next step's first stage leave one ring item unissued: nothing is in
flight for that item, so its wait runs out on an mbarrier phase that never
completes, with the default limit in place. Nothing faults and nothing waits
without a bound. Checked here:
  * granite_ccz4_sync returns GRANITE_ERR_CUDA with the wait-limit message, and
    the sync after it returns GRANITE_OK (the flag is read and cleared);
  * a download after such a step reports the same error instead of handing a
    state the stage could not compute to the host;
  * the context keeps working: the next steps from a fresh upload equal the
    oracle's, with the parity bound of the multi-step tests.
"""
import numpy as np
import pytest

import oracle
from oracle import Geom, Params

from test_parity_gpu import parity

pytestmark = pytest.mark.gpu

CUDA_ERR = -2


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def _case(oracle_lib):
    g = Geom((32, 24, 16), (-4.0, -3.0, -2.0), (4.0, 3.0, 2.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.1, -0.2, 0.05]], r_floor=0.5 * g.dx[0])
    return g, oracle.add_noise(u, 1e-10, 7)


def _evolver(gb, g, u):
    ev = gb.Evolver(gb.CCZ4Params(device=0), gb.VARIANT_TMA)
    b = gb.GridBlock(0, 0, g.n, g.lo, g.hi)
    b.array[...] = u
    ev.add_block(b)
    ev.commit()
    ev.upload()
    return ev, b


def test_withheld_load_is_reported_by_sync_and_context_recovers(gb, oracle_lib):
    g, u = _case(oracle_lib)
    dt = 0.25 * g.dx[0]
    ev, b = _evolver(gb, g, u)
    ev.rk3_step(0, dt, gb.PRECISION_FP64, gb.BC_REFERENCE)
    ev.sync()  # a normal step leaves no error

    ev.test_withhold_tile_load(5)  # field 5 of the CTA's first tile
    ev.rk3_step(0, dt, gb.PRECISION_FP64, gb.BC_REFERENCE)
    with pytest.raises(gb.GraniteError) as ei:
        ev.sync()
    assert ei.value.code == CUDA_ERR
    assert "wait limit" in str(ei.value)
    ev.sync()  # the flag was cleared: the next sync is clean

    # the context still computes correct steps
    b.array[...] = u
    ev.upload()
    for _ in range(2):
        ev.rk3_step(0, dt, gb.PRECISION_FP64, gb.BC_REFERENCE)
    ev.download()
    ref = oracle_lib.rk3_steps(Params(), g, u, dt, 2)
    parity(b.array, ref, rtol=1e-10, what="after a withheld load")
    ev.close()


def test_withheld_load_is_reported_by_download(gb, oracle_lib):
    g, u = _case(oracle_lib)
    dt = 0.25 * g.dx[0]
    ev, b = _evolver(gb, g, u)
    ev.test_withhold_tile_load(3)  # field 3 of the CTA's first tile
    ev.rk3_step(0, dt, gb.PRECISION_FP64, gb.BC_REFERENCE)
    out = np.empty_like(b.array)
    with pytest.raises(gb.GraniteError) as ei:
        ev.download(0, out)
    assert ei.value.code == CUDA_ERR
    ev.sync()
    # and the switch was one-shot: the next step is clean
    ev.upload()
    ev.rk3_step(0, dt, gb.PRECISION_FP64, gb.BC_REFERENCE)
    ev.sync()
    ev.close()

