"""Matter coupling of the CCZ4 RHS on the GPU.

* ``MatterSources.computeMatterSources`` (granite_ccz4_matter_sources_host)
  against the oracle's restatement of GRMHDEvolution::computeMatterSources
  (grmhd.cpp:1034-1103, pinned to the compiled reference): bit for bit, cells
  outside the interior untouched, the golden vector included.
* The RHS with those sources against the oracle RHS (scaled per-point bound of
  test_parity_gpu.py).
* Resident matter (granite_ccz4_enable_matter + upload_primitives): RK3 steps
  with the sources held fixed against the oracle's RK3 step with the same
  sources; resident matter left at zero equals the vacuum step bit for bit.
"""
import os

import numpy as np
import pytest

import oracle
from oracle import Geom, Params

from test_parity_gpu import block_of, evo, parity

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


def device_sources(gb, g: Geom, prim, init=None):
    ms = gb.MatterSources()
    st = block_of(g)
    pb = gb.GridBlock(1, 0, g.n, g.lo, g.hi, g.ng, gb.NUM_PRIMITIVE_VARS)
    pb.array[...] = prim
    out = [np.array(a, dtype=np.float64, copy=True) for a in (init or oracle.matter_zeros(g))]
    ms.computeMatterSources(st, pb, *out)
    ms.close()
    return out


def test_matter_sources_golden(gb):
    z = np.load(os.path.join(GOLD, "matter_sources.npz"))
    g = Geom(tuple(int(x) for x in z["n"]), tuple(float(x) for x in z["lo"]), tuple(float(x) for x in z["hi"]),
             int(z["ng"]))
    prim = oracle.seeded_primitives(g, int(z["seed"]), float(z["superluminal"]))
    it = g.interior()[1:]
    for a, name in zip(device_sources(gb, g, prim), ("rho", "Si", "Sij", "S")):
        assert np.array_equal(a[it], z[name]), name


@pytest.mark.parametrize("n,seed,superluminal", [((33, 17, 9), 5, 0.1), ((5, 7, 6), 6, 0.0),
                                                  ((64, 8, 4), 7, 0.5)])
def test_matter_sources_vs_oracle(gb, oracle_lib, n, seed, superluminal):
    g = Geom(n, (-1.0, -0.5, 0.25), (1.0 + n[0] * 0.01, 0.5, 1.25))
    prim = oracle.seeded_primitives(g, seed, superluminal)
    init = tuple(oracle.hash_noise(a.shape, 70 + k) for k, a in enumerate(oracle.matter_zeros(g)))
    want = oracle_lib.matter_sources(g, prim, init)
    got = device_sources(gb, g, prim, init)
    for a, b, name in zip(got, want, ("rho", "Si", "Sij", "S")):
        assert np.array_equal(a, b), name


def test_rhs_with_device_sources(gb, oracle_lib):
    g = Geom((20, 16, 12), (-2.0, -1.6, -1.2), (2.0, 1.6, 1.2))
    u = oracle.seeded_state(g, 17)
    prim = oracle.seeded_primitives(g, 8, 0.02)
    prim[0] *= 1e-2  # a dilute fluid
    m = device_sources(gb, g, prim)
    rhs = block_of(g)
    evo(gb, Params()).computeRHS(block_of(g, u), rhs, *m)
    want = oracle_lib.rhs(Params(), g, u, *m)
    parity(rhs.array[g.interior()], want[g.interior()], what="rhs with matter from primitives")


def resident(gb, g: Geom, u, variant, matter: bool, prim=None):
    ev = gb.Evolver(gb.CCZ4Params(), variant)
    if matter:
        ev.enable_matter()
    b = block_of(g, u)
    ev.add_block(b)
    ev.commit()
    ev.upload()
    if prim is not None:
        ev.upload_primitives(0, prim)
    return ev, b


@pytest.mark.parametrize("variant", [0, 4])
def test_resident_matter_steps_vs_oracle(gb, oracle_lib, variant):
    g = Geom((24, 24, 24), (-6.0, -6.0, -6.0), (6.0, 6.0, 6.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * g.dx[0])
    u = oracle.add_noise(u, 1e-10, 4242)
    prim = oracle.seeded_primitives(g, 9, 0.0)  # a dilute, weakly magnetised fluid
    prim[0] *= 1e-3
    prim[4] *= 1e-4
    prim[5:8] *= 1e-2
    m = oracle_lib.matter_sources(g, prim)
    dt = 0.25 * g.dx[0]
    want = oracle_lib.rk3_steps(Params(), g, u, dt, 4, matter=m)
    vac = oracle_lib.rk3_steps(Params(), g, u, dt, 4)
    ev, b = resident(gb, g, u, variant, True, prim)
    for _ in range(4):
        ev.rk3_step(0, dt, gb.PRECISION_FP64, gb.BC_REFERENCE)
    ev.download()
    assert np.isfinite(want).all() and np.abs(want - vac).max() > 1e-3  # the sources act
    parity(b.array, want, rtol=1e-10, what="resident matter, 4 steps")
    ev.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_resident_matter_zero_equals_vacuum(gb, oracle_lib, precision):
    g = Geom((16, 16, 16), (-4.0, -4.0, -4.0), (4.0, 4.0, 4.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * g.dx[0])
    dt = 0.25 * g.dx[0]
    out = []
    for matter in (False, True):
        ev, b = resident(gb, g, u, 4, matter)
        for _ in range(3):
            ev.rk3_step(0, dt, precision, gb.BC_REFERENCE)
        ev.download()
        out.append(b.array.copy())
        ev.close()
    assert np.array_equal(out[0], out[1])


def test_matter_api_errors(gb):
    g = Geom((8, 8, 8), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    ev, _ = resident(gb, g, oracle.seeded_state(g, 1), 0, False)
    with pytest.raises(gb.GraniteError):  # matter not enabled
        ev.upload_primitives(0, oracle.seeded_primitives(g, 1))
    with pytest.raises(gb.GraniteError):  # after commit
        ev.enable_matter()
    ev.close()
