"""GPU Berger-Oliger hierarchy step against the hierarchy oracle.

GRANITE_AMR_REFERENCE is checked on the reference's own tracking-sphere
hierarchy (built by the compiled AMRHierarchy where available, else rebuilt
from its recorded geometry) and GRANITE_AMR_GHOSTS on seeded multi-block
hierarchies, both with the scaled per-point bound of test_parity_gpu.py.
"""
import numpy as np
import pytest

import oracle
from oracle import Geom, Params
from oracle.hierarchy import HierarchyOracle

from test_parity_gpu import VARIANTS, parity

pytestmark = pytest.mark.gpu

BL_M = [0.5, 0.5]
BL_X = [[1.5, 0.0, 0.0], [-1.5, 0.0, 0.0]]

# geometry of the reference hierarchy of test_hierarchy_cpu (base 16^3 on [-8, 8]^3,
# tracking spheres at x = +-1.5, radius 2, min_level 2), as AMRHierarchy builds it
REF_LAYOUT = None


def reference_layout():
    global REF_LAYOUT
    if REF_LAYOUT is None:
        if oracle.reference_available("strict"):
            from oracle.hierarchy import RefHierarchy
            rh = RefHierarchy(oracle.Reference("strict"), (16, 16, 16), (-8.0, -8.0, -8.0), (8.0, 8.0, 8.0),
                              [((1.5, 0.0, 0.0), 2.0, 2), ((-1.5, 0.0, 0.0), 2.0, 2)])
            REF_LAYOUT = (rh.geoms, rh.levels)
        else:  # the layout AMRHierarchy::regrid produces for these spheres (amr.cpp:147-300)
            REF_LAYOUT = ([Geom((16, 16, 16), (-8.0, -8.0, -8.0), (8.0, 8.0, 8.0)),
                           Geom((22, 16, 16), (-6.0, -4.0, -4.0), (5.0, 4.0, 4.0)),
                           Geom((28, 16, 16), (-3.5, -2.0, -2.0), (3.5, 2.0, 2.0))], [0, 1, 2])
    return REF_LAYOUT


def gpu_hierarchy(gb, geoms, levels, states, variant=None):
    ev = gb.Evolver(gb.CCZ4Params(), variant)
    blocks = []
    for i, (g, L) in enumerate(zip(geoms, levels)):
        b = gb.GridBlock(i, L, g.n, g.lo, g.hi)
        b.array[...] = states[i]
        ev.add_block(b)
        blocks.append(b)
    ev.commit()
    ev.upload()
    return ev, blocks


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


@pytest.mark.parametrize("variant", VARIANTS)
def test_reference_mode_matches_oracle(gb, oracle_lib, variant):
    geoms, levels = reference_layout()
    states = []
    for i, g in enumerate(geoms):
        u = oracle_lib.init_brill_lindquist(g, BL_M, BL_X)
        states.append(u + 1e-8 * oracle.hash_noise(g.shape, 100 + i))
    ho = HierarchyOracle(geoms, levels, oracle_lib)
    for i, u in enumerate(states):
        ho.u[i][...] = u
    dt = 0.25 * geoms[0].dx[0]
    ho.step(Params(), dt, "reference", 2)
    ev, blocks = gpu_hierarchy(gb, geoms, levels, states, variant)
    for _ in range(2):
        ev.hierarchy_step(dt, gb.PRECISION_FP64, gb.AMR_REFERENCE)
    ev.download()
    for i, b in enumerate(blocks):
        parity(b.array, ho.u[i], rtol=1e-10, what=f"reference-mode block {i} level {levels[i]}")


def small_hierarchy(seed=5, levels=3):
    from granite_b200.hierarchy import make_binary_hierarchy
    h = make_binary_hierarchy(seed=seed, levels=levels, coarse_n=32, extent=16.0, sizes=(8, 16, 24),
                              blocks_per_level=(8, 40))
    geoms = [Geom(b.ncells, b.lo, b.hi) for b in h.blocks]
    return h, geoms, [b.level for b in h.blocks]


@pytest.mark.parametrize("variant", VARIANTS)
def test_ghosts_mode_matches_oracle(gb, oracle_lib, variant):
    h, geoms, levels = small_hierarchy()
    states = []
    for i, g in enumerate(geoms):
        u = oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0])
        states.append(oracle.add_noise(u, 1e-10, 12345 + i))
    ho = HierarchyOracle(geoms, levels, oracle_lib)
    for i, u in enumerate(states):
        ho.u[i][...] = u
    dt = 0.25 * geoms[0].dx[0]
    ho.step(Params(), dt, "ghosts", 2)
    ev, blocks = gpu_hierarchy(gb, geoms, levels, states, variant)
    for _ in range(2):
        ev.hierarchy_step(dt, gb.PRECISION_FP64, gb.AMR_GHOSTS)
    ev.download()
    for i, b in enumerate(blocks):
        parity(b.array, ho.u[i], rtol=1e-10, what=f"ghosts-mode block {i} level {levels[i]}")


def test_hierarchy_graph_replay_deterministic(gb, oracle_lib):
    h, geoms, levels = small_hierarchy(seed=9, levels=2)
    states = [oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]) for g in geoms]
    dt = 0.25 * geoms[0].dx[0]
    outs = []
    for _ in range(2):
        ev, blocks = gpu_hierarchy(gb, geoms, levels, states)
        for _ in range(3):
            ev.hierarchy_step(dt, gb.PRECISION_FP64, gb.AMR_GHOSTS)
        ev.download()
        outs.append([b.array.copy() for b in blocks])
        ev.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("mode", ["ghosts", "reference"])
def test_unbatched_equals_batched(gb, oracle_lib, mode):
    # per-block eager launches compute exactly what the batched graph does
    h, geoms, levels = small_hierarchy(seed=13, levels=2)
    states = [oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]) for g in geoms]
    dt = 0.25 * geoms[0].dx[0]
    amr = gb.AMR_GHOSTS if mode == "ghosts" else gb.AMR_REFERENCE
    outs = []
    for batched in (True, False):
        ev, blocks = gpu_hierarchy(gb, geoms, levels, states)
        ev.set_batching(batched)
        for _ in range(2):
            ev.hierarchy_step(dt, gb.PRECISION_FP64, amr)
        ev.download()
        outs.append([b.array.copy() for b in blocks])
        ev.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_hierarchy_mixed_close_to_fp64(gb, oracle_lib):
    h, geoms, levels = small_hierarchy(seed=11, levels=2)
    states = [oracle.add_noise(oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]),
                               1e-10, 7 + i) for i, g in enumerate(geoms)]
    dt = 0.25 * geoms[0].dx[0]
    res = {}
    for prec in (gb.PRECISION_FP64, gb.PRECISION_MIXED):
        ev, blocks = gpu_hierarchy(gb, geoms, levels, states)
        for _ in range(4):
            ev.hierarchy_step(dt, prec, gb.AMR_GHOSTS)
        ev.download()
        res[prec] = [b.array.copy() for b in blocks]
        ev.close()
    # mixed-precision deviation from the FP64 run, relative to each tensor's scale
    for a, b in zip(res[gb.PRECISION_FP64], res[gb.PRECISION_MIXED]):
        parity(b, a, rtol=1e-5, what="mixed vs fp64")


@pytest.mark.parametrize("precision,layout", [(0, "small"), (1, "small"), (0, "tma"), (1, "tma")])
def test_finest_prefill_skip_is_exact(gb, oracle_lib, precision, layout):
    # the graph-captured step leaves out the fill before the finest level's second
    # substep (its inputs are those of the fill that ended the first one), and
    # once the fill after a level's step has made its same-level copies current,
    # its fill before the next step copies only cells whose source a restriction
    # rewrote in between (within a coarse step and across coarse steps); the
    # uncaptured step with the regrid hook (interval 0: no regrid) performs every
    # fill in full, as amr.cpp does: the two agree bit for bit
    if layout == "small":
        h, geoms, levels = small_hierarchy(seed=17, levels=3)
    else:  # blocks of 16 to 32 cells (the TMA stage kernel on every level)
        from granite_b200.hierarchy import make_binary_hierarchy
        h = make_binary_hierarchy(seed=23, levels=3, coarse_n=48, extent=16.0, sizes=(16, 24, 32),
                                  blocks_per_level=(8, 40))
        geoms = [Geom(b.ncells, b.lo, b.hi) for b in h.blocks]
        levels = [b.level for b in h.blocks]
    states = [oracle.add_noise(oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]),
                               1e-10, 90 + i) for i, g in enumerate(geoms)]
    dt = 0.25 * geoms[0].dx[0]
    outs = []
    for hooked in (False, True):
        ev, blocks = gpu_hierarchy(gb, geoms, levels, states)
        ev.set_fp64_chi_threshold(0.5)
        for _ in range(3):
            if hooked:
                ev.hierarchy_step_regrid(dt, None, 0, precision=precision, amr_mode=gb.AMR_GHOSTS)
            else:
                ev.hierarchy_step(dt, precision, gb.AMR_GHOSTS)
        ev.download()
        outs.append([b.array.copy() for b in blocks])
        ev.close()
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision,chi", [(0, 0.0), (1, 0.0), (1, 0.5)])
def test_ghost_push_equals_copy_fills(gb, oracle_lib, precision, chi):
    # GRANITE_AMR_GHOSTS with pushes on: the stage kernels write the same-level
    # ghost copies themselves (both passes of the per-tile precision included),
    # the fills after the stages leave the copies out, and the fill before a
    # level step refreshes only the copies of cells a restriction rewrote; the
    # result equals the run whose fills copy every same-level ghost cell (the
    # default), bit for bit
    # blocks of 16 to 32 cells, so that every level runs the TMA stage kernel
    from granite_b200.hierarchy import make_binary_hierarchy
    h = make_binary_hierarchy(seed=21, levels=3, coarse_n=48, extent=16.0, sizes=(16, 24, 32),
                              blocks_per_level=(8, 40))
    geoms = [Geom(b.ncells, b.lo, b.hi) for b in h.blocks]
    levels = [b.level for b in h.blocks]
    states = [oracle.add_noise(oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]),
                               1e-10, 60 + i) for i, g in enumerate(geoms)]
    dt = 0.25 * geoms[0].dx[0]
    outs = []
    for push in (True, False):
        ev, blocks = gpu_hierarchy(gb, geoms, levels, states, gb.VARIANT_TMA)
        ev.set_ghost_push(push)
        if chi > 0.0:
            ev.set_fp64_chi_threshold(chi)
        for _ in range(3):  # the second and third steps fill before each level step without copies
            ev.hierarchy_step(dt, precision, gb.AMR_GHOSTS)
        ev.download()
        res = [b.array.copy() for b in blocks]
        # an upload invalidates the pushed copies: the next step fills them again
        for b, u in zip(blocks, states):
            b.array[...] = u
        ev.upload()
        ev.hierarchy_step(dt, precision, gb.AMR_GHOSTS)
        ev.download()
        outs.append(res + [b.array.copy() for b in blocks])
        ev.close()
    for i, (a, b) in enumerate(zip(*outs)):
        assert np.array_equal(a, b), f"array {i}: pushed ghost copies differ from copied ones"


def test_three_context_pipeline_host_round_trips(gb, oracle_lib):
    """The host round trip of bench.py's e2e: three contexts take the steps in
    turn, each step uploads the input from pinned memory, steps, and queues the
    download (granite_ccz4_download_all_async) while the other contexts work,
    uploads and downloads ordered across the contexts' streams by events; every
    result equals the same step taken alone, bit for bit."""
    import torch
    h, geoms, levels = small_hierarchy(seed=4, levels=3)
    states = [oracle_lib.init_brill_lindquist(g, h.masses, h.positions, r_floor=0.5 * g.dx[0]) for g in geoms]
    dt = 0.25 * geoms[0].dx[0]
    ev, blocks = gpu_hierarchy(gb, geoms, levels, states)
    ev.hierarchy_step(dt, gb.PRECISION_MIXED, gb.AMR_GHOSTS)
    ev.download()
    want = [b.array.copy() for b in blocks]
    ev.close()

    def pinned(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        v = t.numpy().reshape(a.shape)
        v[...] = a
        return t, v

    pin_in = [pinned(s) for s in states]
    vin = [v for _, v in pin_in]
    nctx = 3
    evs, outs = [], []
    for _ in range(nctx):
        e, _b = gpu_hierarchy(gb, geoms, levels, states)
        evs.append(e)
        outs.append([pinned(np.zeros_like(s)) for s in states])
    streams = [torch.cuda.ExternalStream(e.stream_handle(), device="cuda:0") for e in evs]
    try:
        last_up = last_down = None
        for s in range(9):
            e, o, st = evs[s % nctx], outs[s % nctx], streams[s % nctx]
            e.sync()
            if s >= nctx:  # the result of step s - nctx, read before its buffers are reused
                for a, b in zip(want, o):
                    assert np.array_equal(a, b[1])
                for _, v in o:
                    v[...] = 0.0
            if last_up is not None:
                st.wait_event(last_up)
            e.upload(None, vin)
            last_up = torch.cuda.Event()
            last_up.record(st)
            e.hierarchy_step(dt, gb.PRECISION_MIXED, gb.AMR_GHOSTS)
            if last_down is not None:
                st.wait_event(last_down)
            e.download(None, [v for _, v in o], wait=False)
            last_down = torch.cuda.Event()
            last_down.record(st)
        for e, o in zip(evs, outs):
            e.sync()
            for a, b in zip(want, o):
                assert np.array_equal(a, b[1])
    finally:
        for e in evs:
            e.close()
