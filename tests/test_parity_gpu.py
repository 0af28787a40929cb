"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle and the
golden vectors of the compiled reference.

Tolerance (plain FP64): per field v and interior point,
    |gpu - oracle| <= 1e-12 * max(|oracle|, s_v),
    s_v = max |oracle_w| over the block and over the components w of v's tensor
          (chi; gt_ij; At_ij; K; Gamma-hat^i; Theta; alpha; beta^i),
the per-point bound of the parity contract. A relative bound alone is
ill-posed where the RHS crosses zero, and a component that is analytically
zero (gt_xy of a 1-D gauge wave) holds only rounding noise of the size of its
tensor's other components, so components are scaled by their tensor. Ghost
fills, RK combines and floors are exact re-evaluations of the reference loops
and are compared bit for bit where they are isolated; multi-step runs use the
same scaled bound on the state plus a 1e-10 relative bound on the constraint
norms.
"""
import os

import numpy as np
import pytest

import oracle
from oracle import Geom, Params

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-12


# tensor groups of the 22 evolved fields (types.hpp:104-130)
GROUPS = [[0], [1, 2, 3, 4, 5, 6], [7, 8, 9, 10, 11, 12], [13], [14, 15, 16], [17], [18],
          [19, 20, 21]]
GROUP_OF = {v: g for g in GROUPS for v in g}


def parity(gpu, ref, rtol=RTOL, what="", scale=None):
    """Scaled per-point bound over the leading (field) axis; returns the worst ratio.
    scale: per-field magnitudes to use for s_v instead of this array's own
    maxima (for one block of a multi-block state: the field's magnitude over all
    blocks)."""
    worst = 0.0
    nf = ref.shape[0]
    for v in range(nf):
        o = ref[v]
        g = gpu[v]
        grp = GROUP_OF[v] if nf == 22 else [v]
        s = max((np.abs(ref[w]).max() if scale is None else scale[w]) for w in grp)
        bound = rtol * np.maximum(np.abs(o), s)
        err = np.abs(g - o)
        if s == 0.0:
            assert err.max() <= 1e-300 + rtol, f"{what} field {v}: nonzero where reference is 0"
            continue
        ratio = (err / bound).max()
        worst = max(worst, ratio)
        assert ratio <= 1.0, f"{what} field {v}: max |d| = {err.max():.3e}, s_v = {s:.3e}, ratio {ratio:.2f}"
    return worst


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    g = Geom(tuple(int(x) for x in z["n"]), tuple(float(x) for x in z["lo"]),
             tuple(float(x) for x in z["hi"]), int(z["ng"]))
    return g, z


def block_of(g: Geom, u=None, level=0):
    import granite_b200 as gb
    b = gb.GridBlock(0, level, g.n, g.lo, g.hi, g.ng)
    if u is not None:
        b.array[...] = u
    return b


@pytest.fixture(scope="module")
def gb():
    import granite_b200
    return granite_b200


# stencils from global memory / staged through shared memory / global with 168 and
# 128 registers per thread / streamed through a TMA ring by persistent CTAs
VARIANTS = [0, 1, 2, 3, 4]


def evo(gb, p: Params, precision=0, variant=None):
    return gb.CCZ4Evolution(gb.CCZ4Params(kappa1=p.kappa1, kappa2=p.kappa2, eta=p.eta,
                                          ko_sigma=p.ko_sigma, chi_blend_center=p.chi_blend_center,
                                          chi_blend_width=p.chi_blend_width), precision, variant)


# ---------------------------------------------------------------------------
# single RHS evaluations
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("name,ko", [("rhs_random", 0.1), ("rhs_random_noko", 0.0)])
def test_rhs_golden(gb, name, ko, variant):
    g, z = load(name)
    u = oracle.seeded_state(g, int(z["seed"]))
    rhs = block_of(g)
    evo(gb, Params(ko_sigma=ko), variant=variant).computeRHSVacuum(block_of(g, u), rhs)
    parity(rhs.array[g.interior()], z["rhs"], what=name)


def test_rhs_matter_golden(gb):
    g, z = load("rhs_matter")
    u = oracle.seeded_state(g, int(z["seed"]))
    rho, Si, Sij, S = oracle.seeded_matter(g, int(z["matter_seed"]))
    rhs = block_of(g)
    evo(gb, Params()).computeRHS(block_of(g, u), rhs, rho, Si.reshape(-1, 3), Sij.reshape(-1, 6), S)
    parity(rhs.array[g.interior()], z["rhs"], what="matter")


@pytest.mark.parametrize("variant", VARIANTS)
def test_rhs_bl_golden(gb, variant):
    g, z = load("rhs_bl")
    o = oracle.Oracle()
    u = o.init_brill_lindquist(g, [0.5, 0.5], [[0.7, 0.1, -0.05], [-0.8, -0.05, 0.1]])
    u = u + 1e-6 * oracle.hash_noise(g.shape, int(z["seed"]))
    rhs = block_of(g)
    evo(gb, Params(), variant=variant).computeRHSVacuum(block_of(g, u), rhs)
    parity(rhs.array[g.interior()], z["rhs"], what="bl")


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("seed,n", [(1, (33, 17, 9)), (2, (16, 16, 16)), (3, (40, 8, 12)), (4, (5, 7, 6))])
def test_rhs_random_vs_oracle(gb, oracle_lib, seed, n, variant):
    # uneven, non-cubic blocks (partial tiles), shifts of both signs, strong gradients
    g = Geom(n, (-1.3, -0.7, -2.0), (1.1, 0.9, -0.2))
    u = oracle.seeded_state(g, seed, amp=0.2, noise=1e-2)
    p = Params(kappa1=0.05, kappa2=0.1, eta=1.5, ko_sigma=0.3)
    ref = oracle_lib.rhs(p, g, u)
    rhs = block_of(g)
    evo(gb, p, variant=variant).computeRHSVacuum(block_of(g, u), rhs)
    parity(rhs.array[g.interior()], ref[g.interior()], what=f"seed {seed}")
    # ghosts of rhs are untouched (the reference writes interior cells only)
    mask = np.ones(g.shape[1:], bool)
    mask[g.interior()[1:]] = False
    assert np.all(rhs.array[:, mask] == 0.0)


@pytest.mark.parametrize("variant", VARIANTS)
def test_rhs_puncture_vs_oracle(gb, oracle_lib, variant):
    # chi through the blend window and the 1e-4 clamp near the puncture
    g = Geom((24, 20, 16), (-1.5, -1.25, -1.0), (1.5, 1.25, 1.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.01, 0.02, -0.015]])
    u = oracle.add_noise(u, 1e-10, 12345)
    u[19] += 0.3 * oracle.hash_noise(g.shape[1:], 4)  # beta^x of both signs
    ref = oracle_lib.rhs(Params(), g, u)
    rhs = block_of(g)
    evo(gb, Params(), variant=variant).computeRHSVacuum(block_of(g, u), rhs)
    parity(rhs.array[g.interior()], ref[g.interior()], what="puncture")


def test_rhs_vacuum_equals_zero_matter(gb):
    # test_gauge_wave.cpp:129-166: zero sources give the vacuum RHS exactly
    g = Geom((32, 8, 8), (0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
    o = oracle.Oracle()
    u = o.init_gauge_wave(g, 0.01, 1.0)
    e = evo(gb, Params(ko_sigma=0.0))
    r1, r2 = block_of(g), block_of(g)
    e.computeRHSVacuum(block_of(g, u), r1)
    N = g.cells
    e.computeRHS(block_of(g, u), r2, np.zeros(N), np.zeros((N, 3)), np.zeros((N, 6)), np.zeros(N))
    assert np.array_equal(r1.array, r2.array)


def test_dissipation_golden(gb):
    g, z = load("ko_random")
    u = oracle.seeded_state(g, int(z["seed"]))
    rhs = block_of(g)
    evo(gb, Params()).applyDissipation(block_of(g, u), rhs)
    # the KO drop-in re-evaluates the reference loop without contraction: bit-exact
    assert np.array_equal(rhs.array[g.interior()], z["ko"])


@pytest.mark.parametrize("name", ["constraints_random", "constraints_bl"])
def test_constraints_golden(gb, name):
    g, z = load(name)
    if name == "constraints_bl":
        o = oracle.Oracle()
        u = o.init_brill_lindquist(g, [0.5, 0.5], [[0.7, 0.1, -0.05], [-0.8, -0.05, 0.1]])
        u = u + 1e-6 * oracle.hash_noise(g.shape, int(z["seed"]))
    else:
        u = oracle.seeded_state(g, int(z["seed"]))
    ham, mom = evo(gb, Params()).computeConstraints(block_of(g, u))
    sh = g.shape[1:]
    ham = ham.reshape(sh)
    mom = mom.reshape(sh + (3,))
    it = g.interior()[1:]
    parity(ham[it][None], z["ham"][None], what="H")
    parity(np.moveaxis(mom[it], -1, 0), np.moveaxis(z["mom"], -1, 0), what="M")
    mask = np.ones(sh, bool)
    mask[it] = False
    assert np.all(ham[mask] == 0.0) and np.all(mom[mask] == 0.0)


# ---------------------------------------------------------------------------
# reference test-suite assertions through the drop-in API
# ---------------------------------------------------------------------------

def test_reference_suite_flat(gb):
    # test_ccz4_flat.cpp: flat RHS < 1e-10, constraints < 1e-10, KO on constants < 1e-12
    b = gb.GridBlock(0, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    gb.set_flat_spacetime(b)
    rhs = gb.GridBlock(1, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    gb.CCZ4Evolution(gb.CCZ4Params(ko_sigma=0.0)).computeRHSVacuum(b, rhs)
    assert np.abs(rhs.array[b.interior()]).max() < 1e-10
    ham, mom = gb.CCZ4Evolution(gb.CCZ4Params(ko_sigma=0.0)).computeConstraints(b)
    assert np.abs(ham).max() < 1e-10 and np.abs(mom).max() < 1e-10
    gb.CCZ4Evolution(gb.CCZ4Params(ko_sigma=0.35)).computeRHSVacuum(b, rhs)
    assert np.abs(rhs.array[b.interior()]).max() < 1e-12


def test_reference_suite_advection(gb):
    # test_ccz4_flat.cpp:298-373: selective advection finite for chi = 1 and chi = 0.01
    b = gb.GridBlock(0, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    gb.set_flat_spacetime(b)
    X = np.array([b.x(0, i) for i in range(40)])
    b.array[18] = 1.0 + 0.01 * X[None, None, :]
    b.array[19] = 0.5
    rhs = gb.GridBlock(1, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    e = gb.CCZ4Evolution(gb.CCZ4Params(ko_sigma=0.0))
    e.computeRHSVacuum(b, rhs)
    assert np.isfinite(rhs.array[18][6:-6, 6:-6, 6:-6]).all()
    b2 = gb.GridBlock(0, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    gb.set_flat_spacetime(b2)
    b2.array[0] = 0.01
    e.computeRHSVacuum(b2, rhs)
    assert np.isfinite(rhs.array[:, 6:-6, 6:-6, 6:-6]).all()


def test_reference_suite_gauge_wave(gb):
    # test_ccz4_flat.cpp:240-286 and test_gauge_wave.cpp:91-127
    b = gb.GridBlock(10, 0, (64, 8, 8), (0, 0, 0), (1.0, 0.125, 0.125), 4, 22)
    gb.set_gauge_wave_data(b, 0.01, 1.0)
    rhs = gb.GridBlock(11, 0, (64, 8, 8), (0, 0, 0), (1.0, 0.125, 0.125), 4, 22)
    gb.CCZ4Evolution(gb.CCZ4Params(ko_sigma=0.35)).computeRHSVacuum(b, rhs)
    r = rhs.array[:, 7:-7, 7:-7, 7:-7]
    assert np.isfinite(r).all() and 0.0 < np.abs(r).max() < 50.0
    gb.CCZ4Evolution(gb.CCZ4Params(ko_sigma=0.1)).computeRHSVacuum(b, rhs)
    assert np.abs(rhs.array[:, 5:9, 5:9, 5:-5]).max() < 100.0


# ---------------------------------------------------------------------------
# fused RK3 steps against the oracle driver
# ---------------------------------------------------------------------------

def run_steps(gb, g: Geom, u, p: Params, dt, nsteps, bc, precision=0, variant=None):
    ev = gb.Evolver(gb.CCZ4Params(kappa1=p.kappa1, kappa2=p.kappa2, eta=p.eta, ko_sigma=p.ko_sigma),
                    variant)
    b = block_of(g, u)
    ev.add_block(b)
    ev.commit()
    ev.upload()
    for _ in range(nsteps):
        ev.rk3_step(0, dt, precision, bc)
    ev.download()
    return b.array, ev


@pytest.mark.parametrize("variant", VARIANTS)
def test_rk3_golden_bl(gb, variant):
    g, z = load("rk3_bl_3steps")
    o = oracle.Oracle()
    u = o.init_brill_lindquist(g, [0.5, 0.5], [[0.7, 0.1, -0.05], [-0.8, -0.05, 0.1]])
    u = u + 1e-6 * oracle.hash_noise(g.shape, int(z["seed"]))
    out, _ = run_steps(gb, g, u, Params(), float(z["dt"]), int(z["nsteps"]), gb.BC_REFERENCE,
                       variant=variant)
    parity(out[g.interior()], z["u"], rtol=1e-11, what="rk3 bl")


def test_rk3_golden_gauge_wave_periodic(gb):
    g, z = load("rk3_gauge_wave_periodic_4steps")
    o = oracle.Oracle()
    u = o.init_gauge_wave(g, -0.1, 1.0)
    out, _ = run_steps(gb, g, u, Params(), float(z["dt"]), int(z["nsteps"]), gb.BC_PERIODIC)
    parity(out[g.interior()], z["u"], rtol=1e-11, what="rk3 gauge wave")


@pytest.mark.parametrize("variant", VARIANTS)
def test_rk3_single_puncture_vs_oracle(gb, oracle_lib, variant):
    # the single-puncture workload at reduced size: 32^3 on [-16,16]^3, 20 steps
    g = Geom((32, 32, 32), (-16.0, -16.0, -16.0), (16.0, 16.0, 16.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]], r_floor=0.5 * g.dx[0])
    u = oracle.add_noise(u, 1e-10, 12345)
    dt = 0.25 * g.dx[0]
    n = 20
    ref = oracle_lib.rk3_steps(Params(), g, u, dt, n)
    out, ev = run_steps(gb, g, u, Params(), dt, n, gb.BC_REFERENCE, variant=variant)
    parity(out[g.interior()], ref[g.interior()], rtol=1e-10, what="puncture 20 steps")
    # whole block including ghosts (level fill of the last step)
    parity(out, ref, rtol=1e-10, what="puncture ghosts")
    h_ref, m_ref, npts = oracle_lib.constraint_sums(g, ref)
    h, m = ev.constraint_norms(0)
    assert abs(h - np.sqrt(h_ref / npts)) <= 1e-10 * np.sqrt(h_ref / npts)
    assert abs(m - np.sqrt(m_ref / npts)) <= 1e-10 * np.sqrt(m_ref / npts)


def test_rk3_gauge_wave_vs_oracle(gb, oracle_lib):
    # the gauge-wave workload at reduced size and step count
    g = Geom((24, 24, 24), (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))
    u = oracle_lib.init_gauge_wave(g, -0.1, 1.0)
    dt = 0.25 * g.dx[0]
    ref = oracle_lib.rk3_steps(Params(), g, u, dt, 10, bc=oracle.BC_PERIODIC)
    out, _ = run_steps(gb, g, u, Params(), dt, 10, gb.BC_PERIODIC)
    parity(out, ref, rtol=1e-10, what="gauge wave 10 steps")


def test_rk3_graph_replay_is_deterministic(gb, oracle_lib):
    g = Geom((20, 16, 12), (-2.0, -2.0, -2.0), (2.0, 2.0, 2.0))
    u = oracle_lib.init_brill_lindquist(g, [0.5], [[0.1, 0.0, 0.0]])
    a, ev1 = run_steps(gb, g, u, Params(), 0.05, 5, gb.BC_REFERENCE)
    b, ev2 = run_steps(gb, g, u, Params(), 0.05, 5, gb.BC_REFERENCE)
    assert np.array_equal(a, b)
    assert ev1.launch_count() > 0


def test_nonfinite_state_is_floored_and_counted(gb, oracle_lib):
    # failure detection without a GPU fault: a NaN poked into the host state
    # before upload is repaired by the floors (main.cpp:586-608) and counted
    g = Geom((16, 16, 16), (-2.0, -2.0, -2.0), (2.0, 2.0, 2.0))
    u = oracle_lib.init_flat(g)
    u[0, 10, 10, 10] = np.nan
    u[18, 9, 9, 9] = np.inf
    ref = oracle_lib.rk3_steps(Params(), g, u, 0.01, 1)
    out, ev = run_steps(gb, g, u, Params(), 0.01, 1, gb.BC_REFERENCE)
    assert ev.nonfinite_count() > 0
    np.testing.assert_array_equal(np.isfinite(out), np.isfinite(ref))


def test_fma_rate_probe(gb):
    # the compute roofline bench.py reports: FP64 and FP32 FMA rates of the device
    f64 = gb.measure_fma_rate(0, gb.PRECISION_FP64)
    f32 = gb.measure_fma_rate(0, gb.PRECISION_MIXED)
    assert 1.0 < f64 < 1000.0 and 1.0 < f32 < 1000.0
    assert f32 >= f64
