"""Pin the CPU oracle (oracle/ccz4_oracle.c) before trusting it.

1. Against the committed golden vectors (tests/golden, produced by the compiled
   reference): bit for bit.
2. Against the compiled reference itself (oracle/_ref) on fresh seeded inputs,
   where the reference tree was available to build it: bit for bit.
3. Against the known answers of the reference's own tests
   (tests/spacetime/test_ccz4_flat.cpp, test_gauge_wave.cpp,
   tests/initial_data/test_brill_lindquist.cpp, tests/amr/test_amr_basic.cpp).
"""
import glob
import math
import os

import numpy as np
import pytest

import oracle
from oracle import Geom, Params

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    g = Geom(tuple(int(x) for x in z["n"]), tuple(float(x) for x in z["lo"]),
             tuple(float(x) for x in z["hi"]), int(z["ng"]))
    return g, z


BL_M = [0.5, 0.5]
BL_X = [[0.7, 0.1, -0.05], [-0.8, -0.05, 0.1]]


def test_golden_files_present():
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLD, "*.npz"))}
    for n in ["rhs_random", "rhs_matter", "rhs_random_noko", "constraints_random", "ko_random",
              "rhs_bl", "constraints_bl", "rk3_bl_3steps", "init_bl", "init_gauge_wave",
              "rk3_gauge_wave_periodic_4steps", "prolong", "restrict", "matter_sources", "psi4_modes",
              "horizon_flow", "horizon_all", "horizon_all_binary"]:
        assert n in names, n


@pytest.mark.parametrize("name,ko", [("rhs_random", 0.1), ("rhs_random_noko", 0.0)])
def test_oracle_rhs_golden(oracle_lib, name, ko):
    g, z = load(name)
    u = oracle.seeded_state(g, int(z["seed"]))
    out = oracle_lib.rhs(Params(ko_sigma=ko), g, u)
    assert np.array_equal(out[g.interior()], z["rhs"])


def test_oracle_rhs_matter_golden(oracle_lib):
    g, z = load("rhs_matter")
    u = oracle.seeded_state(g, int(z["seed"]))
    m = oracle.seeded_matter(g, int(z["matter_seed"]))
    out = oracle_lib.rhs(Params(), g, u, *m)
    assert np.array_equal(out[g.interior()], z["rhs"])


def test_oracle_matter_sources_golden(oracle_lib):
    """GRMHDEvolution::computeMatterSources (grmhd.cpp:1034-1103), with cells of
    v^2 >= 1 (the W clamp) and of zero density among them."""
    g, z = load("matter_sources")
    prim = oracle.seeded_primitives(g, int(z["seed"]), superluminal=float(z["superluminal"]))
    assert (prim[1] ** 2 + prim[2] ** 2 + prim[3] ** 2 >= 1.0).any() and (prim[0] == 0.0).any()
    out = oracle_lib.matter_sources(g, prim)
    it = g.interior()[1:]
    for a, name in zip(out, ("rho", "Si", "Sij", "S")):
        assert np.array_equal(a[it], z[name]), name
        rest = np.ones(a.shape[:3], dtype=bool)
        rest[it] = False
        assert not a[rest].any(), f"{name}: a cell outside the interior was written"


@pytest.mark.skipif(not oracle.reference_available("strict"), reason="reference library not built")
@pytest.mark.parametrize("seed,superluminal", [(3, 0.0), (4, 0.3), (5, 1.0)])
def test_oracle_matter_sources_vs_reference(oracle_lib, seed, superluminal):
    ref = oracle.Reference("strict")
    g = Geom((9, 7, 5), (-1.0, 0.0, 2.0), (0.8, 1.4, 3.0))
    prim = oracle.seeded_primitives(g, seed, superluminal)
    init = tuple(oracle.hash_noise(a.shape, 90 + k) for k, a in enumerate(oracle.matter_zeros(g)))
    for a, b in zip(oracle_lib.matter_sources(g, prim, init), ref.matter_sources(g, prim, init)):
        assert np.array_equal(a, b)


def test_oracle_psi4_golden(oracle_lib):
    """Psi4Extractor::extract + getMode (postprocess.cpp:245-326) on a seeded block,
    radii fully inside, partly inside and outside it."""
    g, z = load("psi4_modes")
    u = oracle.seeded_state(g, int(z["seed"]))
    got, npts = oracle_lib.psi4_modes(g, u, z["radii"], int(z["n_theta"]), int(z["n_phi"]), int(z["l_max"]),
                                      counts=True)
    assert np.array_equal(got, z["modes"])
    full = int(z["n_theta"]) * int(z["n_phi"])
    assert npts[0] == full and 0 < npts[3] < full and npts[-1] == 0


@pytest.mark.skipif(not oracle.reference_available("strict"), reason="reference library not built")
@pytest.mark.parametrize("l_max,nth,nph", [(2, 8, 12), (5, 21, 17), (3, 40, 80)])
def test_oracle_psi4_vs_reference(oracle_lib, l_max, nth, nph):
    ref = oracle.Reference("strict")
    g = Geom((20, 18, 16), (-5.0, -4.5, -4.0), (5.0, 4.5, 4.0))
    u = oracle.seeded_state(g, 8)
    radii = [1.0, 2.5, 4.2]
    assert np.array_equal(oracle_lib.psi4_modes(g, u, radii, nth, nph, l_max),
                          ref.psi4_modes(g, u, radii, nth, nph, l_max))


def test_oracle_horizon_golden(oracle_lib):
    """findHorizon (horizon_finder.cpp:310-449): the flow, its converged iteration
    and the surface integrals, bit for bit."""
    g, z = load("horizon_flow")
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.0, 0.0, 0.0]]) + 1e-9 * oracle.hash_noise(g.shape, int(z["seed"]))
    it, h, res = oracle_lib.find_horizon(g, u, (0.0, 0.0, 0.0), int(z["max_iterations"]), float(z["tolerance"]),
                                         int(z["angular_resolution"]), float(z["initial_guess_radius"]))
    assert it > 0 and np.array_equal(res, z["res"])
    from granite_b200.horizon import surface_points
    assert np.array_equal(np.array(surface_points((0.0, 0.0, 0.0), h)), z["surface"])


@pytest.mark.skipif(not oracle.reference_available("strict"), reason="reference library not built")
def test_oracle_horizon_vs_reference(oracle_lib):
    ref = oracle.Reference("strict")
    g = Geom((24, 20, 22), (-1.2, -1.0, -1.1), (1.2, 1.0, 1.1))
    u = ref.init_brill_lindquist(g, [0.8], [[0.0, 0.0, 0.0]]) + 1e-7 * oracle.hash_noise(g.shape, 3)
    for center, tol in [((0.0, 0.0, 0.0), 1e-2), ((0.02, -0.01, 0.03), 1e-2), ((0.0, 0.0, 0.0), 1e-12)]:
        it, h, res = oracle_lib.find_horizon(g, u, center, 800, tol, 6, 0.9)
        found, rres, surf = ref.find_horizon(g, u, center, 800, tol, 6, 0.9)
        assert found == (it > 0) and np.array_equal(res, rres)
        if found:
            from granite_b200.horizon import surface_points
            assert np.array_equal(np.array(surface_points(center, h)), surf)


def test_oracle_constraints_golden(oracle_lib):
    g, z = load("constraints_random")
    u = oracle.seeded_state(g, int(z["seed"]))
    h, m = oracle_lib.constraints(g, u)
    it = g.interior()[1:]
    assert np.array_equal(h[it], z["ham"])
    assert np.array_equal(m[it], z["mom"])


def test_oracle_ko_golden(oracle_lib):
    g, z = load("ko_random")
    u = oracle.seeded_state(g, int(z["seed"]))
    ko = oracle_lib.dissipation(Params(), g, u, np.zeros(g.shape))
    assert np.array_equal(ko[g.interior()], z["ko"])


def _bl_state(o, g, seed):
    u = o.init_brill_lindquist(g, BL_M, BL_X)
    return u + 1e-6 * oracle.hash_noise(g.shape, seed)


def test_oracle_bl_golden(oracle_lib):
    g, z = load("init_bl")
    u = oracle_lib.init_brill_lindquist(g, BL_M, BL_X)
    assert np.array_equal(u[list(z["fields"])], z["u"])
    g, z = load("rhs_bl")
    out = oracle_lib.rhs(Params(), g, _bl_state(oracle_lib, g, int(z["seed"])))
    assert np.array_equal(out[g.interior()], z["rhs"])
    g, z = load("constraints_bl")
    h, m = oracle_lib.constraints(g, _bl_state(oracle_lib, g, int(z["seed"])))
    it = g.interior()[1:]
    assert np.array_equal(h[it], z["ham"]) and np.array_equal(m[it], z["mom"])


def test_oracle_rk3_golden(oracle_lib):
    g, z = load("rk3_bl_3steps")
    u = _bl_state(oracle_lib, g, int(z["seed"]))
    out = oracle_lib.rk3_steps(Params(), g, u, float(z["dt"]), int(z["nsteps"]))
    assert np.array_equal(out[g.interior()], z["u"])


def test_oracle_gauge_wave_golden(oracle_lib):
    g, z = load("init_gauge_wave")
    u = oracle_lib.init_gauge_wave(g, float(z["amplitude"]), float(z["wavelength"]))
    assert np.array_equal(u, z["u"])
    g2, z2 = load("rk3_gauge_wave_periodic_4steps")
    out = oracle_lib.rk3_steps(Params(), g2, u, float(z2["dt"]), int(z2["nsteps"]),
                               bc=oracle.BC_PERIODIC)
    assert np.array_equal(out[g2.interior()], z2["u"])


def test_oracle_prolong_restrict_golden(oracle_lib):
    gf, zf = load("prolong")
    gc, zc = load("restrict")
    uc = oracle.seeded_state(gc, int(zf["seed_c"]))
    uf = oracle.seeded_state(gf, int(zf["seed_f"]))
    assert np.array_equal(oracle_lib.prolongate(gc, uc, gf, uf)[:4], zf["u"])
    assert np.array_equal(oracle_lib.restrict(gf, uf, gc, uc)[gc.interior()], zc["u"])


# ---------------------------------------------------------------------------
# against the compiled reference on fresh inputs
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("seed", [101, 202])
def test_oracle_equals_reference_random(oracle_lib, reference_lib, seed):
    g = Geom((9, 7, 11), (-0.6, -1.1, -0.4), (0.9, 0.3, 1.2))
    u = oracle.seeded_state(g, seed, amp=0.1, noise=1e-2)
    p = Params(kappa1=0.05, kappa2=0.1, eta=1.5, ko_sigma=0.3)
    assert np.array_equal(oracle_lib.rhs(p, g, u), reference_lib.rhs(p, g, u))
    m = oracle.seeded_matter(g, seed + 7)
    assert np.array_equal(oracle_lib.rhs(p, g, u, *m), reference_lib.rhs(p, g, u, *m))
    h1, m1 = oracle_lib.constraints(g, u)
    h2, m2 = reference_lib.constraints(g, u)
    assert np.array_equal(h1, h2) and np.array_equal(m1, m2)


def test_oracle_equals_reference_rk3(oracle_lib, reference_lib):
    g = Geom((12, 10, 8), (-3.0, -2.5, -2.0), (3.0, 2.5, 2.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.1, -0.2, 0.05]])
    u = u + 1e-6 * oracle.hash_noise(g.shape, 5)
    dt = 0.25 * g.dx[0]
    a = oracle_lib.rk3_steps(Params(), g, u, dt, 4)
    b = reference_lib.rk3_steps(Params(), g, u, dt, 4)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("bc", [oracle.BC_SOMMERFELD, oracle.BC_PERIODIC])
def test_oracle_equals_reference_rk3_with_matter(oracle_lib, reference_lib, bc):
    """The oracle's RK3 step with fixed matter sources (the checker of the resident
    matter path) against the reference's computeRHS with the same sources in
    every stage, sources from the compiled computeMatterSources."""
    g = Geom((12, 10, 8), (-3.0, -2.5, -2.0), (3.0, 2.5, 2.0))
    u = oracle_lib.init_brill_lindquist(g, [1.0], [[0.1, -0.2, 0.05]])
    u = u + 1e-6 * oracle.hash_noise(g.shape, 6)
    prim = oracle.seeded_primitives(g, 31, superluminal=0.0)
    prim[0] *= 1e-3  # a dilute, weakly magnetised fluid: the coupling acts, the state stays finite
    prim[4] *= 1e-4
    prim[5:8] *= 1e-2
    m = reference_lib.matter_sources(g, prim)
    dt = 0.25 * g.dx[0]
    a = oracle_lib.rk3_steps(Params(), g, u, dt, 3, bc, matter=m)
    b = reference_lib.rk3_steps(Params(), g, u, dt, 3, bc, matter=m)
    assert np.isfinite(a).all() and np.array_equal(a, b)
    assert not np.array_equal(a, reference_lib.rk3_steps(Params(), g, u, dt, 3, bc))


def test_oracle_level_fill_equals_reference(oracle_lib, reference_lib):
    g = Geom((6, 5, 7), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    u = oracle.seeded_state(g, 9)
    a = oracle_lib.fill(g, u.copy(), "zero_gradient")
    assert np.array_equal(a, reference_lib.fill_level0(g, u))


# ---------------------------------------------------------------------------
# known answers of the reference's own tests
# ---------------------------------------------------------------------------

def test_known_answers_brill_lindquist(oracle_lib):
    # test_brill_lindquist.cpp:16-100
    one = [[0.0, 0.0, 0.0]]
    assert abs(oracle_lib.bl_conformal_factor([1.0], one, 1.0, 0, 0) - 1.5) < 1e-10
    assert abs(oracle_lib.bl_conformal_factor([1.0], one, 0.5, 0, 0) - 2.0) < 1e-10
    two = [[5.0, 0, 0], [-5.0, 0, 0]]
    assert abs(oracle_lib.bl_conformal_factor([1, 1], two, 3, 0, 0)
               - oracle_lib.bl_conformal_factor([1, 1], two, -3, 0, 0)) < 1e-10
    assert abs(oracle_lib.bl_conformal_factor([1, 1], two, 0, 0, 0) - 1.2) < 1e-10
    pent = [[10 * math.cos(2 * math.pi * a / 5), 10 * math.sin(2 * math.pi * a / 5), 0.0]
            for a in range(5)]
    assert abs(oracle_lib.bl_conformal_factor([1.0] * 5, pent, 0, 0, 0) - 1.25) < 1e-10
    prev = 1e100
    for r in [0.1, 0.5, 1.0, 2.0, 5.0, 10.0, 50.0]:
        psi = oracle_lib.bl_conformal_factor([1.0], one, r, 0, 0)
        assert psi < prev
        prev = psi
    assert abs(oracle_lib.bl_conformal_factor([1.0], one, 1000, 0, 0) - 1.0) < 1e-3


def test_known_answers_flat(oracle_lib):
    # test_ccz4_flat.cpp:22-63,106-150,192-230
    g = Geom((32, 32, 32), (-10.0, -10.0, -10.0), (10.0, 10.0, 10.0))
    u = oracle_lib.init_flat(g)
    rhs = oracle_lib.rhs(Params(ko_sigma=0.0), g, u)
    assert np.abs(rhs[g.interior()]).max() < 1e-10
    h, m = oracle_lib.constraints(g, u)
    assert np.abs(h).max() < 1e-10 and np.abs(m).max() < 1e-10
    ko = oracle_lib.rhs(Params(ko_sigma=0.35), g, u)
    assert np.abs(ko[g.interior()]).max() < 1e-12


def test_known_answers_gauge_wave(oracle_lib):
    # test_gauge_wave.cpp:26-89
    g = Geom((64, 8, 8), (0.0, 0.0, 0.0), (1.0, 0.125, 0.125))
    u = oracle_lib.init_gauge_wave(g, 0.01, 1.0)
    iq = 4 + 64 // 4
    assert abs(u[18, 8, 8, iq] - math.sqrt(1.01)) < 1e-4
    x = g.x(0, 4)
    H = 1.0 + 0.01 * math.sin(2 * math.pi * x)
    assert abs(u[0, 8, 8, 4] - H ** (-1.0 / 3.0)) < 5 * g.dx[0] ** 2
    rhs = oracle_lib.rhs(Params(ko_sigma=0.1), g, u)
    assert np.isfinite(rhs[g.interior()]).all()
    assert np.abs(rhs[g.interior()]).max() < 100.0


def test_known_answers_amr_constants(oracle_lib):
    # test_amr_basic.cpp:110-184
    gc = Geom((8, 8, 8), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    gf = Geom((8, 8, 8), (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))
    uc = np.full(gc.shape, 42.0)
    uf = oracle_lib.prolongate(gc, uc, gf, np.zeros(gf.shape))
    assert np.abs(uf[gf.interior()] - 42.0).max() < 1e-12
    uf = np.full(gf.shape, 3.14159)
    uc = oracle_lib.restrict(gf, uf, gc, np.zeros(gc.shape))
    err = 0.0
    for k in range(4, 12):
        for j in range(4, 12):
            for i in range(4, 12):
                if all(-0.5 <= gc.x(d, c) <= 0.5 for d, c in ((0, i), (1, j), (2, k))):
                    err = max(err, np.abs(uc[:, k, j, i] - 3.14159).max())
    assert err < 1e-12
