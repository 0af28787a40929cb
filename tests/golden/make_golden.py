"""Generate tests/golden/*.npz by running the compiled GRANITE reference.

Run where the reference tree is present (it builds oracle/_ref from it):

    python tests/golden/make_golden.py

Inputs are not stored: they are rebuilt from oracle.seeded_state /
oracle.seeded_matter / oracle.seeded_primitives (IEEE + and * plus an integer
hash, so identical on any host). Outputs of the reference (strict IEEE build) are stored, interior cells
only, float64. Each case records its geometry and parameters.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import Geom, Params  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, geometry) of the small blocks used by the cases
G_RAND = Geom((10, 8, 6), (-1.0, -0.8, -0.7), (1.0, 0.9, 0.6))
G_BL = Geom((8, 8, 8), (-2.0, -2.0, -2.0), (2.0, 2.0, 2.0))
G_GW = Geom((16, 4, 4), (-0.5, -0.5, -0.5), (0.5, -0.25, -0.25))
G_C = Geom((8, 8, 8), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
G_F = Geom((6, 4, 4), (-0.375, -0.25, -0.25), (0.375, 0.25, 0.25))
BL_M = [0.5, 0.5]
BL_X = [[0.7, 0.1, -0.05], [-0.8, -0.05, 0.1]]
INIT_FIELDS = [0, 14, 15, 16, 18]  # chi, Gamma-hat, alpha: the fields BL sets non-trivially


def geom_dict(g: Geom):
    return dict(n=np.array(g.n), lo=np.array(g.lo), hi=np.array(g.hi), ng=g.ng)


def bl_noise_state(ref, g: Geom, seed: int):
    u = ref.init_brill_lindquist(g, BL_M, BL_X)
    return u + 1e-6 * oracle.hash_noise(g.shape, seed)


def main():
    oracle.build()
    ref = oracle.Reference("strict")
    p = Params()
    cases = {}

    u = oracle.seeded_state(G_RAND, 11)
    cases["rhs_random"] = (G_RAND, dict(rhs=ref.rhs(p, G_RAND, u)[G_RAND.interior()], seed=11))
    m = oracle.seeded_matter(G_RAND, 12)
    cases["rhs_matter"] = (G_RAND, dict(rhs=ref.rhs(p, G_RAND, u, *m)[G_RAND.interior()], seed=11,
                                        matter_seed=12))
    p0 = Params(ko_sigma=0.0)
    cases["rhs_random_noko"] = (G_RAND, dict(rhs=ref.rhs(p0, G_RAND, u)[G_RAND.interior()], seed=11))
    ham, mom = ref.constraints(G_RAND, u)
    it = G_RAND.interior()[1:]
    cases["constraints_random"] = (G_RAND, dict(ham=ham[it], mom=mom[it], seed=11))
    ko = ref.dissipation(p, G_RAND, u, np.zeros(G_RAND.shape))
    cases["ko_random"] = (G_RAND, dict(ko=ko[G_RAND.interior()], seed=11))

    ub = bl_noise_state(ref, G_BL, 21)
    cases["rhs_bl"] = (G_BL, dict(rhs=ref.rhs(p, G_BL, ub)[G_BL.interior()], seed=21))
    hb, mb = ref.constraints(G_BL, ub)
    itb = G_BL.interior()[1:]
    cases["constraints_bl"] = (G_BL, dict(ham=hb[itb], mom=mb[itb], seed=21))
    dt = 0.25 * G_BL.dx[0]
    cases["rk3_bl_3steps"] = (G_BL, dict(u=ref.rk3_steps(p, G_BL, ub, dt, 3)[G_BL.interior()],
                                         seed=21, dt=dt, nsteps=3))
    cases["init_bl"] = (G_BL, dict(u=ref.init_brill_lindquist(G_BL, BL_M, BL_X)[INIT_FIELDS],
                                   fields=np.array(INIT_FIELDS)))

    ug = ref.init_gauge_wave(G_GW, -0.1, 1.0)
    cases["init_gauge_wave"] = (G_GW, dict(u=ug, amplitude=-0.1, wavelength=1.0))
    dtg = 0.25 * G_GW.dx[0]
    cases["rk3_gauge_wave_periodic_4steps"] = (
        G_GW, dict(u=ref.rk3_steps(p, G_GW, ug, dtg, 4, bc=oracle.BC_PERIODIC)[G_GW.interior()],
                   dt=dtg, nsteps=4))

    uc = oracle.seeded_state(G_C, 31)
    uf = oracle.seeded_state(G_F, 32)
    cases["prolong"] = (G_F, dict(u=ref.prolongate(G_C, uc, 0, G_F, uf, 1)[:4], seed_c=31, seed_f=32))
    cases["restrict"] = (G_C, dict(u=ref.restrict(G_F, uf, 1, G_C, uc, 0)[G_C.interior()], seed_c=31,
                                  seed_f=32))

    prim = oracle.seeded_primitives(G_RAND, 41, superluminal=0.05)
    rho, Si, Sij, S = ref.matter_sources(G_RAND, prim)
    it = G_RAND.interior()[1:]
    cases["matter_sources"] = (G_RAND, dict(rho=rho[it], Si=Si[it], Sij=Sij[it], S=S[it], seed=41,
                                            superluminal=0.05))

    gp = Geom((24, 20, 22), (-12.0, -10.0, -11.0), (12.0, 10.0, 11.0))
    up = oracle.seeded_state(gp, 51)
    radii = np.array([3.0, 6.5, 9.7, 10.5, 20.0])
    modes = ref.psi4_modes(gp, up, radii, 16, 32, 4)
    cases["psi4_modes"] = (gp, dict(modes=modes, radii=radii, seed=51, n_theta=16, n_phi=32, l_max=4))

    gh = Geom((32, 32, 32), (-1.6, -1.6, -1.6), (1.6, 1.6, 1.6))
    uh = ref.init_brill_lindquist(gh, [1.0], [[0.0, 0.0, 0.0]]) + 1e-9 * oracle.hash_noise(gh.shape, 61)
    found, res, surf = ref.find_horizon(gh, uh, (0.0, 0.0, 0.0), 3000, 1e-2, 8, 1.0)
    assert found
    cases["horizon_flow"] = (gh, dict(res=res, surface=surf, seed=61, max_iterations=3000, tolerance=1e-2,
                                      angular_resolution=8, initial_guess_radius=1.0))
    ga = Geom((33, 33, 33), (-1.65, -1.65, -1.65), (1.65, 1.65, 1.65))
    ua = ref.init_brill_lindquist(ga, [1.0], [[0.0, 0.0, 0.0]])
    rows = ref.find_all_horizons(ga, ua, 1500, 1e-2, 8, 1.0)
    cases["horizon_all"] = (ga, dict(rows=rows, max_iterations=1500, tolerance=1e-2, angular_resolution=8,
                                     initial_guess_radius=1.0))
    g2 = Geom((41, 33, 33), (-2.05, -1.65, -1.65), (2.05, 1.65, 1.65))
    u2 = ref.init_brill_lindquist(g2, [0.6, 0.4], [[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    rows2 = ref.find_all_horizons(g2, u2, 800, 1e-2, 6, 0.4)
    cases["horizon_all_binary"] = (g2, dict(rows=rows2, max_iterations=800, tolerance=1e-2, angular_resolution=6,
                                            initial_guess_radius=0.4, masses=np.array([0.6, 0.4]),
                                            positions=np.array([[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])))

    for name, (g, data) in cases.items():
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **geom_dict(g), **data)
        print(f"{name}: {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
