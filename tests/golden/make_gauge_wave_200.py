"""Generate tests/golden/gauge_wave_48_200steps.npz with the compiled GRANITE reference.

The gauge-wave workload (48^3 on [-0.5, 0.5]^3, g_xx = 1 - 0.1 sin(2 pi x),
periodic, CFL 0.25, KO sigma = 0.1) evolved 200 RK3 steps by the reference's
own RHS and the restated RK3 loop (strict IEEE build). The full state of every
step would be 31 MB each, so per step and per field the fixture keeps the L2
norm and max |u| over the interior and the values at 8 seeded interior points,
plus the Hamiltonian / momentum constraint L2 norms of the reference monitor.

The evolution amplifies rounding differences (the fields grow several-fold
over the run), so the fixture also records `fast_drift`: per step, how far the
reference's own Release build (-O3 -ffast-math) is from the strict build, as
the largest deviation of the L2 norms and samples divided by the field's
tensor-group scale. A faithful FP64 implementation drifts by about as much.

    python tests/golden/make_gauge_wave_200.py      (takes a few minutes)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import Geom, Params  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gauge_wave_48_200steps.npz")
N, STEPS, NSAMPLE = 48, 200, 8
GEOM = Geom((N, N, N), (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))
GROUPS = [[0], [1, 2, 3, 4, 5, 6], [7, 8, 9, 10, 11, 12], [13], [14, 15, 16], [17], [18], [19, 20, 21]]


def group_scale(maxabs):
    s = np.zeros(22)
    for g in GROUPS:
        s[g] = maxabs[g].max()
    return np.maximum(s, 1e-300)


def sample_points(seed: int = 2024):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.integers(0, N, size=(NSAMPLE, 3))


def step_stats(u, pts):
    it = u[GEOM.interior()]
    flat = it.reshape(22, -1)
    l2 = np.sqrt(np.mean(flat * flat, axis=1))
    mx = np.abs(flat).max(axis=1)
    samples = np.stack([it[:, i, j, k] for i, j, k in pts], axis=1)  # (22, NSAMPLE)
    return l2, mx, samples


def constraint_norms(ref, u):
    ham, mom = ref.constraints(GEOM, u)
    sl = GEOM.interior()[1:]
    h = ham.reshape(GEOM.shape[1:])[sl]
    m = mom.reshape(GEOM.shape[1:] + (3,))[sl]
    return np.sqrt(np.mean(h * h)), np.sqrt(np.mean(np.sum(m * m, axis=-1)))


def main():
    oracle.build()
    ref = oracle.Reference("strict")
    p = Params()
    u = ref.init_gauge_wave(GEOM, -0.1, 1.0)
    dt = 0.25 * GEOM.dx[0]
    pts = sample_points()
    fast = oracle.Reference("fast")
    uf = u.copy()
    l2s, mxs, sams, hs, ms, drift = [], [], [], [], [], []
    for s in range(STEPS):
        u = ref.rk3_steps(p, GEOM, u, dt, 1, bc=oracle.BC_PERIODIC)
        uf = fast.rk3_steps(p, GEOM, uf, dt, 1, bc=oracle.BC_PERIODIC)
        l2, mx, sam = step_stats(u, pts)
        l2f, _, samf = step_stats(uf, pts)
        gs = group_scale(mx)
        drift.append(max((np.abs(l2f - l2) / gs).max(), (np.abs(samf - sam) / gs[:, None]).max()))
        h, m = constraint_norms(ref, u)
        l2s.append(l2); mxs.append(mx); sams.append(sam); hs.append(h); ms.append(m)
        if s % 20 == 19:
            print(f"step {s + 1}: ||H|| = {h:.6e}, Release-build drift {drift[-1]:.2e}", flush=True)
    np.savez_compressed(OUT, n=N, steps=STEPS, dt=dt, points=pts, l2=np.array(l2s), maxabs=np.array(mxs),
                        samples=np.array(sams), h_l2=np.array(hs), m_l2=np.array(ms), fast_drift=np.array(drift),
                        amplitude=-0.1, wavelength=1.0)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
