"""Initial data for the workloads (host side; not on the hot path).

Vectorised numpy versions of the reference routines:
  set_flat_spacetime      ccz4.cpp:1165-1188
  set_gauge_wave_data     ccz4.cpp:1190-1221
  brill_lindquist         initial_data.cpp:79-158 (optional floor on r)
"""
from __future__ import annotations

import numpy as np

CHI, GXX, GXY, GXZ, GYY, GYZ, GZZ = 0, 1, 2, 3, 4, 5, 6
AXX = 7
KTR = 13
GHX, GHY, GHZ = 14, 15, 16
THETA, ALPHA = 17, 18
BETAX = 19
PI = 3.14159265358979323846


def _coords(block):
    nz, ny, nx = block.array.shape[1:]
    X = np.array([block.x(0, i) for i in range(nx)])[None, None, :]
    Y = np.array([block.x(1, j) for j in range(ny)])[None, :, None]
    Z = np.array([block.x(2, k) for k in range(nz)])[:, None, None]
    return X, Y, Z


def set_flat_spacetime(block):
    a = block.array
    a[CHI] = 1.0
    a[GXX] = 1.0
    a[GXY] = 0.0
    a[GXZ] = 0.0
    a[GYY] = 1.0
    a[GYZ] = 0.0
    a[GZZ] = 1.0
    a[ALPHA] = 1.0
    return block


def set_gauge_wave_data(block, amplitude: float, wavelength: float):
    """gamma_xx = (1 + H) chi-conformal, alpha = sqrt(1 + H), H = A sin(2 pi x / L).

    amplitude < 0 gives the g_xx = 1 - |A| sin(2 pi x) variant of the gauge-wave workload."""
    X, _, _ = _coords(block)
    H = amplitude * np.sin(2.0 * PI * X / wavelength)
    chi = np.power(1.0 + H, -1.0 / 3.0)
    a = block.array
    shape = a.shape[1:]
    a[CHI] = np.broadcast_to(chi, shape)
    a[GXX] = np.broadcast_to((1.0 + H) * chi, shape)
    a[GXY] = 0.0
    a[GXZ] = 0.0
    a[GYY] = np.broadcast_to(chi, shape)
    a[GYZ] = 0.0
    a[GZZ] = np.broadcast_to(chi, shape)
    a[ALPHA] = np.broadcast_to(np.sqrt(1.0 + H), shape)
    return block


def gauge_wave(block, amplitude: float = -0.1, wavelength: float = 1.0):
    block.array[:] = 0.0
    return set_gauge_wave_data(block, amplitude, wavelength)


def brill_lindquist(block, masses, positions, r_floor: float = 0.0):
    """Brill-Lindquist punctures: psi = 1 + sum m/(2r), chi = psi^-4, alpha = psi^-2,
    Gamma-hat^i = (8/3) d_i psi / psi (analytic), everything else flat."""
    X, Y, Z = _coords(block)
    shape = block.array.shape[1:]
    psi = np.ones(shape)
    dpx = np.zeros(shape)
    dpy = np.zeros(shape)
    dpz = np.zeros(shape)
    for m, p in zip(masses, positions):
        dx, dy, dz = X - p[0], Y - p[1], Z - p[2]
        r = np.sqrt(dx * dx + dy * dy + dz * dz + 1.0e-30)
        r = np.maximum(r, r_floor)
        psi = psi + m / (2.0 * r)
        r2 = dx * dx + dy * dy + dz * dz + 1.0e-20
        r2 = np.maximum(r2, r_floor * r_floor)
        r3 = r2 * np.sqrt(r2)
        c = -m / (2.0 * r3)
        dpx = dpx + c * dx
        dpy = dpy + c * dy
        dpz = dpz + c * dz
    a = block.array
    a[:] = 0.0
    set_flat_spacetime(block)
    psi2 = psi * psi
    chi = 1.0 / (psi2 * psi2)
    a[CHI] = chi
    a[ALPHA] = np.sqrt(chi)
    gf = 8.0 / (3.0 * psi)
    a[GHX] = gf * dpx
    a[GHY] = gf * dpy
    a[GHZ] = gf * dpz
    return block


def add_noise(block, amplitude: float, seed: int):
    """Uniform(-a, a) on all fields and cells from a seeded PCG64 stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    block.array += rng.uniform(-amplitude, amplitude, size=block.array.shape)
    return block
