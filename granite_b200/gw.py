"""Gravitational-wave extraction with the reference's Psi4Extractor interface.

``Psi4Extractor.extract`` (postprocess.cpp:245-314) runs on the GPU
(``granite_ccz4_psi4_modes*``): Psi4 on coordinate spheres from the state of a
device-resident block (or a host GridBlock) and its projection on the
spin-weight -2 harmonics. The time series it accumulates and the analysis
built on them (strain, radiated energy, spectrum, extrapolation;
postprocess.cpp:316-475) are small host-side arrays and stay in Python, in
the reference's arithmetic.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import GridBlock, _dp, _f64

PI = 3.14159265358979323846  # constants::PI (types.hpp:71)


@dataclass
class GWExtractionParams:
    """postprocess.hpp:23-28."""
    extraction_radii: list = field(default_factory=lambda: [100.0, 200.0, 300.0, 500.0])
    l_max: int = 4
    n_theta: int = 100
    n_phi: int = 200


def mode_list(l_max: int):
    """(l, m) in the order of the mode arrays: l = 2..l_max, m = -l..l."""
    return [(l, m) for l in range(2, l_max + 1) for m in range(-l, l + 1)]


class Psi4Extractor:
    """postprocess.hpp:34-69: data[r][(l, m)] = [(time, Psi4^lm)]."""

    def __init__(self, params: GWExtractionParams | None = None):
        self.params = params or GWExtractionParams()
        self.data: dict = {}

    def _modes(self, call):
        p = self.params
        radii = np.ascontiguousarray(p.extraction_radii, dtype=np.float64)
        nm = (p.l_max + 1) ** 2 - 4
        out = np.zeros((len(radii), nm, 2))
        npts = (C.c_int * len(radii))()
        call(_dp(radii), len(radii), p.n_theta, p.n_phi, p.l_max, _dp(out), npts)
        return radii, out[..., 0] + 1j * out[..., 1], list(npts)

    def _record(self, time, radii, modes, npts):
        keys = mode_list(self.params.l_max)
        for r, (r_ext, n) in enumerate(zip(radii, npts)):
            if n == 0:  # no sphere point inside the block: the reference records nothing
                continue
            per_r = self.data.setdefault(float(r_ext), {})
            for q, key in enumerate(keys):
                series = per_r.setdefault(key, [])
                if series and series[-1][0] == time:
                    series[-1] = (time, series[-1][1] + modes[r, q])
                else:
                    series.append((time, complex(modes[r, q])))

    def extract(self, evolver, block_index: int, time: float):
        """Psi4Extractor::extract on block ``block_index`` of a committed Evolver."""
        ctx = evolver.ctx

        def call(*a):
            ctx.check(ctx.lib.granite_ccz4_psi4_modes(ctx.h, block_index, *a))

        self._record(time, *self._modes(call))

    def extract_block(self, runner, spacetime: GridBlock, time: float):
        """Psi4Extractor::extract on a host GridBlock; ``runner`` is any object of this
        package with a context (a CCZ4Evolution, an Evolver); the block is copied in."""
        c = runner.ctx

        def call(*a):
            c.check(c.lib.granite_ccz4_psi4_modes_host(c.h, C.byref(spacetime.desc()), _dp(_f64(spacetime.array)),
                                                      *a))

        self._record(time, *self._modes(call))

    # -- host analysis, postprocess.cpp:316-475 -----------------------------
    def getTimeSeries(self, l: int, m: int, r_ext: float):
        return self.data.get(float(r_ext), {}).get((l, m), [])

    def getMode(self, l: int, m: int, r_ext: float) -> complex:
        s = self.getTimeSeries(l, m, r_ext)
        return s[-1][1] if s else 0j

    def computeStrain(self, l: int, m: int, r_ext: float) -> complex:
        """Trapezoid double integration of the mode (postprocess.cpp:328-353)."""
        s = self.getTimeSeries(l, m, r_ext)
        if len(s) < 3:
            return 0j
        h_dot, h = 0j, 0j
        for i in range(1, len(s)):
            dt = s[i][0] - s[i - 1][0]
            h_dot += 0.5 * (s[i][1] + s[i - 1][1]) * dt
            h += h_dot * dt
        return h

    def computeRadiatedEnergy(self, r_ext: float) -> float:
        """r^2 / (16 pi) times the sum over modes of the time integral of |h_dot|^2
        (postprocess.cpp:355-377)."""
        per_r = self.data.get(float(r_ext))
        if per_r is None:
            return 0.0
        E = 0.0
        for key in sorted(per_r):
            s = per_r[key]
            if len(s) < 2:
                continue
            hdot = 0j
            for i in range(1, len(s)):
                dt = s[i][0] - s[i - 1][0]
                hdot += 0.5 * (s[i][1] + s[i - 1][1]) * dt
                E += (hdot.real * hdot.real + hdot.imag * hdot.imag) * dt
        return r_ext * r_ext / (16.0 * PI) * E

    def computeRadiatedMomentum(self, r_ext: float):
        """Zero, as the reference returns (postprocess.cpp:379-385)."""
        return (0.0, 0.0, 0.0)

    def computeEnergySpectrum(self, l: int, m: int, r_ext: float):
        """(f, dE/df) from a direct DFT of the doubly integrated mode (postprocess.cpp:387-433)."""
        s = self.getTimeSeries(l, m, r_ext)
        N = len(s)
        if N < 2:
            return []
        T = s[-1][0] - s[0][0]
        dt = T / (N - 1)
        h = [0j] * N
        h_dot, h_val = 0j, 0j
        for i in range(1, N):
            dti = s[i][0] - s[i - 1][0]
            h_dot += 0.5 * (s[i][1] + s[i - 1][1]) * dti
            h_val += h_dot * dti
            h[i] = h_val
        out = []
        df = 1.0 / T
        for k in range(min(N // 2, 500)):
            f = k * df
            ht = 0j
            for i in range(N):
                phase = -2.0 * PI * f * s[i][0]
                ht += h[i] * complex(math.cos(phase), math.sin(phase)) * dt
            out.append((f, (PI * r_ext * r_ext / 2.0) * f * f * (ht.real * ht.real + ht.imag * ht.imag)))
        return out

    def extrapolateToInfinity(self, l: int, m: int) -> complex:
        """Richardson extrapolation in 1/r over the two outermost radii (postprocess.cpp:435-456)."""
        radii = self.params.extraction_radii
        if len(radii) < 2:
            return self.getMode(l, m, radii[-1] if radii else 0.0)
        r1, r2 = radii[-2], radii[-1]
        p1, p2 = self.getMode(l, m, r1), self.getMode(l, m, r2)
        r1sq, r2sq = r1 * r1, r2 * r2
        denom = r1sq - r2sq
        if abs(denom) < 1.0e-12:
            return p2
        return (r1sq * p2 - r2sq * p1) / denom
