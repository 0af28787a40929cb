"""CPU oracle for the CCZ4 RHS + SSP-RK3 hot path -- TEST INFRASTRUCTURE ONLY.

The product library (granite_b200) never imports this package. Only tests/,
the smoke check in __graft_entry__.py and the cpu_baseline leg of bench.py use
it, always as the checker or as the timed CPU baseline.

Two backends with one Python surface:

* ``Oracle``  -- liboracle.so, this project's C restatement (ccz4_oracle.c).
* ``Reference`` -- oracle/_ref/libgranite_ref_*.so, the reference GRANITE
  sources compiled unmodified behind ref_shim.cpp (built only where the
  reference tree is present; the built file travels with the repository).

Arrays use the reference GridBlock layout (grid.hpp:109-116): a numpy float64
array of shape (22, nz+2g, ny+2g, nx+2g), C order, i.e. u[v, k, j, i].
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NV = 22

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Geom:
    """Block geometry with the reference's conventions (grid.cpp:12-31)."""

    n: tuple  # interior cells (nx, ny, nz)
    lo: tuple
    hi: tuple
    ng: int = 4

    @property
    def dx(self):
        return tuple((self.hi[d] - self.lo[d]) / self.n[d] for d in range(3))

    @property
    def shape(self):
        nx, ny, nz = self.n
        g = 2 * self.ng
        return (NV, nz + g, ny + g, nx + g)

    @property
    def cells(self):
        s = self.shape
        return s[1] * s[2] * s[3]

    def zeros(self):
        return np.zeros(self.shape, dtype=np.float64)

    def interior(self):
        g = self.ng
        nx, ny, nz = self.n
        return (slice(None), slice(g, g + nz), slice(g, g + ny), slice(g, g + nx))

    def x(self, d, idx):
        return self.lo[d] + (float(idx) - self.ng + 0.5) * self.dx[d]


class _orc_geom(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("ng", C.c_int), ("lo", C.c_double * 3),
                ("dx", C.c_double * 3)]


class _orc_params(C.Structure):
    _fields_ = [("kappa1", C.c_double), ("kappa2", C.c_double), ("eta", C.c_double),
                ("ko_sigma", C.c_double), ("chi_blend_center", C.c_double),
                ("chi_blend_width", C.c_double)]


@dataclass
class Params:
    """CCZ4Params defaults, ccz4.hpp:25-34."""

    kappa1: float = 0.02
    kappa2: float = 0.0
    eta: float = 2.0
    ko_sigma: float = 0.1
    chi_blend_center: float = 0.05
    chi_blend_width: float = 0.02

    def as6(self):
        return np.array([self.kappa1, self.kappa2, self.eta, self.ko_sigma,
                         self.chi_blend_center, self.chi_blend_width], dtype=np.float64)


BC_SOMMERFELD = 0
BC_PERIODIC = 1


def build(force: bool = False) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree exists);
    make rebuilds what is older than its sources and nothing else. Where make
    cannot run but the libraries are already built, those are used."""
    r = subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []) + ["all"], capture_output=True,
                       text=True)
    if r.returncode != 0 and (force or not os.path.exists(os.path.join(HERE, "liboracle.so"))):
        raise RuntimeError(f"oracle build failed:\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")


def _cg(g: Geom) -> _orc_geom:
    o = _orc_geom()
    for d in range(3):
        o.n[d] = g.n[d]
        o.lo[d] = g.lo[d]
        o.dx[d] = g.dx[d]
    o.ng = g.ng
    return o


def _cp(p: Params) -> _orc_params:
    return _orc_params(p.kappa1, p.kappa2, p.eta, p.ko_sigma, p.chi_blend_center,
                       p.chi_blend_width)


class Oracle:
    """This project's C restatement (liboracle.so)."""

    kind = "port"

    def __init__(self, threads: int = 0):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        if threads:
            self.lib.orc_set_threads(threads)

    def rhs(self, p: Params, g: Geom, u, rho=None, Si=None, Sij=None, S=None):
        out = g.zeros()
        self.lib.orc_rhs(C.byref(_cp(p)), C.byref(_cg(g)), _p(u), _p(out), _p(rho), _p(Si),
                         _p(Sij), _p(S))
        return out

    def dissipation(self, p: Params, g: Geom, u, rhs):
        rhs = np.array(rhs, dtype=np.float64, copy=True)
        self.lib.orc_dissipation(C.byref(_cp(p)), C.byref(_cg(g)), _p(u), _p(rhs))
        return rhs

    def constraints(self, g: Geom, u):
        ham = np.zeros(g.shape[1:], dtype=np.float64)
        mom = np.zeros(g.shape[1:] + (3,), dtype=np.float64)
        self.lib.orc_constraints(C.byref(_cg(g)), _p(u), _p(ham), _p(mom))
        return ham, mom

    def matter_sources(self, g: Geom, prim, out=None):
        """GRMHDEvolution::computeMatterSources (grmhd.cpp:1034-1103): (rho, Si, Sij, S)
        shaped (nz, ny, nx[, 3 | 6]) incl. ghosts; only interior cells are written
        (``out`` supplies the initial arrays, zeros by default)."""
        rho, Si, Sij, S = out if out is not None else matter_zeros(g)
        rho, Si, Sij, S = (np.array(a, dtype=np.float64, copy=True) for a in (rho, Si, Sij, S))
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        self.lib.orc_matter_sources(C.byref(_cg(g)), _p(prim), _p(rho), _p(Si), _p(Sij), _p(S))
        return rho, Si, Sij, S

    def psi4_modes(self, g: Geom, u, radii, n_theta: int, n_phi: int, l_max: int, counts: bool = False):
        """Psi4Extractor::extract on one block (postprocess.cpp:245-314): complex
        modes [len(radii), (l_max + 1)^2 - 4], l = 2..l_max, m = -l..l (and the
        sphere points inside the block per radius when ``counts``)."""
        nm = (l_max + 1) ** 2 - 4
        out = np.zeros((len(radii), nm, 2))
        r = np.ascontiguousarray(radii, dtype=np.float64)
        hi = np.ascontiguousarray(g.hi, dtype=np.float64)
        npts = (C.c_int * len(r))()
        self.lib.orc_psi4_modes(C.byref(_cg(g)), _p(hi), _p(np.ascontiguousarray(u, dtype=np.float64)), _p(r),
                                C.c_int(len(r)), C.c_int(n_theta), C.c_int(n_phi), C.c_int(l_max), _p(out), npts)
        modes = out[..., 0] + 1j * out[..., 1]
        return (modes, list(npts)) if counts else modes

    def find_horizon(self, g: Geom, u, center, max_iterations=200, tol=1e-10, ang_res=50, init_r=1.0):
        """findHorizon's flow and surface integrals (horizon_finder.cpp:310-449):
        (iterations or -1, h[ang_res, 2 ang_res], [area, M_irr, spin, C_eq, C_pol])."""
        h = np.full((ang_res, 2 * ang_res), float(init_r))
        res = np.zeros(5)
        self.lib.orc_find_horizon.restype = C.c_int
        it = self.lib.orc_find_horizon(C.byref(_cg(g)), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                       _p(np.ascontiguousarray(center, dtype=np.float64)), C.c_int(max_iterations),
                                       C.c_double(tol), C.c_int(ang_res), _p(h), _p(res))
        return it, h, res

    def horizon_expansion(self, g: Geom, u, p, n):
        self.lib.orc_horizon_expansion.restype = C.c_double
        return self.lib.orc_horizon_expansion(C.byref(_cg(g)), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                              *[C.c_double(x) for x in (*p, *n)])

    def constraint_sums(self, g: Geom, u):
        h2, m2, n = C.c_double(), C.c_double(), C.c_long()
        self.lib.orc_constraint_sums(C.byref(_cg(g)), _p(u), C.byref(h2), C.byref(m2),
                                     C.byref(n))
        return h2.value, m2.value, n.value

    def fill(self, g: Geom, u, kind: str):
        fn = {"zero_gradient": self.lib.orc_fill_zero_gradient,
              "sommerfeld": self.lib.orc_fill_sommerfeld,
              "periodic": self.lib.orc_fill_periodic,
              "floors": self.lib.orc_floors,
              "algebraic": self.lib.orc_algebraic}[kind]
        fn(C.byref(_cg(g)), _p(u))
        return u

    def rk3_steps(self, p: Params, g: Geom, u, dt: float, nsteps: int, bc: int = BC_SOMMERFELD,
                  matter=None):
        """nsteps RK3 steps; ``matter`` = (rho, Si, Sij, S) held fixed, or None (vacuum)."""
        u = np.array(u, dtype=np.float64, copy=True)
        stage = g.zeros()
        rhs = g.zeros()
        m = [None] * 4 if matter is None else [np.ascontiguousarray(a, dtype=np.float64) for a in matter]
        for _ in range(nsteps):
            self.lib.orc_rk3_step_matter(C.byref(_cp(p)), C.byref(_cg(g)), _p(u), _p(stage), _p(rhs),
                                         C.c_double(dt), C.c_int(bc), *[_p(a) for a in m])
        return u

    def init_flat(self, g: Geom):
        u = g.zeros()
        self.lib.orc_init_flat(C.byref(_cg(g)), _p(u))
        return u

    def init_gauge_wave(self, g: Geom, amplitude: float, wavelength: float):
        u = g.zeros()
        self.lib.orc_init_gauge_wave(C.byref(_cg(g)), _p(u), C.c_double(amplitude),
                                     C.c_double(wavelength))
        return u

    def init_brill_lindquist(self, g: Geom, masses, positions, r_floor: float = 0.0):
        u = g.zeros()
        m = np.ascontiguousarray(masses, dtype=np.float64)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self.lib.orc_init_brill_lindquist(C.byref(_cg(g)), _p(u), C.c_int(len(m)), _p(m),
                                          _p(pos), C.c_double(r_floor))
        return u

    def bl_conformal_factor(self, masses, positions, x, y, z, r_floor=0.0):
        m = np.ascontiguousarray(masses, dtype=np.float64)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self.lib.orc_bl_conformal_factor.restype = C.c_double
        return self.lib.orc_bl_conformal_factor(C.c_int(len(m)), _p(m), _p(pos), C.c_double(x),
                                                C.c_double(y), C.c_double(z),
                                                C.c_double(r_floor))

    def prolongate(self, gc: Geom, uc, gf: Geom, uf, ghosts_only: bool = False):
        uf = np.array(uf, dtype=np.float64, copy=True)
        self.lib.orc_prolongate(C.byref(_cg(gc)), _p(uc), C.byref(_cg(gf)), _p(uf),
                                C.c_int(int(ghosts_only)))
        return uf

    def restrict(self, gf: Geom, uf, gc: Geom, uc):
        uc = np.array(uc, dtype=np.float64, copy=True)
        self.lib.orc_restrict(C.byref(_cg(gf)), _p(uf), C.byref(_cg(gc)), _p(uc))
        return uc


def _host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return all(x in flags for x in ("avx512f", "avx512dq", "avx512bw", "avx512vl"))
    except OSError:
        return False


def reference_path(variant: str = "strict") -> str:
    """Path of a compiled reference library: 'strict' (IEEE, for pinning) or
    'fast' (reference Release flags, for timing; ISA level picked for this host)."""
    if variant == "fast":
        variant = "fast_v4" if _host_has_avx512() else "fast_v3"
    return os.path.join(HERE, "_ref", f"libgranite_ref_{variant}.so")


def reference_available(variant: str = "strict") -> bool:
    return os.path.exists(reference_path(variant))


class Reference:
    """The compiled reference sources behind ref_shim.cpp."""

    kind = "reference"

    def __init__(self, variant: str = "strict", threads: int = 0):
        self.path = reference_path(variant)
        self.lib = C.CDLL(self.path)
        if threads:
            self.lib.ref_set_threads(threads)
        self.lib.ref_bl_conformal_factor.restype = C.c_double

    @staticmethod
    def _g(g: Geom):
        n = (C.c_int * 3)(*g.n)
        lo = (C.c_double * 3)(*g.lo)
        hi = (C.c_double * 3)(*g.hi)
        return n, C.c_int(g.ng), lo, hi

    def max_threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def last_loop_seconds(self) -> float:
        """Wall seconds of the step loop alone of the last rk3_steps call (without
        the hierarchy set-up, block allocation and copies around it)."""
        self.lib.ref_last_loop_seconds.restype = C.c_double
        return float(self.lib.ref_last_loop_seconds())

    def rhs(self, p: Params, g: Geom, u, rho=None, Si=None, Sij=None, S=None):
        out = g.zeros()
        p6 = p.as6()
        self.lib.ref_rhs(_p(p6), *self._g(g), _p(u), _p(out), _p(rho), _p(Si), _p(Sij), _p(S))
        return out

    def dissipation(self, p: Params, g: Geom, u, rhs):
        rhs = np.array(rhs, dtype=np.float64, copy=True)
        p6 = p.as6()
        self.lib.ref_dissipation(_p(p6), *self._g(g), _p(u), _p(rhs))
        return rhs

    def constraints(self, g: Geom, u):
        ham = np.zeros(g.shape[1:], dtype=np.float64)
        mom = np.zeros(g.shape[1:] + (3,), dtype=np.float64)
        self.lib.ref_constraints(*self._g(g), _p(u), _p(ham), _p(mom))
        return ham, mom

    def matter_sources(self, g: Geom, prim, out=None):
        """The compiled GRMHDEvolution::computeMatterSources (grmhd.cpp:1034-1103)."""
        rho, Si, Sij, S = out if out is not None else matter_zeros(g)
        rho, Si, Sij, S = (np.array(a, dtype=np.float64, copy=True) for a in (rho, Si, Sij, S))
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        self.lib.ref_matter_sources(*self._g(g), _p(prim), _p(rho), _p(Si), _p(Sij), _p(S))
        return rho, Si, Sij, S

    def psi4_modes(self, g: Geom, u, radii, n_theta: int, n_phi: int, l_max: int):
        """The compiled Psi4Extractor::extract + getMode (postprocess.cpp:245-326)."""
        nm = (l_max + 1) ** 2 - 4
        out = np.zeros((len(radii), nm, 2))
        r = np.ascontiguousarray(radii, dtype=np.float64)
        self.lib.ref_psi4_modes(*self._g(g), _p(np.ascontiguousarray(u, dtype=np.float64)), _p(r), C.c_int(len(r)),
                                C.c_int(n_theta), C.c_int(n_phi), C.c_int(l_max), _p(out))
        return out[..., 0] + 1j * out[..., 1]

    def psi4_series(self, g: Geom, states, times, radii, n_theta: int, n_phi: int, l_max: int, spectrum_mode):
        """The compiled Psi4Extractor over a time series (postprocess.cpp:245-475):
        extract(states[t], times[t]) for every t, then a dict with the recorded
        series per (radius index, mode index) as [(time, complex)], strain[r, q],
        energy[r], extrap[q] and the energy spectrum of spectrum_mode = (l, m, radius
        index) as [(f, dE/df)]."""
        nt, nr = len(times), len(radii)
        nm = (l_max + 1) ** 2 - 4
        u = np.ascontiguousarray(np.stack([np.asarray(s, dtype=np.float64) for s in states]))
        count = np.zeros((nr, nm), dtype=np.int32)
        series = np.zeros((nr, nm, nt, 3))
        strain = np.zeros((nr, nm, 2))
        energy = np.zeros(nr)
        extrap = np.zeros((nm, 2))
        spec = np.zeros((500, 2))
        sl, sm, sr = spectrum_mode
        ns = self.lib.ref_psi4_series(*self._g(g), _p(u), _p(np.ascontiguousarray(times, dtype=np.float64)),
                                      C.c_int(nt), _p(np.ascontiguousarray(radii, dtype=np.float64)), C.c_int(nr),
                                      C.c_int(n_theta), C.c_int(n_phi), C.c_int(l_max),
                                      count.ctypes.data_as(C.POINTER(C.c_int)), _p(series), _p(strain), _p(energy),
                                      _p(extrap), C.c_int(sl), C.c_int(sm), C.c_int(sr), _p(spec), C.c_int(500))
        rec = {(r, q): [(series[r, q, t, 0], complex(series[r, q, t, 1], series[r, q, t, 2]))
                        for t in range(count[r, q])] for r in range(nr) for q in range(nm)}
        return dict(series=rec, strain=strain[..., 0] + 1j * strain[..., 1], energy=energy,
                    extrap=extrap[:, 0] + 1j * extrap[:, 1], spectrum=[tuple(x) for x in spec[:min(ns, 500)]])

    def find_horizon(self, g: Geom, u, center, max_iterations=200, tol=1e-10, ang_res=50, init_r=1.0):
        """The compiled ApparentHorizonFinder::findHorizon: (found, [area, M_irr, spin,
        C_eq, C_pol], surface points [ang_res * 2 ang_res, 3])."""
        res = np.zeros(5)
        surf = np.zeros((ang_res * 2 * ang_res, 3))
        found = self.lib.ref_find_horizon(*self._g(g), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                          _p(np.ascontiguousarray(center, dtype=np.float64)), C.c_int(max_iterations),
                                          C.c_double(tol), C.c_int(ang_res), C.c_double(init_r), _p(res), _p(surf))
        return bool(found), res, surf

    def find_all_horizons(self, g: Geom, u, max_iterations=200, tol=1e-10, ang_res=50, init_r=1.0, cap=16):
        """The compiled findAllHorizons: rows (cx, cy, cz, area, M_irr, spin)."""
        out = np.zeros((cap, 6))
        n = self.lib.ref_find_all_horizons(*self._g(g), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                           C.c_int(max_iterations), C.c_double(tol), C.c_int(ang_res),
                                           C.c_double(init_r), _p(out), C.c_int(cap))
        return out[:min(n, cap)]

    def find_common_horizon(self, g: Geom, u, centroids, masses, circ_eq, max_iterations=200, tol=1e-10,
                            ang_res=50, init_r=1.0):
        """The compiled findCommonHorizon over horizons given by centroid, irreducible
        mass and equatorial circumference: (found, [area, M_irr, spin, C_eq, C_pol],
        surface points, (centroid, id))."""
        nh = len(masses)
        hz = np.ascontiguousarray(np.reshape(centroids, (nh, 3)), dtype=np.float64)
        mc = np.ascontiguousarray(np.stack([np.asarray(masses, float), np.asarray(circ_eq, float)], axis=1))
        res = np.zeros(5)
        surf = np.zeros((ang_res * 2 * ang_res, 3))
        cid = np.zeros(4)
        found = self.lib.ref_find_common_horizon(*self._g(g), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                                 _p(hz), _p(mc), C.c_int(nh), C.c_int(max_iterations),
                                                 C.c_double(tol), C.c_int(ang_res), C.c_double(init_r), _p(res),
                                                 _p(surf), _p(cid))
        return bool(found), res, surf, (tuple(cid[:3]), int(cid[3]))

    def compute_spin(self, c_eq: float, c_pol: float) -> float:
        """The compiled ApparentHorizonFinder::computeSpin of a horizon with these circumferences."""
        self.lib.ref_compute_spin.restype = C.c_double
        return self.lib.ref_compute_spin(C.c_double(c_eq), C.c_double(c_pol))

    def init_flat(self, g: Geom):
        u = g.zeros()
        self.lib.ref_init_flat(*self._g(g), _p(u))
        return u

    def init_gauge_wave(self, g: Geom, amplitude: float, wavelength: float):
        u = g.zeros()
        self.lib.ref_init_gauge_wave(*self._g(g), _p(u), C.c_double(amplitude),
                                     C.c_double(wavelength))
        return u

    def init_brill_lindquist(self, g: Geom, masses, positions):
        u = g.zeros()
        m = np.ascontiguousarray(masses, dtype=np.float64)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self.lib.ref_init_brill_lindquist(*self._g(g), _p(u), C.c_int(len(m)), _p(m), _p(pos))
        return u

    def tag_count(self, g: Geom, u, var: int, threshold: float) -> int:
        """gradientChiTagger / gradientLapseTagger (amr.cpp:653-731) over the interior."""
        self.lib.ref_tag_count.restype = C.c_longlong
        return int(self.lib.ref_tag_count(*self._g(g), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                          C.c_int(var), C.c_double(threshold)))

    def composite_tag_count(self, g: Geom, u, taggers) -> int:
        """compositeTagger (amr.cpp:723-731) of [(var, threshold), ...] over the interior."""
        self.lib.ref_composite_tag_count.restype = C.c_longlong
        v = (C.c_int * len(taggers))(*[int(t[0]) for t in taggers])
        th = np.ascontiguousarray([float(t[1]) for t in taggers], dtype=np.float64)
        return int(self.lib.ref_composite_tag_count(*self._g(g), _p(np.ascontiguousarray(u, dtype=np.float64)),
                                                    C.c_int(len(taggers)), v, _p(th)))

    def bl_conformal_factor(self, masses, positions, x, y, z):
        m = np.ascontiguousarray(masses, dtype=np.float64)
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        return self.lib.ref_bl_conformal_factor(C.c_int(len(m)), _p(m), _p(pos), C.c_double(x),
                                                C.c_double(y), C.c_double(z))

    def fill_level0(self, g: Geom, u):
        u = np.array(u, dtype=np.float64, copy=True)
        self.lib.ref_fill_level0(*self._g(g), _p(u))
        return u

    def prolongate(self, gc: Geom, uc, clevel, gf: Geom, uf, flevel):
        uf = np.array(uf, dtype=np.float64, copy=True)
        cn, _, clo, chi = self._g(gc)
        fn, ng, flo, fhi = self._g(gf)
        self.lib.ref_prolongate(cn, clo, chi, C.c_int(clevel), _p(uc), fn, flo, fhi,
                                C.c_int(flevel), _p(uf), ng)
        return uf

    def restrict(self, gf: Geom, uf, flevel, gc: Geom, uc, clevel):
        uc = np.array(uc, dtype=np.float64, copy=True)
        cn, _, clo, chi = self._g(gc)
        fn, ng, flo, fhi = self._g(gf)
        self.lib.ref_restrict(fn, flo, fhi, C.c_int(flevel), _p(uf), cn, clo, chi,
                              C.c_int(clevel), _p(uc), ng)
        return uc

    def rk3_steps(self, p: Params, g: Geom, u, dt: float, nsteps: int, bc: int = BC_SOMMERFELD,
                  matter=None):
        """nsteps RK3 steps; ``matter`` = (rho, Si, Sij, S) held fixed, or None (vacuum)."""
        u = np.array(u, dtype=np.float64, copy=True)
        p6 = p.as6()
        if matter is None:
            self.lib.ref_rk3_steps(_p(p6), *self._g(g), _p(u), C.c_double(dt), C.c_int(nsteps),
                                   C.c_int(bc))
        else:
            m = [np.ascontiguousarray(a, dtype=np.float64) for a in matter]
            self.lib.ref_rk3_steps_matter(_p(p6), *self._g(g), _p(u), C.c_double(dt), C.c_int(nsteps),
                                          C.c_int(bc), *[_p(a) for a in m])
        return u


# ---------------------------------------------------------------------------
# Seeded workloads shared by tests and bench (same draws on every backend)
# ---------------------------------------------------------------------------

NPRIM = 11  # PrimitiveVar::NUM_VARS (types.hpp:149-162)


def matter_zeros(g: Geom):
    cells = g.shape[1:]
    return (np.zeros(cells), np.zeros(cells + (3,)), np.zeros(cells + (6,)), np.zeros(cells))


def seeded_primitives(g: Geom, seed: int, superluminal: float = 0.0):
    """Primitives (PrimitiveVar order) of a magnetised fluid on every cell, from
    the integer hash of hash_noise (identical on every host): rho in [1e-3, 1]
    with ~1 % exact zeros, |v_a| < 0.5 (a fraction ``superluminal`` of cells with
    v^x in [0.9, 1.2], where the W clamp of computeMatterSources acts), p in
    [1e-4, 0.1], B in [-0.2, 0.2], eps in [0.01, 1], T and Ye arbitrary."""
    cells = g.shape[1:]

    def h(s):
        return hash_noise(cells, seed * 16 + s) + 0.5  # [0, 1)

    p = np.empty((NPRIM,) + cells)
    p[0] = 1e-3 + (1.0 - 1e-3) * h(1)
    p[0][h(2) < 0.01] = 0.0
    for a in range(3):
        p[1 + a] = h(3 + a) - 0.5
    fast = h(6) < superluminal
    p[1][fast] = 0.9 + 0.3 * h(7)[fast]
    p[4] = 1e-4 + 0.1 * h(8)
    for a in range(3):
        p[5 + a] = 0.4 * (h(9 + a) - 0.5)
    p[8] = 0.01 + h(12)
    p[9] = 10.0 * h(13)
    p[10] = 0.05 + 0.45 * h(14)
    return p


def add_noise(u, amplitude: float, seed: int):
    """Uniform(-a, a) noise on every field and cell, numpy PCG64 stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return u + rng.uniform(-amplitude, amplitude, size=u.shape)


def random_state(g: Geom, seed: int, amp: float = 0.05):
    """A smooth, strongly non-flat but well-conditioned state for RHS parity."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nz, ny, nx = g.shape[1:]
    X = np.array([g.x(0, i) for i in range(nx)])[None, None, :]
    Y = np.array([g.x(1, j) for j in range(ny)])[None, :, None]
    Z = np.array([g.x(2, k) for k in range(nz)])[:, None, None]
    L = [g.hi[d] - g.lo[d] for d in range(3)]
    u = np.zeros(g.shape)
    base = np.zeros(NV)
    base[[0, 1, 4, 6, 18]] = 1.0  # chi, gxx, gyy, gzz, alpha
    for v in range(NV):
        a = rng.uniform(-1, 1, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        u[v] = base[v] + amp * (a[0] * np.sin(2 * np.pi * X / L[0] * 1.3 + ph[0])
                                * np.cos(2 * np.pi * Y / L[1] * 0.7 + ph[1])
                                + a[1] * np.sin(2 * np.pi * Z / L[2] * 1.1 + ph[2])
                                + a[2] * np.cos(2 * np.pi * (X / L[0] + Y / L[1] - Z / L[2])))
    return u


def hash_noise(shape, seed: int):
    """Deterministic uniform(-0.5, 0.5) values from an integer hash (splitmix64),
    exactly representable (k / 2^24 - 1/2), identical on every host."""
    n = int(np.prod(shape))
    with np.errstate(over="ignore"):
        x = np.arange(n, dtype=np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    k = (x >> np.uint64(40)).astype(np.float64)  # 24 bits
    return (k / 16777216.0 - 0.5).reshape(shape)


def seeded_state(g: Geom, seed: int, amp: float = 0.05, noise: float = 1e-3):
    """Smooth polynomial background + hash noise, built from IEEE + and * only so
    the same inputs are reproduced bit for bit on any machine."""
    nz, ny, nx = g.shape[1:]
    X = np.array([g.x(0, i) for i in range(nx)])[None, None, :]
    Y = np.array([g.x(1, j) for j in range(ny)])[None, :, None]
    Z = np.array([g.x(2, k) for k in range(nz)])[:, None, None]
    L = max(g.hi[d] - g.lo[d] for d in range(3))
    X, Y, Z = X / L, Y / L, Z / L
    co = hash_noise((NV, 10), seed + 1000)
    u = np.zeros(g.shape)
    base = np.zeros(NV)
    base[[0, 1, 4, 6, 18]] = 1.0
    for v in range(NV):
        c = co[v]
        poly = (c[0] * X + c[1] * Y + c[2] * Z + c[3] * X * Y + c[4] * Y * Z + c[5] * X * Z
                + c[6] * X * X + c[7] * Y * Y + c[8] * Z * Z + c[9] * X * Y * Z)
        u[v] = base[v] + amp * poly
    u += noise * hash_noise(g.shape, seed)
    return u


def seeded_matter(g: Geom, seed: int, amp: float = 1e-2):
    N = g.cells
    rho = amp * (hash_noise((N,), seed + 1) + 0.5)
    Si = amp * hash_noise((N * 3,), seed + 2)
    Sij = amp * hash_noise((N * 6,), seed + 3)
    S = amp * (hash_noise((N,), seed + 4) + 0.5)
    return rho, Si, Sij, S
