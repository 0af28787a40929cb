"""Hierarchy drivers for the oracle -- TEST INFRASTRUCTURE ONLY.

* ``RefHierarchy``: the compiled reference's own AMRHierarchy (tracking
  spheres, subcycle; amr.cpp:34-350) behind oracle/ref_shim.cpp, with the
  restated spacetime RK3 step as evolve_func. Regridding inside the step is
  off; ``regrid`` runs AMRHierarchy::regrid on demand.
* ``tag_count``: the gradient taggers (amr.cpp:653-731) restated in numpy.
* In-step regrid (amr.cpp:343-349) for both drivers: ``HierarchyOracle`` keeps
  each level's current_time and calls ``regrid_hook(self, level)`` at the
  reference's regrid points (``add_blocks`` prolongates the new blocks);
  ``RefHierarchy(..., regrid_interval=k)`` runs the reference's own.
* ``HierarchyOracle``: a restatement of the same Berger-Oliger step over the
  oracle's C pieces, in two modes:
    - "reference": amr.cpp literally (prolongation from every coarse block into
      all cells of each fine block, last one wins, amr.cpp:313-318,438;
      zero-gradient on faces no coarse block covers, amr.cpp:420-480; 1/r
      falloff on every block after every stage, main.cpp:351-521; restriction
      fine block by fine block, amr.cpp:566-626);
    - "ghosts": ghost cells filled block-locally (zero-gradient around a step,
      1/r falloff after a stage), then from the coarse block whose interior
      holds the cell centre (prolongation formula of amr.cpp:484-564), then
      from the same-level block whose interior holds it (copy); coarse cells
      whose eight children lie in one fine interior are restricted.
  The "ghosts" source of every ghost cell is decided here from cell-centre
  coordinates, independently of the box lists the library builds.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import Geom, Oracle, Params, Reference, _cg, _cp, _p

NG = 4


class RefHierarchy:
    def __init__(self, ref: Reference, n, lo, hi, spheres, max_levels=15, regrid_interval=0):
        self.ref = ref
        lib = ref.lib
        lib.ref_hier_create.restype = C.c_void_p
        lib.ref_hier_num_blocks.argtypes = [C.c_void_p]
        lib.ref_hier_block_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                            C.POINTER(C.c_int), C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
        lib.ref_hier_get.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        lib.ref_hier_set.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        lib.ref_hier_step.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_int]
        lib.ref_hier_destroy.argtypes = [C.c_void_p]
        cen = np.ascontiguousarray([s[0] for s in spheres], dtype=np.float64).reshape(-1, 3)
        rad = np.ascontiguousarray([s[1] for s in spheres], dtype=np.float64)
        mlv = (C.c_int * len(spheres))(*[int(s[2]) for s in spheres])
        lib.ref_hier_update_spheres.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        lib.ref_hier_regrid.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
        lib.ref_hier_set_tagger.argtypes = [C.c_void_p, C.c_int, C.c_double]
        self.h = lib.ref_hier_create((C.c_int * 3)(*n), (C.c_double * 3)(*lo), (C.c_double * 3)(*hi),
                                     C.c_int(max_levels), C.c_int(len(spheres)), _p(cen), _p(rad), mlv,
                                     C.c_int(regrid_interval))
        self._read_layout()

    def _read_layout(self):
        lib = self.ref.lib
        self.geoms, self.levels = [], []
        for i in range(lib.ref_hier_num_blocks(self.h)):
            lv = C.c_int()
            nn = (C.c_int * 3)()
            blo = (C.c_double * 3)()
            bhi = (C.c_double * 3)()
            lib.ref_hier_block_info(self.h, i, C.byref(lv), nn, blo, bhi)
            self.geoms.append(Geom(tuple(nn), tuple(blo), tuple(bhi)))
            self.levels.append(lv.value)

    def update_spheres(self, centers):
        """AMRHierarchy::updateTrackingSpheres (amr.cpp:632-636)."""
        c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        self.ref.lib.ref_hier_update_spheres(self.h, C.c_int(len(c)), _p(c))

    def regrid(self, level: int, var: int = -1, threshold: float = 0.0):
        """AMRHierarchy::regrid (amr.cpp:80-301) with the chi (var 0) or lapse (var 18)
        gradient tagger, or one that never tags; the block list is re-read (level
        order, then creation order)."""
        self.ref.lib.ref_hier_regrid(self.h, C.c_int(level), C.c_int(var), C.c_double(threshold))
        self._read_layout()

    def get(self, i):
        u = self.geoms[i].zeros()
        self.ref.lib.ref_hier_get(self.h, i, _p(u))
        return u

    def set(self, i, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.ref.lib.ref_hier_set(self.h, i, _p(u))

    def set_tagger(self, var: int, threshold: float):
        """The tagger subcycle's regrids use (var 0 chi, 18 lapse, other: none)."""
        self.ref.lib.ref_hier_set_tagger(self.h, C.c_int(var), C.c_double(threshold))

    def step(self, p: Params, dt: float, nsteps: int = 1):
        p6 = p.as6()
        self.ref.lib.ref_hier_step(self.h, _p(p6), C.c_double(dt), C.c_int(nsteps))
        self._read_layout()

    def __del__(self):
        try:
            self.ref.lib.ref_hier_destroy(self.h)
        except Exception:
            pass


def tag_count(g: Geom, u, var: int, threshold: float) -> int:
    """Interior cells of one block tagged by gradientChiTagger (var 0) or
    gradientLapseTagger (var 18), amr.cpp:653-731: |grad f| / (|f| + 1e-30) >
    threshold with grad f from centred differences (f[+1] - f[-1]) / (2 dx),
    squares summed x, y, z from 0.0 (separately rounded, no contraction)."""
    a = np.asarray(u, dtype=np.float64)[var]
    nx, ny, nz = g.n
    s = slice(NG, NG + nz), slice(NG, NG + ny), slice(NG, NG + nx)

    def shifted(axis, o):
        sl = list(s)
        sl[2 - axis] = slice(NG + o, NG + o + g.n[axis])
        return a[tuple(sl)]

    grad2 = np.zeros((nz, ny, nx))
    for d in range(3):
        df = (shifted(d, 1) - shifted(d, -1)) / (2.0 * g.dx[d])
        grad2 = grad2 + df * df
    return int(np.count_nonzero(np.sqrt(grad2) / (np.abs(a[s]) + 1e-30) > threshold))


def _centres(g: Geom):
    nz, ny, nx = g.shape[1:]
    X = np.array([g.x(0, i) for i in range(nx)])
    Y = np.array([g.x(1, j) for j in range(ny)])
    Z = np.array([g.x(2, k) for k in range(nz)])
    return X, Y, Z


def _ghost_mask(g: Geom):
    m = np.ones(g.shape[1:], dtype=bool)
    m[g.interior()[1:]] = False
    return m


class HierarchyOracle:
    """Blocks (geometry, level, state) advanced by the restated hierarchy step."""

    def __init__(self, geoms, levels, oracle: Oracle | None = None):
        self.o = oracle or Oracle()
        self.geoms = list(geoms)
        self.levels = list(levels)
        self.nlev = max(self.levels) + 1
        self.by_level = [[i for i, l in enumerate(self.levels) if l == L] for L in range(self.nlev)]
        self.u = [g.zeros() for g in self.geoms]
        self.s1 = [g.zeros() for g in self.geoms]
        self.s2 = [g.zeros() for g in self.geoms]
        self.rhs = [g.zeros() for g in self.geoms]
        self._ghost_plan = None
        # in-step regrid (amr.cpp:343-349): Level::current_time per level and the
        # hook called as hook(self, level) at the regrid points
        self.time = [0.0] * self.nlev
        self.regrid_interval = 0
        self.regrid_hook = None

    def add_blocks(self, geoms, levels):
        """New blocks after the existing ones, each prolongated in all its cells
        from every block of the coarser level in list order (the regrid's
        amr.cpp:291-293 with prolongate, amr.cpp:484-564); a new level starts
        at its parent's time (amr.cpp:137-143)."""
        lib = self.o.lib
        for g, L in zip(geoms, levels):
            assert 1 <= L <= self.nlev
            i = len(self.geoms)
            self.geoms.append(g)
            self.levels.append(L)
            if L == self.nlev:
                self.nlev += 1
                self.by_level.append([])
                self.time.append(self.time[L - 1])
            u = g.zeros()
            for c in self.by_level[L - 1]:
                lib.orc_prolongate(C.byref(_cg(self.geoms[c])), _p(self.u[c]), C.byref(_cg(g)), _p(u), C.c_int(0))
            self.by_level[L].append(i)
            self.u.append(u)
            self.s1.append(g.zeros())
            self.s2.append(g.zeros())
            self.rhs.append(g.zeros())
        self._ghost_plan = None

    # -- reference mode ----------------------------------------------------
    def _ref_fill(self, L, arrs):
        lib = self.o.lib
        for f in self.by_level[L]:
            gf = self.geoms[f]
            mask = 0x3F
            if L > 0:
                flo = [False] * 3
                fhi = [False] * 3
                for c in self.by_level[L - 1]:
                    gc = self.geoms[c]
                    for d in range(3):
                        if gc.x(d, NG) <= gf.x(d, NG) + 0.5 * gf.dx[d]:
                            flo[d] = True
                        if gc.x(d, NG + gc.n[d] - 1) >= gf.x(d, NG + gf.n[d] - 1) - 0.5 * gf.dx[d]:
                            fhi[d] = True
                    lib.orc_prolongate(C.byref(_cg(gc)), _p(self.u[c]), C.byref(_cg(gf)), _p(arrs[f]),
                                       C.c_int(0))
                mask = sum((0 if flo[d] else 1 << (2 * d)) | (0 if fhi[d] else 1 << (2 * d + 1))
                           for d in range(3))
            lib.orc_fill_zero_gradient_masked(C.byref(_cg(gf)), _p(arrs[f]), C.c_int(mask))

    # -- ghosts mode --------------------------------------------------------
    def _plan(self):
        """For every block: coarse-source masks and same-level copy index maps."""
        plan = []
        for b, g in enumerate(self.geoms):
            L = self.levels[b]
            X, Y, Z = _centres(g)
            ghost = _ghost_mask(g)
            pro = []
            if L > 0:
                for c in self.by_level[L - 1]:
                    gc = self.geoms[c]
                    inx = (X >= gc.lo[0]) & (X < gc.hi[0])
                    iny = (Y >= gc.lo[1]) & (Y < gc.hi[1])
                    inz = (Z >= gc.lo[2]) & (Z < gc.hi[2])
                    if not (inx.any() and iny.any() and inz.any()):
                        continue
                    m = ghost & inz[:, None, None] & iny[None, :, None] & inx[None, None, :]
                    if m.any():
                        pro.append((c, np.ascontiguousarray(m.astype(np.uint8))))
            cop = []
            for a in self.by_level[L]:
                if a == b:
                    continue
                ga = self.geoms[a]
                inx = (X >= ga.lo[0]) & (X < ga.hi[0])
                iny = (Y >= ga.lo[1]) & (Y < ga.hi[1])
                inz = (Z >= ga.lo[2]) & (Z < ga.hi[2])
                if not (inx.any() and iny.any() and inz.any()):
                    continue
                m = ghost & inz[:, None, None] & iny[None, :, None] & inx[None, None, :]
                if not m.any():
                    continue
                kk, jj, ii = np.nonzero(m)
                # matching cell of a: same centre coordinate
                sa = [np.rint((np.array([g.x(d, q) for q in idx]) - ga.lo[d]) / ga.dx[d] - 0.5).astype(int) + NG
                      for d, idx in ((0, ii), (1, jj), (2, kk))]
                cop.append((a, (kk, jj, ii), (sa[2], sa[1], sa[0])))
            plan.append((pro, cop))
        # restriction: coarse cells whose 2x2x2 children lie in one fine interior
        rest = []
        for L in range(self.nlev - 1):
            for c in self.by_level[L]:
                gc = self.geoms[c]
                for f in self.by_level[L + 1]:
                    gf = self.geoms[f]
                    sel = []
                    for d in range(3):
                        ci = np.arange(NG, NG + gc.n[d])
                        xc = gc.lo[d] + (ci - NG + 0.5) * gc.dx[d]
                        lo_child = xc - 0.5 * gf.dx[d]  # centre of the lower child
                        fi = np.rint((lo_child - gf.lo[d]) / gf.dx[d] - 0.5).astype(int)
                        ok = (fi >= 0) & (fi + 2 <= gf.n[d])
                        sel.append((ci[ok], fi[ok] + NG))
                    if all(len(s[0]) for s in sel):
                        rest.append((L, c, f, sel))
        self._ghost_plan = (plan, rest)

    def _ghost_fill(self, L, arrs, level_fill):
        lib = self.o.lib
        plan, _ = self._ghost_plan
        for b in self.by_level[L]:
            g = self.geoms[b]
            fill = lib.orc_fill_zero_gradient if level_fill else lib.orc_fill_sommerfeld
            fill(C.byref(_cg(g)), _p(arrs[b]))
            for c, m in plan[b][0]:
                lib.orc_prolongate_masked(C.byref(_cg(self.geoms[c])), _p(self.u[c]), C.byref(_cg(g)),
                                          _p(arrs[b]), m.ctypes.data_as(C.POINTER(C.c_ubyte)))
        for b in self.by_level[L]:
            for a, dst, src in plan[b][1]:
                arrs[b][:, dst[0], dst[1], dst[2]] = arrs[a][:, src[0], src[1], src[2]]

    def _ghost_restrict(self, L):
        _, rest = self._ghost_plan
        for (lv, c, f, sel) in rest:
            if lv != L:
                continue
            (cx, fx), (cy, fy), (cz, fz) = sel
            uf = self.u[f]
            s = np.zeros((22, len(cz), len(cy), len(cx)))
            for rk in range(2):
                for rj in range(2):
                    for ri in range(2):
                        s = s + uf[:, (fz + rk)[:, None, None], (fy + rj)[None, :, None],
                                   (fx + ri)[None, None, :]]
            self.u[c][:, cz[:, None, None], cy[None, :, None], cx[None, None, :]] = s / 8.0

    # -- the step --------------------------------------------------------------
    def _evolve(self, L, dt, p: Params, mode):
        lib = self.o.lib
        cp = _cp(p)
        a = [(1.0, 0.0, 1.0), (0.75, 0.25, 0.25), (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]
        for s in range(3):
            for b in self.by_level[L]:
                g = self.geoms[b]
                uin = self.u[b] if s == 0 else (self.s1[b] if s == 1 else self.s2[b])
                uout = self.s1[b] if s == 0 else (self.s2[b] if s == 1 else self.u[b])
                lib.orc_stage(C.byref(cp), C.byref(_cg(g)), _p(self.u[b]), _p(uin), _p(uout),
                              _p(self.rhs[b]), C.c_double(a[s][0]), C.c_double(a[s][1]),
                              C.c_double(a[s][2]), C.c_double(dt), C.c_int(1 if s == 2 else 0))
                if mode == "reference":
                    lib.orc_fill_sommerfeld(C.byref(_cg(g)), _p(uout))
            if mode == "ghosts" and s < 2:
                self._ghost_fill(L, self.s1 if s == 0 else self.s2, level_fill=False)

    def _subcycle(self, L, dt, p, mode):
        lib = self.o.lib
        if mode == "ghosts" and self._ghost_plan is None:
            self._plan()
        if mode == "reference":
            if L > 0:
                for f in self.by_level[L]:
                    for c in self.by_level[L - 1]:
                        lib.orc_prolongate(C.byref(_cg(self.geoms[c])), _p(self.u[c]),
                                           C.byref(_cg(self.geoms[f])), _p(self.u[f]), C.c_int(0))
            self._ref_fill(L, self.u)
        else:
            self._ghost_fill(L, self.u, level_fill=True)
        self._evolve(L, dt, p, mode)
        self.time[L] += dt
        if mode == "reference":
            self._ref_fill(L, self.u)
        else:
            self._ghost_fill(L, self.u, level_fill=True)
        if L + 1 < self.nlev:
            for _ in range(2):
                self._subcycle(L + 1, dt / 2.0, p, mode)
            if mode == "ghosts" and self._ghost_plan is None:
                self._plan()
            if mode == "reference":
                for f in self.by_level[L + 1]:
                    for c in self.by_level[L]:
                        lib.orc_restrict(C.byref(_cg(self.geoms[f])), _p(self.u[f]),
                                         C.byref(_cg(self.geoms[c])), _p(self.u[c]))
            else:
                self._ghost_restrict(L)
        if self.regrid_interval > 0 and self.regrid_hook is not None:
            q = self.time[L] / (dt + 1e-15)
            step_num = math.trunc(q)
            if abs(q - step_num) >= 0.5:  # std::round: halves away from zero
                step_num += 1 if q > 0 else -1
            if step_num % self.regrid_interval == 0:
                self.regrid_hook(self, L)

    def step(self, p: Params, dt_coarse: float, mode: str = "reference", nsteps: int = 1):
        if mode == "ghosts" and self._ghost_plan is None:
            self._plan()
        for _ in range(nsteps):
            self._subcycle(0, dt_coarse, p, mode)
