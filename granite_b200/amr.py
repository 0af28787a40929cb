"""AMRHierarchy with the reference's interface (amr.hpp:48-140) over the device.

The block geometry is planned on the host with the reference's steps
(``regrid.RegridPlanner``: initialize, tracking spheres, regrid boxes); the
state lives on the GPU in an ``Evolver`` and every ``subcycle(0)`` is one
Berger-Oliger coarse step there (``granite_ccz4_hierarchy_step``, or
``granite_ccz4_hierarchy_step_regrid`` when ``regrid_interval > 0``), with the
reference's SSP-RK3 step as the evolution function. ``getLevel`` /
``getAllBlocks`` hand out host GridBlocks that hold the current state: after a
step they are brought back from the device on first access, and blocks handed
out are sent to the device again before the next step, so a caller may read
and write them between steps as with the reference.

What differs from the reference, and why:

* ``subcycle`` runs from level 0 only and takes ``evolve_func=None`` (the
  device's fused RK3 step, ``TimeIntegrator::sspRK3Step`` for the spacetime);
  a host evolution function cannot run on the device path.
* Every level must keep dt(0) / 2^L (``setLevelDt`` on level 0 does this);
  refinement ratio 2 and 4 ghost cells, as the device transfers require.
* Taggers are ``(var, threshold)`` pairs: ``gradientChiTagger`` and
  ``gradientLapseTagger`` below build them, ``compositeTagger`` lists them.
* ``fillGhostZones``, ``prolongate`` and ``restrict_data`` are steps inside
  ``subcycle`` on the device and are not offered on host blocks;
  ``redistributeBlocks`` is a stub in the reference (one rank) and here.
"""
from __future__ import annotations

from dataclasses import dataclass

from . import (AMR_REFERENCE, PRECISION_FP64, CCZ4Params, Evolver, GraniteError, GridBlock,
               NUM_SPACETIME_VARS)
from .regrid import CHI, LAPSE, RegridPlanner


@dataclass
class AMRParams:
    """amr.hpp:20-28 (buffer_width, the thresholds and subcycling are unused by the
    reference's hierarchy code, as here)."""
    max_levels: int = 15
    refinement_ratio: int = 2
    regrid_interval: int = 4
    buffer_width: int = 4
    refine_threshold: float = 0.1
    derefine_threshold: float = 0.05
    subcycling: bool = True


@dataclass
class SimulationParams:
    """The SimulationParams fields the hierarchy reads (types.hpp:181-186)."""
    ncells: tuple = (64, 64, 64)
    domain_lo: tuple = (-100.0, -100.0, -100.0)
    domain_hi: tuple = (100.0, 100.0, 100.0)
    ghost_cells: int = 4


def gradientChiTagger(threshold: float):
    """amr.cpp:653-674: |grad chi| / (|chi| + 1e-30) > threshold."""
    return (CHI, float(threshold))


def gradientLapseTagger(threshold: float):
    """amr.cpp:699-720: |grad alpha| / (|alpha| + 1e-30) > threshold."""
    return (LAPSE, float(threshold))


def compositeTagger(taggers):
    """amr.cpp:723-731: a cell is tagged when any of the taggers tags it."""
    return list(taggers)


class AMRHierarchy:
    """amr.hpp:48-140. ``ccz4_params``, ``precision`` and ``amr_mode`` choose the
    device step (defaults: the reference's parameters, FP64, the reference's
    transfers)."""

    def __init__(self, params: AMRParams, sim_params: SimulationParams, ccz4_params: CCZ4Params | None = None,
                 precision: int = PRECISION_FP64, amr_mode: int = AMR_REFERENCE, evolver_factory=None):
        if params.refinement_ratio != 2:
            raise GraniteError(-6, "the device transfers are ratio-2 (prolongation, restriction)")
        if sim_params.ghost_cells != 4:
            raise GraniteError(-1, "ghost_cells must be 4: the upwind stencil reaches i+-4 (ccz4.cpp:109-152)")
        self._params = params
        self._sim = sim_params
        self._ccz4 = ccz4_params or CCZ4Params()
        self._precision = precision
        self._amr_mode = amr_mode
        self._make_evolver = evolver_factory or (lambda: Evolver(self._ccz4))
        self._planner = RegridPlanner(tuple(sim_params.ncells), tuple(sim_params.domain_lo),
                                      tuple(sim_params.domain_hi), max_levels=params.max_levels,
                                      refinement_ratio=params.refinement_ratio)
        self._blocks: list[GridBlock] = []
        self._dt: list[float] = []
        self._ev = None
        self._host_stale = False  # the device holds newer state than the host arrays
        self._host_dirty = True   # host arrays may have been written since the last upload

    # -- tracking spheres, amr.cpp:628-636 ------------------------------------
    def addTrackingSphere(self, center, radius: float, min_level: int):
        self._planner.add_tracking_sphere(tuple(center), float(radius), int(min_level))

    def updateTrackingSpheres(self, new_centers):
        self._planner.update_tracking_spheres([tuple(c) for c in new_centers])

    # -- layout ----------------------------------------------------------------
    def initialize(self, tagger=None):
        """amr.cpp:34-78: the level-0 block over the domain, then the levels the
        tracking spheres require (where the spheres require a level, the tagger
        is not consulted, so it plays no part here). Blocks start zero."""
        del tagger
        self._close_evolver()
        self._blocks = [GridBlock(b.id, b.level, b.ncells, b.lo, b.hi, self._sim.ghost_cells, NUM_SPACETIME_VARS)
                        for b in self._planner.initial_layout()]
        self._dt = [0.0] * self.numLevels()
        self._host_stale = False
        self._host_dirty = True

    def getLevel(self, level: int) -> list:
        self._to_host()
        self._host_dirty = True
        return [b for b in self._blocks if b.level == level]

    def getAllBlocks(self) -> list:
        self._to_host()
        self._host_dirty = True
        return list(self._blocks)

    def numLevels(self) -> int:
        return 1 + max(b.level for b in self._blocks) if self._blocks else 0

    def numBlocks(self) -> int:
        return len(self._blocks)

    def params(self) -> AMRParams:
        return self._params

    def effectiveResolution(self, point=None) -> float:
        """amr.cpp:642-647: the coarsest level's dx (the point is unused there too)."""
        del point
        lv0 = [b for b in self._blocks if b.level == 0]
        return lv0[0].dx(0) if lv0 else 1.0

    def redistributeBlocks(self):
        """amr.cpp:638-640: a stub for one rank."""

    # -- time stepping ---------------------------------------------------------
    def setLevelDt(self, level: int, dt: float):
        """amr.cpp:389-398: dt on ``level``, divided by the ratio for each finer level."""
        if level < 0 or level >= len(self._dt):
            return
        self._dt[level] = float(dt)
        for lv in range(level + 1, len(self._dt)):
            dt /= float(self._params.refinement_ratio)
            self._dt[lv] = dt

    def levelDt(self, level: int) -> float:
        return self._dt[level]

    def currentTime(self, level: int) -> float:
        """Level::current_time (amr.hpp:108-113) after the steps taken so far."""
        return self._ev.level_time(level) if self._ev is not None else 0.0

    def subcycle(self, level: int = 0, evolve_func=None, tagger=None):
        """amr.cpp:303-350 from level 0: one coarse step of dt(0), every level L
        taking 2^L steps of dt(0) / 2^L with the device's RK3 step, and the
        regrid of ``params.regrid_interval`` with ``tagger`` at the reference's
        points. Returns the blocks the regrids added."""
        if level != 0:
            raise GraniteError(-6, "subcycle runs the whole hierarchy from level 0")
        if evolve_func is not None:
            raise GraniteError(-6, "the device evolves with its own SSP-RK3 step: pass evolve_func=None")
        if not self._blocks:
            raise GraniteError(-1, "initialize the hierarchy first")
        dt0 = self._dt[0]
        for lv, dt in enumerate(self._dt):
            if dt != dt0 / float(self._params.refinement_ratio) ** lv:
                raise GraniteError(-6, "every level must keep dt(0) / 2^L: set it with setLevelDt(0, dt)")
        ev = self._device()
        nlev = self.numLevels()
        if self._params.regrid_interval > 0:
            added = ev.hierarchy_step_regrid(dt0, self._planner, self._params.regrid_interval, tagger,
                                             self._precision, self._amr_mode)
        else:
            ev.hierarchy_step(dt0, self._precision, self._amr_mode)
            added = []
        self._blocks = list(ev.blocks)
        for lv in range(nlev, self.numLevels()):  # amr.cpp:137-143: a new level's dt
            self._dt.append(self._dt[lv - 1] / float(self._params.refinement_ratio))
        self._host_stale = True
        return added

    def regrid(self, level: int, tagger=None):
        """amr.cpp:80-301 outside a step: new blocks around the tracking spheres (or
        when the tagger fires), prolongated on the device. Returns the blocks added."""
        ev = self._device()
        nlev = self.numLevels()
        added = ev.regrid(self._planner, level, tagger)
        self._blocks = list(ev.blocks)
        for lv in range(nlev, self.numLevels()):
            self._dt.append(self._dt[lv - 1] / float(self._params.refinement_ratio))
        if added:
            self._host_stale = True
        return added

    def evolver(self) -> Evolver:
        """The device hierarchy (constraint norms, diagnostics, checkpoints)."""
        return self._device()

    def close(self):
        self._close_evolver()

    # -- host <-> device -------------------------------------------------------
    def _device(self):
        if self._ev is None:
            ev = self._make_evolver()
            for b in self._blocks:
                ev.add_block(b)
            ev.commit()
            self._ev = ev
            self._host_dirty = True
        if self._host_dirty:
            self._to_host()
            self._ev.upload()
            self._host_dirty = False
        return self._ev

    def _to_host(self):
        if self._host_stale and self._ev is not None:
            self._ev.download()
        self._host_stale = False

    def _close_evolver(self):
        if self._ev is not None:
            self._ev.close()
        self._ev = None
