"""granite_b200 -- B200-native CCZ4 RHS + SSP-RK3 stage update for GRANITE blocks.

Python mirror of the reference operator interface
(include/granite/spacetime/ccz4.hpp:49-115 of GRANITE) over the C ABI in
include/granite_ccz4.h (libgranite_ccz4.so, CUDA sm_100a). There is no CPU
path: every operator runs the CUDA library and raises if it cannot.

    from granite_b200 import GridBlock, CCZ4Params, CCZ4Evolution
    grid = GridBlock(0, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    rhs = GridBlock(1, 0, (32, 32, 32), (-10, -10, -10), (10, 10, 10), 4, 22)
    set_flat_spacetime(grid)
    CCZ4Evolution(CCZ4Params(ko_sigma=0.0)).computeRHSVacuum(grid, rhs)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

NUM_SPACETIME_VARS = 22

GRANITE_OK = 0
PRECISION_FP64 = 0
PRECISION_MIXED = 1
BC_REFERENCE = 0
BC_PERIODIC = 1
AMR_REFERENCE = 0
AMR_GHOSTS = 1
KERNEL_STAGE, KERNEL_GHOST, KERNEL_TRANSFER, KERNEL_CONSTRAINTS = 0, 1, 2, 3
VARIANT_GLOBAL, VARIANT_SMEM, VARIANT_GLOBAL_R168, VARIANT_GLOBAL_R128, VARIANT_TMA = 0, 1, 2, 3, 4
VARIANT_NAMES = {"global": 0, "smem": 1, "global_r168": 2, "global_r128": 3, "tma": 4}
# configurations of the TMA stage kernel and the block-size classes they are tuned for
STAGE_CONFIGS = 18
STAGE_CLASS_EDGES = (16, 24, 32, 48, 64, 96)

_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "no sm_100 device", -4: "out of memory",
           -5: "non-finite state", -6: "unsupported", -7: "timeout"}


class GraniteError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class _Params(C.Structure):
    _fields_ = [("kappa1", C.c_double), ("kappa2", C.c_double), ("eta", C.c_double),
                ("ko_sigma", C.c_double), ("chi_blend_center", C.c_double),
                ("chi_blend_width", C.c_double), ("fd_order", C.c_int), ("device", C.c_int)]


class _HorizonParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("tolerance", C.c_double), ("angular_resolution", C.c_int),
                ("initial_guess_radius", C.c_double)]


class _Horizon(C.Structure):
    _fields_ = [("found", C.c_int), ("iterations", C.c_int), ("id", C.c_int), ("centroid", C.c_double * 3),
                ("area", C.c_double), ("irreducible_mass", C.c_double), ("spin", C.c_double),
                ("circumference_equatorial", C.c_double), ("circumference_polar", C.c_double)]


class _BlockDesc(C.Structure):
    _fields_ = [("ncells", C.c_int * 3), ("nghost", C.c_int), ("lo", C.c_double * 3),
                ("hi", C.c_double * 3), ("level", C.c_int), ("id", C.c_int)]


_LIB = None


# granite_regrid_fn: int (*)(void* user, int level, long long step_num)
_REGRID_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_longlong)


def library_path() -> str:
    return _build.LIB


def load_library(build_if_missing: bool = True) -> C.CDLL:
    """Load libgranite_ccz4.so (building it with nvcc if it is missing or stale)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if build_if_missing and not _build.up_to_date():
        _build.build()
    if not os.path.exists(_build.LIB):
        raise GraniteError(-6, f"{_build.LIB} is missing: build it with granite_b200/build.py")
    lib = C.CDLL(_build.LIB)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    lib.granite_ccz4_create.argtypes = [C.POINTER(_Params), C.POINTER(vp)]
    lib.granite_ccz4_destroy.argtypes = [vp]
    lib.granite_ccz4_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
    lib.granite_ccz4_sync.argtypes = [vp]
    lib.granite_ccz4_compute_rhs_host.argtypes = [vp, C.POINTER(_BlockDesc), dp, dp, dp, dp, dp, dp,
                                                  C.c_int]
    lib.granite_ccz4_apply_dissipation_host.argtypes = [vp, C.POINTER(_BlockDesc), dp, dp]
    lib.granite_ccz4_compute_constraints_host.argtypes = [vp, C.POINTER(_BlockDesc), dp, dp, dp]
    lib.granite_ccz4_compute_rhs_device.argtypes = [vp, C.POINTER(_BlockDesc), vp, vp, vp, vp, vp,
                                                    vp, C.c_int, vp]
    lib.granite_ccz4_add_block.argtypes = [vp, C.POINTER(_BlockDesc), C.POINTER(C.c_int)]
    lib.granite_ccz4_commit.argtypes = [vp]
    lib.granite_ccz4_num_blocks.argtypes = [vp]
    lib.granite_ccz4_arena_bytes.argtypes = [vp, C.POINTER(C.c_size_t)]
    lib.granite_ccz4_upload_block.argtypes = [vp, C.c_int, dp]
    lib.granite_ccz4_download_block.argtypes = [vp, C.c_int, dp]
    lib.granite_ccz4_rk3_step.argtypes = [vp, C.c_int, C.c_double, C.c_int, C.c_int]
    lib.granite_ccz4_hierarchy_step.argtypes = [vp, C.c_double, C.c_int, C.c_int]
    lib.granite_ccz4_constraint_norms.argtypes = [vp, C.c_int, dp, dp]
    lib.granite_ccz4_nonfinite_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.granite_ccz4_launch_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    lib.granite_ccz4_default_params.argtypes = [C.POINTER(_Params)]
    lib.granite_ccz4_default_params.restype = None
    lib.granite_ccz4_set_profiling.argtypes = [vp, C.c_int]
    lib.granite_ccz4_profile_reset.argtypes = [vp]
    lib.granite_ccz4_profile_get.argtypes = [vp, C.c_int, dp, C.POINTER(C.c_longlong)]
    lib.granite_ccz4_get_stream.argtypes = [vp, C.POINTER(vp)]
    lib.granite_ccz4_set_kernel_variant.argtypes = [vp, C.c_int]
    lib.granite_ccz4_set_batching.argtypes = [vp, C.c_int]
    lib.granite_ccz4_get_kernel_variant.argtypes = [vp, C.POINTER(C.c_int)]
    lib.granite_ccz4_set_fp64_chi_threshold.argtypes = [vp, C.c_double]
    lib.granite_ccz4_measure_fma_rate.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.granite_ccz4_get_fp64_chi_threshold.argtypes = [vp, C.POINTER(C.c_double)]
    lib.granite_ccz4_regrid_add.argtypes = [vp, C.POINTER(_BlockDesc), C.c_int]
    lib.granite_ccz4_upload_all.argtypes = [vp, C.POINTER(dp)]
    lib.granite_ccz4_download_all.argtypes = [vp, C.POINTER(dp)]
    lib.granite_ccz4_download_all_async.argtypes = [vp, C.POINTER(dp)]
    ip = C.POINTER(C.c_int)
    hp = C.POINTER(_HorizonParams)
    lib.granite_ccz4_default_horizon_params.argtypes = [hp]
    lib.granite_ccz4_default_horizon_params.restype = None
    lib.granite_ccz4_find_horizon.argtypes = [vp, C.c_int, hp, dp, C.POINTER(_Horizon), dp]
    lib.granite_ccz4_find_horizon_host.argtypes = [vp, C.POINTER(_BlockDesc), dp, hp, dp, C.POINTER(_Horizon), dp]
    lib.granite_ccz4_find_all_horizons.argtypes = [vp, C.c_int, hp, C.POINTER(_Horizon), C.c_int, ip]
    lib.granite_ccz4_psi4_modes.argtypes = [vp, C.c_int, dp, C.c_int, C.c_int, C.c_int, C.c_int, dp, ip]
    lib.granite_ccz4_psi4_modes_host.argtypes = [vp, C.POINTER(_BlockDesc), dp, dp, C.c_int, C.c_int, C.c_int,
                                                 C.c_int, dp, ip]
    lib.granite_ccz4_psi4_modes_device.argtypes = [vp, C.POINTER(_BlockDesc), vp, dp, C.c_int, C.c_int, C.c_int,
                                                   C.c_int, dp, ip]
    lib.granite_ccz4_checkpoint_write.argtypes = [vp, C.c_char_p, C.c_int, C.c_double]
    lib.granite_ccz4_checkpoint_read.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int), dp]
    lib.granite_ccz4_checkpoint_header.argtypes = [C.c_char_p, C.POINTER(C.c_int), dp, C.POINTER(C.c_int),
                                                   C.POINTER(_BlockDesc), C.c_int, C.POINTER(C.c_int)]
    lib.granite_ccz4_matter_sources_host.argtypes = [vp, C.POINTER(_BlockDesc), dp, dp, dp, dp, dp]
    lib.granite_ccz4_matter_sources_device.argtypes = [vp, C.POINTER(_BlockDesc), vp, vp, vp, vp, vp, vp]
    lib.granite_ccz4_enable_matter.argtypes = [vp, C.c_int]
    lib.granite_ccz4_upload_primitives.argtypes = [vp, C.c_int, dp]
    lib.granite_ccz4_set_primitives_device.argtypes = [vp, C.c_int, vp]
    lib.granite_ccz4_hierarchy_step_regrid.argtypes = [vp, C.c_double, C.c_int, C.c_int, C.c_int, _REGRID_FN, vp]
    lib.granite_ccz4_level_time.argtypes = [vp, C.c_int, dp]
    lib.granite_ccz4_tag_count.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_longlong)]
    lib.granite_ccz4_test_withhold_tile_load.argtypes = [vp, C.c_int]
    lib.granite_ccz4_set_ghost_push.argtypes = [vp, C.c_int]
    lib.granite_ccz4_set_pass_overlap.argtypes = [vp, C.c_int]
    ip_ = C.POINTER(C.c_int)
    lib.granite_ccz4_set_stage_config.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.granite_ccz4_get_stage_config.argtypes = [vp, C.c_int, C.c_int, ip_]
    lib.granite_ccz4_force_stage_config.argtypes = [vp, C.c_int]
    lib.granite_ccz4_stage_config_info.argtypes = [C.c_int, ip_, ip_, ip_, ip_]
    lib.granite_ccz4_stage_config_schedule.argtypes = [C.c_int, ip_, ip_, ip_, ip_]
    lib.granite_ccz4_block_stage_class.argtypes = [C.POINTER(_BlockDesc), ip_]
    lib.granite_ccz4_compare_states.argtypes = [vp, vp, dp, dp, C.POINTER(C.c_longlong)]
    _LIB = lib
    return lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---------------------------------------------------------------------------
# GridBlock (include/granite/core/grid.hpp:44-162)
# ---------------------------------------------------------------------------

def stage_config_info(cfg: int) -> dict:
    """Tile depth, ring slots, shared-memory options and schedule of a TMA configuration."""
    lib = load_library()
    v = [C.c_int() for _ in range(4)]
    rc = lib.granite_ccz4_stage_config_info(int(cfg), *[C.byref(x) for x in v])
    if rc != GRANITE_OK:
        raise GraniteError(rc, f"unknown stage configuration {cfg}")
    w = [C.c_int() for _ in range(4)]
    lib.granite_ccz4_stage_config_schedule(int(cfg), *[C.byref(x) for x in w])
    return {"tile": (16, 4, v[0].value), "ring_slots": v[1].value, "shared_input": bool(v[2].value),
            "shared_hessian": bool(v[3].value), "warp_specialized": bool(w[0].value), "ctas_per_sm": w[1].value,
            "items_per_barrier": w[2].value, "x_remainder_tiles": bool(w[3].value)}


def block_stage_class(ncells) -> int:
    """Block-size class (index into STAGE_CLASS_EDGES) of a block with these interior cells."""
    lib = load_library()
    d = block_desc(ncells, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    v = C.c_int()
    rc = lib.granite_ccz4_block_stage_class(C.byref(d), C.byref(v))
    if rc != GRANITE_OK:
        raise GraniteError(rc, "bad block size")
    return v.value


def measure_fma_rate(device: int = 0, precision: int = 0) -> float:
    """Sustained FMA rate of a device in TFLOP/s: FP64 (precision 0) or FP32 (1)."""
    lib = load_library()
    v = C.c_double()
    rc = lib.granite_ccz4_measure_fma_rate(int(device), int(precision), C.byref(v))
    if rc != 0:
        raise GraniteError(rc, "granite_ccz4_measure_fma_rate failed")
    return v.value


class GridBlock:
    """Field-major block storage with the reference GridBlock layout.

    ``array`` is a float64 numpy array of shape (num_vars, nz+2g, ny+2g, nx+2g);
    its flat buffer is exactly GridBlock::flatBuffer() (grid.hpp:109-116).
    """

    def __init__(self, id: int, level: int, ncells, lo, hi, nghost: int = 4,
                 num_vars: int = NUM_SPACETIME_VARS):
        self.id = int(id)
        self.level = int(level)
        self.ncells = tuple(int(n) for n in ncells)
        self.lo = tuple(float(x) for x in lo)
        self.hi = tuple(float(x) for x in hi)
        self.nghost = int(nghost)
        self.num_vars = int(num_vars)
        self.dx_ = tuple((self.hi[d] - self.lo[d]) / self.ncells[d] for d in range(3))  # grid.cpp:20-22
        g = 2 * self.nghost
        nx, ny, nz = self.ncells
        self.array = np.zeros((self.num_vars, nz + g, ny + g, nx + g), dtype=np.float64)

    # accessors mirroring the reference
    def getId(self):
        return self.id

    def getLevel(self):
        return self.level

    def getNumGhost(self):
        return self.nghost

    def getNumVars(self):
        return self.num_vars

    def totalCells(self, d):
        return self.ncells[d] + 2 * self.nghost

    def totalSize(self):
        return self.totalCells(0) * self.totalCells(1) * self.totalCells(2)

    def dx(self, d):
        return self.dx_[d]

    def x(self, d, idx):
        return self.lo[d] + (float(idx) - self.nghost + 0.5) * self.dx_[d]

    def istart(self, d=0):
        return self.nghost

    def iend(self, d):
        return self.nghost + self.ncells[d]

    def data(self, var, i, j, k):
        return self.array[var, k, j, i]

    def set(self, var, i, j, k, value):
        self.array[var, k, j, i] = value

    def flatBuffer(self):
        return self.array.reshape(-1)

    def rawData(self, var):
        """Field ``var``'s plane of the flat buffer (grid.hpp:125-129), a view."""
        return self.array[var].reshape(-1)

    def numCells(self):
        return self.ncells

    def lowerCorner(self):
        return self.lo

    def upperCorner(self):
        return self.hi

    def desc(self) -> _BlockDesc:
        d = _BlockDesc()
        for a in range(3):
            d.ncells[a] = self.ncells[a]
            d.lo[a] = self.lo[a]
            d.hi[a] = self.hi[a]
        d.nghost = self.nghost
        d.level = self.level
        d.id = self.id
        return d

    def interior(self):
        g = self.nghost
        nx, ny, nz = self.ncells
        return (slice(None), slice(g, g + nz), slice(g, g + ny), slice(g, g + nx))


def block_desc(ncells, lo, hi, level=0, id=0, nghost=4) -> _BlockDesc:
    return GridBlock(id, level, ncells, lo, hi, nghost, 1).desc()


# ---------------------------------------------------------------------------
# CCZ4Evolution (include/granite/spacetime/ccz4.hpp:49-115)
# ---------------------------------------------------------------------------

@dataclass
class CCZ4Params:
    """CCZ4Params, ccz4.hpp:25-34."""

    kappa1: float = 0.02
    kappa2: float = 0.0
    eta: float = 2.0
    ko_sigma: float = 0.1
    fd_order: int = 4
    use_moving_puncture: bool = True
    chi_blend_center: float = 0.05
    chi_blend_width: float = 0.02
    device: int = 0

    def _c(self) -> _Params:
        return _Params(self.kappa1, self.kappa2, self.eta, self.ko_sigma, self.chi_blend_center,
                       self.chi_blend_width, self.fd_order, self.device)


class _Context:
    def __init__(self, params: CCZ4Params):
        self.lib = load_library()
        self.h = C.c_void_p()
        self._p = params._c()
        rc = self.lib.granite_ccz4_create(C.byref(self._p), C.byref(self.h))
        if rc != GRANITE_OK:
            raise GraniteError(rc, "granite_ccz4_create failed (no usable sm_100 GPU?)")

    def check(self, rc: int):
        if rc != GRANITE_OK:
            buf = C.create_string_buffer(512)
            self.lib.granite_ccz4_last_error(self.h, buf, 512)
            raise GraniteError(rc, buf.value.decode())

    def close(self):
        if self.h:
            self.lib.granite_ccz4_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _f64(a):
    a = np.asarray(a)
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("expected a C-contiguous float64 array")
    return a


class CCZ4Evolution:
    """GPU CCZ4 operator with the reference's method names and semantics."""

    def __init__(self, params: CCZ4Params | None = None, precision: int = PRECISION_FP64,
                 variant: int | None = None):
        self.params_ = params or CCZ4Params()
        self.precision = precision
        self.ctx = _Context(self.params_)
        if variant is not None:
            self.ctx.check(self.ctx.lib.granite_ccz4_set_kernel_variant(self.ctx.h, variant))

    def params(self):
        return self.params_

    def computeRHS(self, grid: GridBlock, rhs: GridBlock, rho_matter, Si_matter, Sij_matter,
                   S_trace):
        """ccz4.hpp:69-74. Matter arrays: rho[N], Si[N,3], Sij[N,6], S[N] (N = totalSize)."""
        N = grid.totalSize()
        rho = _f64(np.ascontiguousarray(rho_matter, dtype=np.float64).reshape(N))
        Si = _f64(np.ascontiguousarray(Si_matter, dtype=np.float64).reshape(N * 3))
        Sij = _f64(np.ascontiguousarray(Sij_matter, dtype=np.float64).reshape(N * 6))
        S = _f64(np.ascontiguousarray(S_trace, dtype=np.float64).reshape(N))
        self.ctx.check(self.ctx.lib.granite_ccz4_compute_rhs_host(
            self.ctx.h, C.byref(grid.desc()), _dp(grid.array), _dp(rhs.array), _dp(rho), _dp(Si),
            _dp(Sij), _dp(S), self.precision))

    def computeRHSVacuum(self, grid: GridBlock, rhs: GridBlock):
        """ccz4.hpp:81."""
        self.ctx.check(self.ctx.lib.granite_ccz4_compute_rhs_host(
            self.ctx.h, C.byref(grid.desc()), _dp(grid.array), _dp(rhs.array), None, None, None,
            None, self.precision))

    def applyDissipation(self, grid: GridBlock, rhs: GridBlock):
        """ccz4.hpp:99."""
        self.ctx.check(self.ctx.lib.granite_ccz4_apply_dissipation_host(
            self.ctx.h, C.byref(grid.desc()), _dp(grid.array), _dp(rhs.array)))

    def computeConstraints(self, grid: GridBlock):
        """ccz4.hpp:90-92. Returns (ham[N], mom[N,3]) over the whole block, ghosts zero."""
        N = grid.totalSize()
        ham = np.zeros(N, dtype=np.float64)
        mom = np.zeros((N, 3), dtype=np.float64)
        self.ctx.check(self.ctx.lib.granite_ccz4_compute_constraints_host(
            self.ctx.h, C.byref(grid.desc()), _dp(grid.array), _dp(ham), _dp(mom)))
        return ham, mom


NUM_PRIMITIVE_VARS = 11  # PrimitiveVar (types.hpp:149-162)


class MatterSources:
    """GRMHDEvolution::computeMatterSources (grmhd.hpp:333-338, grmhd.cpp:1034-1103)
    on the GPU: the ADM matter sources of the CCZ4 RHS from a primitive
    GridBlock (11 fields in PrimitiveVar order). Only this coupling of the
    GRMHD module is provided; its own evolution is not."""

    def __init__(self):
        self.ctx = _Context(CCZ4Params())

    def computeMatterSources(self, spacetime_grid: GridBlock, prim_grid: GridBlock, rho_src, Si, Sij,
                             S_trace):
        """Fills the interior cells of rho_src[N], Si[N,3], Sij[N,6], S_trace[N]
        (float64 C-contiguous arrays, N = totalSize; other cells keep their values)."""
        if prim_grid.num_vars != NUM_PRIMITIVE_VARS or prim_grid.ncells != spacetime_grid.ncells:
            raise ValueError("prim_grid: 11 primitive fields on the spacetime grid's cells")
        N = spacetime_grid.totalSize()
        arrs = [_f64(a) for a in (rho_src, Si, Sij, S_trace)]
        if [a.size for a in arrs] != [N, 3 * N, 6 * N, N]:
            raise ValueError("matter arrays must hold N, 3N, 6N and N values")
        self.ctx.check(self.ctx.lib.granite_ccz4_matter_sources_host(
            self.ctx.h, C.byref(spacetime_grid.desc()), _dp(prim_grid.array), *[_dp(a) for a in arrs]))

    def close(self):
        self.ctx.close()


# ---------------------------------------------------------------------------
# Resident hierarchy + RK3 driver (main.cpp TimeIntegrator, amr.cpp subcycle)
# ---------------------------------------------------------------------------

def checkpoint_header(path: str) -> dict:
    """Step, time, has_matter and the GridBlocks (geometry only, in order) of a
    checkpoint written by Evolver.checkpoint_write."""
    lib = load_library()
    n, step, mat = C.c_int(), C.c_int(), C.c_int()
    t = C.c_double()
    rc = lib.granite_ccz4_checkpoint_header(os.fsencode(path), C.byref(step), C.byref(t), C.byref(mat), None, 0,
                                            C.byref(n))
    if rc != GRANITE_OK:
        raise GraniteError(rc, f"cannot read checkpoint header of {path}")
    descs = (_BlockDesc * max(n.value, 1))()
    rc = lib.granite_ccz4_checkpoint_header(os.fsencode(path), None, None, None, descs, n.value, C.byref(n))
    if rc != GRANITE_OK:
        raise GraniteError(rc, f"cannot read checkpoint header of {path}")
    blocks = [GridBlock(d.id, d.level, tuple(d.ncells), tuple(d.lo), tuple(d.hi), d.nghost)
              for d in descs[:n.value]]
    return dict(step=step.value, time=t.value, has_matter=bool(mat.value), blocks=blocks)


class Evolver:
    """Device-resident blocks advanced by the fused RK3 step.

    add blocks, commit(), upload(), then rk3_step(level, dt) / hierarchy_step(dt).
    """

    def __init__(self, params: CCZ4Params | None = None, variant: int | None = None):
        self.params = params or CCZ4Params()
        self.ctx = _Context(self.params)
        self.blocks: list[GridBlock] = []
        self.committed = False
        if variant is not None:
            self.ctx.check(self.ctx.lib.granite_ccz4_set_kernel_variant(self.ctx.h, variant))

    def set_ghost_push(self, on: bool):
        """GRANITE_AMR_GHOSTS: stage kernels write the same-level ghost copies (default) or the fills copy them."""
        self.ctx.check(self.ctx.lib.granite_ccz4_set_ghost_push(self.ctx.h, int(bool(on))))

    def set_pass_overlap(self, on: bool):
        """Per-tile precision: the FP64 pass beside the FP32 pass on a second stream (default) or after it."""
        self.ctx.check(self.ctx.lib.granite_ccz4_set_pass_overlap(self.ctx.h, int(bool(on))))

    def set_batching(self, batched: bool):
        self.ctx.check(self.ctx.lib.granite_ccz4_set_batching(self.ctx.h, int(bool(batched))))

    def set_stage_config(self, precision: int, cls: int, cfg: int):
        """TMA configuration of block-size class cls (-1: every class) for steps
        in `precision`; cfg -1 restores the built-in default. Before commit."""
        self.ctx.check(self.ctx.lib.granite_ccz4_set_stage_config(self.ctx.h, int(precision), int(cls), int(cfg)))

    def stage_config(self, precision: int, cls: int) -> int:
        v = C.c_int()
        self.ctx.check(self.ctx.lib.granite_ccz4_get_stage_config(self.ctx.h, int(precision), int(cls), C.byref(v)))
        return v.value

    def force_stage_config(self, cfg: int):
        """One TMA configuration for every block and precision (-1: the per-class table). Before commit."""
        self.ctx.check(self.ctx.lib.granite_ccz4_force_stage_config(self.ctx.h, int(cfg)))

    def apply_stage_table(self, table: dict):
        """A tuner table {"fp64": [cfg per class], "mixed": [...]} (granite_b200.tuner)."""
        for name, prec in (("fp64", PRECISION_FP64), ("mixed", PRECISION_MIXED)):
            for cls, cfg in enumerate(table.get(name, [])):
                self.set_stage_config(prec, cls, int(cfg))

    def set_fp64_chi_threshold(self, chi_fp64: float):
        """MIXED steps: tiles with a point of chi below chi_fp64 run the FP64 algebra (0 = off)."""
        self.ctx.check(self.ctx.lib.granite_ccz4_set_fp64_chi_threshold(self.ctx.h, float(chi_fp64)))

    def fp64_chi_threshold(self) -> float:
        v = C.c_double()
        self.ctx.check(self.ctx.lib.granite_ccz4_get_fp64_chi_threshold(self.ctx.h, C.byref(v)))
        return v.value

    def variant(self) -> int:
        v = C.c_int()
        self.ctx.check(self.ctx.lib.granite_ccz4_get_kernel_variant(self.ctx.h, C.byref(v)))
        return v.value

    def enable_matter(self, on: bool = True):
        """Before commit: every block gets matter sources (zero = vacuum) that the
        RHS of every step reads (the non-vacuum applyRHS, main.cpp:296-302)."""
        self.ctx.check(self.ctx.lib.granite_ccz4_enable_matter(self.ctx.h, int(bool(on))))

    def upload_primitives(self, idx: int, prim):
        """Block idx's matter sources from its primitives (11 x totalSize float64,
        PrimitiveVar order) by computeMatterSources on the device; they hold
        until the next upload."""
        self.ctx.check(self.ctx.lib.granite_ccz4_upload_primitives(self.ctx.h, idx, _dp(_f64(prim))))

    def add_block(self, b: GridBlock) -> int:
        idx = C.c_int()
        self.ctx.check(self.ctx.lib.granite_ccz4_add_block(self.ctx.h, C.byref(b.desc()),
                                                           C.byref(idx)))
        self.blocks.append(b)
        return idx.value

    def commit(self):
        self.ctx.check(self.ctx.lib.granite_ccz4_commit(self.ctx.h))
        self.committed = True

    def arena_bytes(self) -> int:
        n = C.c_size_t()
        self.ctx.check(self.ctx.lib.granite_ccz4_arena_bytes(self.ctx.h, C.byref(n)))
        return n.value

    def upload(self, idx: int | None = None, array=None):
        """Block idx (all blocks when None) from its host array or ``array`` (for
        all blocks: a list of arrays, one per block, in block order)."""
        if idx is None:
            arrs = [b.array for b in self.blocks] if array is None else [_f64(a) for a in array]
            ptrs = (C.POINTER(C.c_double) * len(arrs))(*[_dp(a) for a in arrs])
            self.ctx.check(self.ctx.lib.granite_ccz4_upload_all(self.ctx.h, ptrs))
            self._keep = arrs  # the copies are stream-ordered: keep the buffers alive
            return
        a = self.blocks[idx].array if array is None else _f64(array)
        self.ctx.check(self.ctx.lib.granite_ccz4_upload_block(self.ctx.h, idx, _dp(a)))

    def download(self, idx: int | None = None, out=None, wait: bool = True):
        """Block idx (all blocks when None, one synchronisation) into its host array or ``out``.
        For all blocks, ``wait=False`` queues the copies on the context's stream and
        returns at once (granite_ccz4_download_all_async): the arrays hold the state
        after the next sync()."""
        if idx is None:
            arrs = [b.array for b in self.blocks] if out is None else [_f64(a) for a in out]
            ptrs = (C.POINTER(C.c_double) * len(arrs))(*[_dp(a) for a in arrs])
            fn = self.ctx.lib.granite_ccz4_download_all if wait else self.ctx.lib.granite_ccz4_download_all_async
            self.ctx.check(fn(self.ctx.h, ptrs))
            if not wait:
                self._keep_out = arrs
            return
        assert wait, "single-block downloads wait"
        a = self.blocks[idx].array if out is None else _f64(out)
        self.ctx.check(self.ctx.lib.granite_ccz4_download_block(self.ctx.h, idx, _dp(a)))

    def regrid_add(self, blocks):
        """Append GridBlocks to the committed hierarchy; the device fills every cell of
        each (ghosts included) by prolongation from the coarser level's last block
        (granite_ccz4_regrid_add). Existing blocks keep their state and indices."""
        blocks = list(blocks)
        if not blocks:
            return
        descs = (_BlockDesc * len(blocks))(*[b.desc() for b in blocks])
        self.ctx.check(self.ctx.lib.granite_ccz4_regrid_add(self.ctx.h, descs, len(blocks)))
        self.blocks.extend(blocks)

    def tag_count(self, level: int, var: int, threshold: float) -> int:
        """Interior cells of ``level`` that gradientChiTagger (var 0) or
        gradientLapseTagger (var 18) tags (amr.cpp:653-731), counted on the device."""
        n = C.c_longlong()
        self.ctx.check(self.ctx.lib.granite_ccz4_tag_count(self.ctx.h, level, var, float(threshold),
                                                           C.byref(n)))
        return n.value

    def regrid(self, planner, level: int, tagger=None):
        """AMRHierarchy::regrid(level, tagger) (amr.cpp:80-301) on the device state.

        ``planner`` is a ``regrid.RegridPlanner``; ``tagger`` is None (never tags),
        (var, threshold) for the chi / lapse gradient tagger, or a list of those
        (compositeTagger), consulted only when no tracking sphere requires
        level + 1, as in the reference (``regrid.tagger_fires``). Returns the
        GridBlocks added (their host arrays stay zero until ``download``).
        """
        from .regrid import tagger_fires
        if not any(b.level == level for b in self.blocks):
            return []
        if not planner.spheres_require(level + 1):
            if not tagger_fires(tagger, lambda var, threshold: self.tag_count(level, var, threshold)):
                return []
        new = [GridBlock(bx.id, bx.level, bx.ncells, bx.lo, bx.hi)
               for bx in planner.plan(level, self.blocks)]
        self.regrid_add(new)
        return new

    def rk3_step(self, level: int, dt: float, precision: int = PRECISION_FP64,
                 bc: int = BC_REFERENCE):
        self.ctx.check(self.ctx.lib.granite_ccz4_rk3_step(self.ctx.h, level, dt, precision, bc))

    def hierarchy_step(self, dt_coarse: float, precision: int = PRECISION_FP64,
                       amr_mode: int = AMR_REFERENCE):
        self.ctx.check(self.ctx.lib.granite_ccz4_hierarchy_step(self.ctx.h, dt_coarse, precision,
                                                                amr_mode))

    def hierarchy_step_regrid(self, dt_coarse: float, planner, regrid_interval: int, tagger=None,
                              precision: int = PRECISION_FP64, amr_mode: int = AMR_REFERENCE):
        """One coarse step of AMRHierarchy::subcycle with its in-step regrid
        (amr.cpp:303-350): at every level step whose step number is a multiple of
        ``regrid_interval``, ``regrid(planner, level, tagger)`` runs before the
        step goes on, as in the reference. Returns the GridBlocks added."""
        added, errors = [], []

        def on_regrid(_user, level, _step_num):
            try:
                added.extend(self.regrid(planner, level, tagger))
                return 0
            except Exception as e:  # reported after the step returns
                errors.append(e)
                return -1

        fn = _REGRID_FN(on_regrid)
        rc = self.ctx.lib.granite_ccz4_hierarchy_step_regrid(self.ctx.h, dt_coarse, precision, amr_mode,
                                                             int(regrid_interval), fn, None)
        if errors:
            raise errors[0]
        self.ctx.check(rc)
        return added

    def checkpoint_write(self, path: str, step: int = 0, time: float = 0.0):
        """The resident state (every block's state, level times, matter sources) to
        ``path``, with the data model of HDF5Writer::writeCheckpoint (hdf5_io.cpp:166-233)."""
        self.ctx.check(self.ctx.lib.granite_ccz4_checkpoint_write(self.ctx.h, os.fsencode(path), int(step),
                                                                  float(time)))

    def checkpoint_read(self, path: str):
        """Restore a checkpoint of this hierarchy (same blocks in the same order);
        returns (step, time)."""
        step, t = C.c_int(), C.c_double()
        self.ctx.check(self.ctx.lib.granite_ccz4_checkpoint_read(self.ctx.h, os.fsencode(path), C.byref(step),
                                                                 C.byref(t)))
        return step.value, t.value

    @classmethod
    def from_checkpoint(cls, path: str, params: CCZ4Params | None = None, variant: int | None = None):
        """A committed Evolver holding the checkpoint's blocks and state; returns
        (evolver, step, time). The blocks' host arrays stay zero until download()."""
        hdr = checkpoint_header(path)
        ev = cls(params, variant)
        if hdr["has_matter"]:
            ev.enable_matter()
        for b in hdr["blocks"]:
            ev.add_block(b)
        ev.commit()
        step, t = ev.checkpoint_read(path)
        return ev, step, t

    def level_time(self, level: int) -> float:
        """Level::current_time of the reference hierarchy (amr.hpp:108-113)."""
        t = C.c_double()
        self.ctx.check(self.ctx.lib.granite_ccz4_level_time(self.ctx.h, level, C.byref(t)))
        return t.value

    def sync(self):
        self.ctx.check(self.ctx.lib.granite_ccz4_sync(self.ctx.h))

    def compare_states(self, other: "Evolver"):
        """(max |a - b|, max |a|) per field over the interior cells of all blocks
        (numpy arrays of 22), and the non-finite counts (a, b); a = this
        context's state, b = other's (same block geometry, same device)."""
        dev = np.zeros(22)
        mag = np.zeros(22)
        nf = (C.c_longlong * 2)()
        self.ctx.check(self.ctx.lib.granite_ccz4_compare_states(self.ctx.h, other.ctx.h, _dp(dev), _dp(mag), nf))
        return dev, mag, (nf[0], nf[1])

    def test_withhold_tile_load(self, item: int):
        """Test switch: the next rk3_step's first stage leaves ring item `item` of
        the first persistent CTA unissued, so its bounded wait runs out and the
        next sync() raises GraniteError (GRANITE_ERR_CUDA)."""
        self.ctx.check(self.ctx.lib.granite_ccz4_test_withhold_tile_load(self.ctx.h, int(item)))

    def constraint_norms(self, level: int = -1):
        h = C.c_double()
        m = C.c_double()
        self.ctx.check(self.ctx.lib.granite_ccz4_constraint_norms(self.ctx.h, level, C.byref(h),
                                                                  C.byref(m)))
        return h.value, m.value

    def nonfinite_count(self) -> int:
        n = C.c_longlong()
        self.ctx.check(self.ctx.lib.granite_ccz4_nonfinite_count(self.ctx.h, C.byref(n)))
        return n.value

    def launch_count(self) -> int:
        n = C.c_longlong()
        self.ctx.check(self.ctx.lib.granite_ccz4_launch_count(self.ctx.h, C.byref(n)))
        return n.value

    def set_profiling(self, on: bool):
        self.ctx.check(self.ctx.lib.granite_ccz4_set_profiling(self.ctx.h, int(bool(on))))

    def profile_reset(self):
        self.ctx.check(self.ctx.lib.granite_ccz4_profile_reset(self.ctx.h))

    def profile(self, kernel_class: int):
        """(total device ms, launches) of a kernel class since the last reset."""
        ms = C.c_double()
        n = C.c_longlong()
        self.ctx.check(self.ctx.lib.granite_ccz4_profile_get(self.ctx.h, kernel_class,
                                                             C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def stream_handle(self) -> int:
        s = C.c_void_p()
        self.ctx.check(self.ctx.lib.granite_ccz4_get_stream(self.ctx.h, C.byref(s)))
        return s.value or 0

    def close(self):
        self.ctx.close()


from .initial_data import (  # noqa: E402
    brill_lindquist, gauge_wave, set_flat_spacetime, set_gauge_wave_data)
from .hierarchy import (  # noqa: E402,F401
    Hierarchy, block_states, make_binary_hierarchy, make_hierarchy, make_triple_hierarchy)
