// ccz4_kernels.h -- host-side launchers of the CCZ4 device kernels.
#pragma once

#include <cuda_runtime.h>

#include "ccz4_common.cuh"

namespace granite_b200 {

enum { EPI_STORE = 0, EPI_RK = 1 };

// Kernel variants of the fused stage: 0 = stencils from global memory
// (32x4x1 tiles), 1 = fields staged through shared memory with cp.async
// (16x4x2 tiles); 2, 3 = variant 0 with the registers capped at 168 / 128 per
// thread (3 / 4 CTAs per SM); 4 = persistent CTAs that stream every field of
// a 16x4x4 tile and its halo into a ring of shared-memory slots with TMA
// (cp.async.bulk.tensor) and mbarriers. The constraint and KO kernels always
// use variant-0 tiles.
enum {
    VARIANT_GLOBAL = 0, VARIANT_SMEM = 1, VARIANT_GLOBAL_R168 = 2, VARIANT_GLOBAL_R128 = 3, VARIANT_TMA = 4,
    NUM_VARIANTS = 5
};

// Tile shape of a stage-kernel variant (points per CTA along x, y, z); cfg
// selects the TMA configuration.
int stage_tile_dims(int variant, int cfg, int* tx, int* ty, int* tz);

// Configurations of the TMA variant (the autotuner's candidates): tiles of
// 16 x 4 x tz points (tz * 64 threads per CTA; tz = 2 asks for two resident
// CTAs per SM), a ring of nbuf field boxes; tin: the stage input's centre values
// are kept in shared memory for the RK epilogue and the epilogue's u^n and the
// next tile's pointwise cells are prefetched into L2; hs: the Hessian-field
// loop's 36 values live in shared memory instead of local memory.
// ws: the mixed RK kernels are warp-specialized (stencil warps feed algebra
// warps through shared memory; ccz4_stage_ws.cuh), the FP64 ones those of
// configuration 4. Configuration 0 is the only one with the store (drop-in
// RHS) epilogue; the defaults per precision and block-size class are in
// ccz4_capi.cu (DEFAULT_CLASS_CFG).
struct TmaCfg {
    int tz, nbuf, tin, hs, ws;
    int minb;  // resident CTAs per SM the register allocation is sized for (__launch_bounds__)
    int bar;   // ring items per CTA barrier (1 or 2; the barrier frees that many slots)
    // x-remainder tiles: a block whose x extent leaves 8 cells after its
    // 16-wide tiles covers them with 8 x 4 x 2tz tiles (Tile::w = -8, every
    // thread on a point) instead of 16-wide tiles half outside the block;
    // rem = 1 loads them with the 24 x 12 x (2tz + 8) box shape (ring slots
    // sized for it), rem = 2 as two boxes of the configuration's own shape (one
    // per half along z, two ring items; needs bar = 2)
    int rem;
    int pf;  // L2 prefetches of u^n and the next tile's pointwise cells without tin (tin implies them)
};
constexpr int NUM_TMA_CFGS = 18;
constexpr TmaCfg TMA_CFGS[NUM_TMA_CFGS] = {
    {4, 3, 0, 0, 0, 1, 1, 0, 0}, {4, 3, 1, 1, 0, 1, 1, 0, 0}, {2, 3, 1, 1, 0, 2, 1, 0, 0},
    {2, 2, 1, 1, 0, 2, 1, 0, 0}, {2, 3, 1, 0, 0, 2, 1, 0, 0}, {2, 3, 0, 0, 1, 2, 1, 0, 0},
    {2, 3, 0, 0, 0, 3, 1, 0, 0}, {2, 2, 1, 0, 0, 3, 1, 0, 0}, {2, 3, 1, 0, 0, 2, 2, 0, 0},
    {2, 4, 0, 0, 0, 2, 2, 0, 0}, {4, 4, 0, 0, 0, 1, 2, 0, 0}, {2, 3, 1, 0, 0, 2, 1, 1, 0},
    {2, 3, 0, 0, 0, 2, 1, 1, 0}, {2, 2, 1, 0, 0, 2, 1, 1, 0}, {2, 3, 0, 0, 0, 2, 1, 1, 1},
    {4, 4, 0, 0, 0, 1, 2, 1, 0}, {4, 4, 0, 0, 0, 1, 2, 2, 0}, {2, 4, 0, 0, 0, 2, 2, 2, 0}};
// Points of an x-remainder tile along x.
constexpr int TMA_REM_X = 8;
// The box (cells incl. the 4-cell halo) one tensor-map load brings in per
// field: 24 x 12 x (tz + 8). Tensor maps exist per box shape: shape 0 (tz =
// 4), shape 1 (tz = 2) and shape 2 (tz = 8, the remainder tiles of tz = 4
// configurations; a block less than 8 cells deep has none, and its tz = 4
// remainder columns keep 16-wide tiles).
constexpr int TMA_BOX_X = 16 + 8, TMA_BOX_Y = 4 + 8;
constexpr int TMA_SHAPES = 3;
constexpr int TMA_SHAPE_TZ[TMA_SHAPES] = {4, 2, 8};
constexpr int tma_shape_for_tz(int tz) { return tz == 4 ? 0 : (tz == 2 ? 1 : (tz == 8 ? 2 : -1)); }
constexpr int tma_shape_of(int cfg) { return tma_shape_for_tz(TMA_CFGS[cfg].tz); }
// box shape of a configuration's x-remainder tiles (-1: none)
constexpr int tma_rem_shape_of(int cfg) {
    return TMA_CFGS[cfg].rem == 1 ? tma_shape_for_tz(2 * TMA_CFGS[cfg].tz)
                                  : (TMA_CFGS[cfg].rem == 2 ? tma_shape_of(cfg) : -1);
}
// Per-tile precision launches of the TMA kernel keep each CTA's selected tiles
// in shared memory: at most TMA_SEL_CAP per CTA, i.e. ntiles <= grid x TMA_SEL_CAP.
constexpr int TMA_SEL_CAP = 1024;
// Grid of the FP64 pass of the per-tile precision, in resident grids (on the
// bench hierarchy 1: 76 us per level-stage, 4: 63 us, 8: 55 us, 16: 61 us, the
// scans of the CTAs without a selected tile outweighing the spread).
constexpr int TMA_FP64_SPREAD = 8;
// The resident grid of a TMA configuration's per-tile precision passes on the
// current device, the smaller of the two (0 before configure_stage_kernels).
int tma_grid(int cfg);
// Tensor map of one 22-field block buffer (dims x, y, z, field; cells incl.
// ghosts) with the box of tile depth tz. Returns false when the buffer cannot
// be described (odd x extent, misaligned base, box larger than the block);
// such blocks use the global-load kernel.
bool encode_block_tmap(void* map128, const double* base, const DevBlock& d, int tz);

// Per-device kernel attributes (shared-memory opt-in); call with the device current.
cudaError_t configure_stage_kernels();

// Precision modes of the stage kernels: FP64 algebra with the reference-order
// FP64 stencils, FP32 algebra (mixed), or FP64 algebra with pair-difference
// FP64 stencils (PM_FP64F, RK epilogue only: the FP64 pass of the per-tile
// precision, where parity is with the FP64 path to rounding, not bit for bit).
enum { PM_FP64 = 0, PM_MIXED = 1, PM_FP64F = 2 };

// Fused RHS (+KO) over a tile work-list in precision mode `precision` (PM_*);
// with args.tile_prec set, only the tiles flagged args.want_prec. cfg: the TMA
// configuration (ignored by the other variants); args.tmaps must hold the
// tensor maps of that configuration's box shape.
cudaError_t launch_stage(int variant, int cfg, int precision, int epi, const DevBlock* blocks,
                         const Tile* tiles, int ntiles, const StageArgs& args, cudaStream_t stream);

// Per-tile precision flags of tiles [first, first + ntiles): flag[ti] = 1 when a
// point of the tile has chi < chi_fp64 in slot `sel` (FP64 algebra), else 0.
cudaError_t launch_classify(int variant, int cfg, const DevBlock* blocks, const Tile* tiles, int first, int ntiles,
                            int sel, double chi_fp64, unsigned char* flag, cudaStream_t stream);

// KO dissipation only: rhs += KO(u) at interior points of one block.
cudaError_t launch_dissipation(const DevBlock* block, int in_sel, double* rhs, int ntiles,
                               const Tile* tiles, cudaStream_t stream);

// Ghost-cell work items: one per (block, ghost cell); built on the host.
struct GhostItem {
    int block;
    int cell;  // linear cell index within the block (incl. ghosts)
};

enum GhostMode {
    GHOST_ZERO_GRADIENT = 0,    // all faces (amr.cpp:447-480)
    GHOST_SOMMERFELD = 1,       // 1/r falloff (main.cpp:351-463)
    GHOST_PERIODIC = 2,         // periodic wrap (gauge-wave workload)
    GHOST_ZERO_GRADIENT_MASKED = 3  // only the faces flagged in a per-block 6-bit mask
};

// Fill every listed ghost cell of buffer slot `sel` for all 22 fields.
// facemask (per block; bit 2d = low face of axis d, bit 2d+1 = high face) is
// read only by GHOST_ZERO_GRADIENT_MASKED.
cudaError_t launch_ghost_fill(int mode, const DevBlock* blocks, const GhostItem* items, int nitems,
                              int sel, const unsigned char* facemask, cudaStream_t stream);

// A box of cells moved between two blocks. Coordinates are block-local cell
// indices including ghosts.
//   copy:     dst <- src, same level, cell for cell (s0 = source origin)
//   prolong:  dst (fine) <- trilinear interpolation of src (coarse), amr.cpp:484-564
//   restrict: dst (coarse) <- mean of the 2x2x2 fine cells of src at s0 + 2 (a, b, c),
//             amr.cpp:566-626
struct XferBox {
    int dst, src;
    int d0[3];
    int s0[3];
    int n[3];
};
// One CTA of a transfer launch: XFER_CHUNK consecutive cells of a box.
struct BoxChunk {
    int box;
    int start;
};
constexpr int XFER_CHUNK = 256;
enum XferKind { XFER_COPY = 0, XFER_PROLONG = 1, XFER_RESTRICT = 2 };

// Transfers of slot src_sel of the source blocks into slot dst_sel of the destinations.
cudaError_t launch_xfer(int kind, const DevBlock* blocks, const XferBox* boxes, const BoxChunk* chunks,
                        int nchunks, int dst_sel, int src_sel, cudaStream_t stream);

// One ghost cell of a level and where its value comes from (GRANITE_AMR_GHOSTS):
//   src_block >= 0, src_cell >= 0: copy of that cell of a same-level block
//   src_block >= 0, src_cell <  0: prolongation from that coarse block
//   src_block <  0               : the block's own fill (zero-gradient or 1/r falloff)
struct GhostSrc {
    int dst_block, dst_cell, src_block, src_cell;
};

// Every listed ghost cell written once: copies and local fills read slot
// `sel`, prolongations read slot 0 of the coarse block. local_mode:
// GHOST_ZERO_GRADIENT or GHOST_SOMMERFELD.
cudaError_t launch_ghost_sources(const DevBlock* blocks, const GhostSrc* items, long long nitems, int sel,
                                 int local_mode, cudaStream_t stream);

// Constraint monitor (ccz4.cpp:941-1159) over a tile work-list. Writes ham /
// mom (single-block drop-in; may be null) and per-CTA partial sums of H^2 and
// |M|^2 to partials[2 * tile] (may be null).
cudaError_t launch_constraints(const DevBlock* blocks, const Tile* tiles, int ntiles, int sel,
                               double* ham, double* mom, double* partials, cudaStream_t stream);

// Regrid tagger (amr.cpp:653-731) over the interior cells of slot 0 of the
// listed tiles (32x4x1 monitor shape): adds the number of tagged cells to *count.
cudaError_t launch_tag_count(const DevBlock* blocks, const Tile* tiles, int ntiles, int var, double threshold,
                             unsigned long long* count, cudaStream_t stream);

// Matter sources of the CCZ4 RHS from GRMHD primitives (grmhd.cpp:1034-1103)
// at the interior cells of one block. prim: NPRIM fields of B.stride cells.
// Outputs: rho[c], S[c], Si[c * si_cell + a * si_comp], Sij[c * sij_cell + q * sij_comp]
// (the reference's AoS arrays: si_cell 3, si_comp 1, sij_cell 6, sij_comp 1).
constexpr int NPRIM = 11;
struct MatterOut {
    double* rho;
    double* Si;
    double* Sij;
    double* S;
    long long si_cell, si_comp, sij_cell, sij_comp;
};
cudaError_t launch_matter_sources(const DevBlock& B, const double* prim, const MatterOut& out, cudaStream_t stream);

// Psi4Extractor::extract (postprocess.cpp:245-314) on one block: modes[r * nm + q]
// (q over l = 2..l_max, m = -l..l; nm = (l_max + 1)^2 - 4) at the nr radii (device
// array); psi4_scratch holds nr * n_theta * n_phi values; inside_count[r] gets the
// number of sphere points of radius r inside the block. hi: the block's upper corner.
cudaError_t launch_psi4_modes(const DevBlock& B, const double* u, const double hi[3], const double* radii, int nr,
                              int n_theta, int n_phi, int l_max, double2* psi4_scratch, double2* modes,
                              unsigned int* inside_count, cudaStream_t stream);

// Apparent-horizon flow (horizon_finder.cpp:310-449) on one block. tab holds
// sin(theta_i), cos(theta_i) (nth each), sin(phi_j), cos(phi_j) (nph each),
// evaluated by the host's libm.
struct HorizonArgs {
    double center[3];
    double flow_step, rmin;  // 0.05 dx and 1e-6 dx
    double dth, dph;         // pi / nth, 2 pi / nph
    int nth, nph;
};
// iters flow iterations of every surface point from the radii h (updated in
// place): radii after iteration k at hist[k * N + p], max |Theta| of iteration k
// as the bits of a non-negative double in itmax[k] (zeroed here).
cudaError_t launch_horizon_flow(const DevBlock& B, const double* u, const HorizonArgs& a, const double* tab,
                                double* h, int iters, double* hist, unsigned long long* itmax, cudaStream_t stream);
// terms[3 p ..] = area term, J_z term, 1 (0 where chi < 1e-12) of surface point p.
cudaError_t launch_horizon_surface(const DevBlock& B, const double* u, const HorizonArgs& a, const double* tab,
                                   const double* h, double* terms, cudaStream_t stream);
// findAllHorizons' candidate cells (lapse minima below 0.5), up to cap cell indices
// in arbitrary order; *count = all found.
cudaError_t launch_lapse_minima(const DevBlock& B, const double* u, long long* out, unsigned int* count,
                                unsigned int cap, cudaStream_t stream);

// Per field v: out[v] = max |a - b|, out[22 + v] = max |a| over the interior
// cells of slot 0 of blocks a[i], b[i] (i < nblocks, identical geometry), as the
// bits of non-negative doubles; out[44], out[45] = non-finite values in a, in b.
cudaError_t launch_compare_states(const DevBlock* a, const DevBlock* b, int nblocks, unsigned long long* out,
                                  cudaStream_t stream);

// Deterministic fixed-order sum of n partial pairs into out[2].
cudaError_t launch_sum_partials(const double* partials, int n, double* out, cudaStream_t stream);

}  // namespace granite_b200
