// ccz4_kernels.h -- host-side launchers of the CCZ4 device kernels.
#pragma once

#include <cuda_runtime.h>

#include "ccz4_common.cuh"

namespace granite_b200 {

enum { EPI_STORE = 0, EPI_RK = 1 };

// Kernel variants of the fused stage: 0 = stencils from global memory
// (32x4x1 tiles), 1 = fields staged through shared memory with cp.async
// (16x4x2 tiles). The constraint and KO kernels always use variant-0 tiles.
enum { VARIANT_GLOBAL = 0, VARIANT_SMEM = 1, NUM_VARIANTS = 2 };

// Tile shape of a stage-kernel variant (points per CTA along x, y, z).
int stage_tile_dims(int variant, int* tx, int* ty, int* tz);

// Per-device kernel attributes (shared-memory opt-in); call with the device current.
cudaError_t configure_stage_kernels();

// Fused RHS (+KO) over a tile work-list. precision: 0 = FP64, 1 = mixed.
cudaError_t launch_stage(int variant, int precision, int epi, const DevBlock* blocks,
                         const Tile* tiles, int ntiles, const StageArgs& args, cudaStream_t stream);

// KO dissipation only: rhs += KO(u) at interior points of one block.
cudaError_t launch_dissipation(const DevBlock* block, int in_sel, double* rhs, int ntiles,
                               const Tile* tiles, cudaStream_t stream);

// Ghost-cell work items: one per (block, ghost cell); built on the host.
struct GhostItem {
    int block;
    int cell;  // linear cell index within the block (incl. ghosts)
};

enum GhostMode { GHOST_ZERO_GRADIENT = 0, GHOST_SOMMERFELD = 1, GHOST_PERIODIC = 2 };

// Fill every listed ghost cell of buffer slot `sel` for all 22 fields.
cudaError_t launch_ghost_fill(int mode, const DevBlock* blocks, const GhostItem* items, int nitems,
                              int sel, cudaStream_t stream);

// Trilinear prolongation (amr.cpp:484-564) of coarse block `cb` into the
// listed fine cells of fine block `fb` (slot sel of both).
struct ProlongItem {
    int fine_block;
    int coarse_block;
    int cell;  // fine cell index
};
cudaError_t launch_prolong(const DevBlock* blocks, const ProlongItem* items, int nitems, int sel,
                           cudaStream_t stream);

// 2x2x2 restriction (amr.cpp:566-626) into listed coarse cells.
struct RestrictItem {
    int coarse_block;
    int fine_block;
    int cell;      // coarse cell index
    int fine_base; // fine cell index of the (0,0,0) corner of the 2x2x2 stencil
};
cudaError_t launch_restrict(const DevBlock* blocks, const RestrictItem* items, int nitems, int sel,
                            cudaStream_t stream);

// Same-level ghost copy: dst cell of block a takes src cell of block b.
struct CopyItem {
    int dst_block, dst_cell, src_block, src_cell;
};
cudaError_t launch_copy(const DevBlock* blocks, const CopyItem* items, int nitems, int sel,
                        cudaStream_t stream);

// Constraint monitor (ccz4.cpp:941-1159) over a tile work-list. Writes ham /
// mom (single-block drop-in; may be null) and per-CTA partial sums of H^2 and
// |M|^2 to partials[2 * tile] (may be null).
cudaError_t launch_constraints(const DevBlock* blocks, const Tile* tiles, int ntiles, int sel,
                               double* ham, double* mom, double* partials, cudaStream_t stream);

// Deterministic fixed-order sum of n partial pairs into out[2].
cudaError_t launch_sum_partials(const double* partials, int n, double* out, cudaStream_t stream);

}  // namespace granite_b200
