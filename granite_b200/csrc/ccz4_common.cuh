// ccz4_common.cuh -- device-side data layout shared by the CCZ4 kernels.
//
// A block's fields use the reference GridBlock layout (grid.hpp:109-116):
// field-major, x fastest, 22 fields of double, nghost = 4. Every block of the
// hierarchy owns three such buffers in one device arena: the evolved state
// (slot 0) and two RK stage buffers (slots 1, 2) that the three stages
// ping-pong through, so no stage reads a buffer that the same launch writes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace granite_b200 {

constexpr int NV = 22;
constexpr int NG = 4;

// SpacetimeVar order, types.hpp:104-130
enum Var : int {
    CHI = 0, GXX, GXY, GXZ, GYY, GYZ, GZZ, AXX, AXY, AXZ, AYY, AYZ, AZZ,
    KTR, GHX, GHY, GHZ, THETA, ALPHA, BETAX, BETAY, BETAZ
};

// Block descriptor as the kernels see it (one per block, in device memory).
struct DevBlock {
    double* buf[3];      // state, stage A, stage B (slot 0/1/2)
    int n[3];            // interior cells
    int tx, ty, tz;      // cells incl. ghosts
    long long stride;    // cells per field
    double lo[3];
    double dx[3];
    double inv12h[3];    // 1/(12 dx)      first derivative (ccz4.cpp:72)
    double inv12h2[3];   // 1/(12 dx^2)    second derivative (ccz4.cpp:158)
    double inv4hh[3];    // 1/(4 dx_a dx_b) mixed (xy, xz, yz) (ccz4.cpp:188)
    double kocf[3];      // sigma/(64 dx)  KO (ccz4.cpp:886-887)
    double kow[3][4];    // kocf[d] * {1, -6, 15, -20}: the KO weights of ccz4.cpp:921
    int level;
    int moff;            // resident matter: cell offset of the block in the context's matter arrays
};

// One unit of the batched work-list: a tile of interior points of a block.
struct Tile {
    int block;
    int i0, j0, k0;  // interior-relative origin of the tile
    int w;           // tile width along x for the global-load stage kernels (32, 16 or 8;
                     // 128 threads cover w x 128/w points); 0 for fixed-shape kernels;
                     // -8 for an x-remainder tile of the TMA kernel (8 x 4 x 2 tz points)
};

// Interior cells of a source block that are ghost cells of a same-level
// neighbour (GRANITE_AMR_GHOSTS): the stage kernel that writes such a cell
// also writes it into the neighbour's ghost cell of the same buffer slot, so
// the fill after the stage leaves those cells out. Source interior indices
// [lo, hi) per axis; the destination cell of source interior index (i, j, k)
// is base + i + tx j + txy k in the neighbour's buffers (its pointers, field
// stride and row / plane lengths are carried here, so a push needs no lookup
// of the neighbour's descriptor).
struct PushBox {
    double* buf[3];
    long long stride;
    long long base;
    int tx, txy;
    int lo[3], hi[3];
};
// Push boxes of one tile staged in shared memory by the TMA stage kernel
// (more than this many: read from global memory).
constexpr int PUSH_STAGE_MAX = 16;

// Arguments of one fused RHS launch.
struct StageArgs {
    int in_sel;      // buffer slot the stencils read
    int n_sel;       // slot of u^n (pointwise, RK combine)
    int out_sel;     // slot written
    int final_stage; // 1: apply the algebraic constraints after the floors
    double a1, a2, a3dt;  // out = a1 u^n + a2 u_in + a3dt L(u_in)
    double chi_c, chi_w, kappa1, kappa2, eta;
    // standalone RHS output (EPI_STORE): rhs base per block is given by rhs_ptr
    double* rhs;     // single-block RHS destination (EPI_STORE only)
    // matter sources (nullable): rho[N], Si[N][3], Sij[N][6], S[N] over the cells of
    // all blocks, block b's cell c at N-index B.moff + c
    const double* rho; const double* Si; const double* Sij; const double* S;
    unsigned long long* nonfinite;  // floor hits on non-finite chi/alpha (nullable)
    const void* tmaps;     // TMA variant: CUtensorMap of (block b, slot s) at tmaps[3 b + s]
    const void* tmaps_rem; // TMA variant with x-remainder tiles: the same for their box shape
    unsigned int* errflag; // TMA variant: set to 1 when a bounded mbarrier wait gives up (nullable)
    // Per-tile precision (nullable): the launch covers only tiles ti with tile_prec[ti] == want_prec.
    const unsigned char* tile_prec;
    int want_prec;
    // Test switch of the TMA variant, 0 = off: CTA 0 never issues ring item
    // test_withhold - 1, so its bounded wait for that item runs out (no copy is
    // in flight for it) and the launch reports through errflag.
    int test_withhold;
    // Same-level ghost copies pushed from the RK epilogue (nullable): tile ti of
    // the launch's list pushes push[tile_push[ti].x .. + tile_push[ti].y).
    const PushBox* push;
    const int2* tile_push;
};

__host__ __device__ inline long long cell_index(const DevBlock& b, int i, int j, int k) {
    return (long long)i + (long long)b.tx * ((long long)j + (long long)b.ty * k);
}

// Cell-centre coordinate without FMA contraction, grid.hpp:92-94.
__device__ inline double coord(const DevBlock& b, int d, int idx) {
    return __dadd_rn(b.lo[d], __dmul_rn(__dadd_rn((double)(idx - NG), 0.5), b.dx[d]));
}

// Asymptotic value of the 1/r falloff, main.cpp:382-394.
__host__ __device__ inline double f_inf(int v) {
    return (v == CHI || v == GXX || v == GYY || v == GZZ || v == ALPHA) ? 1.0 : 0.0;
}

}  // namespace granite_b200
