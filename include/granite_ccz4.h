/*
 * granite_ccz4.h -- C ABI of the B200-native CCZ4 right-hand side and SSP-RK3
 * stage update (libgranite_ccz4.so, CUDA sm_100a).
 *
 * Drop-in boundary for GRANITE's spacetime operator and RK3 driver. Every
 * entry point below names the reference interface it replaces (paths inside
 * the GRANITE tree). Field data always uses the reference GridBlock layout
 * (include/granite/core/grid.hpp:109-116):
 *
 *   buf[v * stride + i + tx * (j + ty * k)],   tx = nx + 2 ng,  ty = ny + 2 ng,
 *   stride = tx * ty * (nz + 2 ng),  v in SpacetimeVar order
 *   (include/granite/core/types.hpp:104-130), 22 fields of double.
 *
 * so GridBlock::flatBuffer() can be passed unchanged.
 *
 * Conventions
 *   - Every function returns an int status: GRANITE_OK (0) or a negative
 *     GRANITE_ERR_* code; nothing aborts or traps. The message of the last
 *     failure on a context is available from granite_ccz4_last_error().
 *   - A context owns one CUDA device, one CUDA stream and all device memory it
 *     allocates. A context is not re-entrant: call it from one host thread at
 *     a time (the reference operator is const and re-entrant on the host; a
 *     caller that needs concurrency creates one context per thread).
 *   - "_host" entry points take host pointers and block until results are in
 *     host memory. Resident-block entry points enqueue work on the context's
 *     stream; granite_ccz4_sync() waits for it.
 *   - There is no CPU fallback: without a usable sm_100 device,
 *     granite_ccz4_create() fails with GRANITE_ERR_NO_DEVICE.
 */
#ifndef GRANITE_CCZ4_H
#define GRANITE_CCZ4_H

#include <stddef.h>

#if defined(__GNUC__)
#define GRANITE_API __attribute__((visibility("default")))
#else
#define GRANITE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define GRANITE_CCZ4_NUM_VARS 22
#define GRANITE_CCZ4_ABI_VERSION 1

/* status codes */
#define GRANITE_OK 0
#define GRANITE_ERR_INVALID (-1)     /* bad argument, size or state */
#define GRANITE_ERR_CUDA (-2)        /* CUDA runtime error (message has the detail) */
#define GRANITE_ERR_NO_DEVICE (-3)   /* no sm_100 device / driver */
#define GRANITE_ERR_NOMEM (-4)       /* device or pinned allocation failed */
#define GRANITE_ERR_NONFINITE (-5)   /* non-finite values detected in the evolved state */
#define GRANITE_ERR_UNSUPPORTED (-6) /* option the library does not implement */
#define GRANITE_ERR_TIMEOUT (-7)     /* a bounded host-side wait gave up */
#define GRANITE_ERR_TOO_LARGE (-8)   /* request exceeds a fixed capacity of the library */

/* arithmetic of the RHS algebra */
#define GRANITE_PRECISION_FP64 0  /* plain FP64 throughout */
#define GRANITE_PRECISION_MIXED 1 /* FP32 algebra from FP64 stencil differences;
                                     FP64 state, RK3 accumulation, chi, inverse metric */

/* boundary treatment of a single-level (level-0) step */
#define GRANITE_BC_REFERENCE 0 /* zero-gradient level fill (amr.cpp:400-482) before and after
                                  the step, 1/r falloff on every stage buffer (main.cpp:351-521) */
#define GRANITE_BC_PERIODIC 1  /* periodic wrap everywhere (gauge-wave test; the reference has
                                  no periodic boundary) */

/* Berger-Oliger inter-level semantics of granite_ccz4_hierarchy_step */
#define GRANITE_AMR_REFERENCE 0  /* prolongate coarse data into ALL cells of a fine block before
                                    and after each fine step, as amr.cpp:313-318,438 do */
#define GRANITE_AMR_GHOSTS 1     /* prolongate into fine ghost cells only; same-level
                                    neighbours copy ghosts from each other */

/* CCZ4Params, include/granite/spacetime/ccz4.hpp:25-34 */
typedef struct {
    double kappa1;           /* 0.02 */
    double kappa2;           /* 0.0 */
    double eta;              /* 2.0 */
    double ko_sigma;         /* 0.1; <= 0 disables KO exactly as applyDissipation does */
    double chi_blend_center; /* 0.05 */
    double chi_blend_width;  /* 0.02 */
    int fd_order;            /* must be 4: the only order ccz4.cpp implements */
    int device;              /* CUDA device ordinal */
} granite_ccz4_params;

/* Geometry of one GridBlock, mirroring its constructor (grid.hpp:55-61,
 * grid.cpp:12-31): dx = (hi - lo) / ncells. nghost must be 4 (the upwind
 * stencil reaches i +- 4, ccz4.cpp:109-152). */
typedef struct {
    int ncells[3];
    int nghost;
    double lo[3];
    double hi[3];
    int level; /* AMR level, 0 = coarsest */
    int id;    /* caller's block id (informational) */
} granite_block_desc;

/* ---- context --------------------------------------------------------- */

/* Fills p with the CCZ4Params defaults (ccz4.hpp:25-34), device 0. */
GRANITE_API void granite_ccz4_default_params(granite_ccz4_params* p);

/* Replaces: CCZ4Evolution::CCZ4Evolution(const CCZ4Params&), ccz4.hpp:60. */
GRANITE_API int granite_ccz4_create(const granite_ccz4_params* p, void** ctx);
GRANITE_API int granite_ccz4_destroy(void* ctx);
/* Copies the message of the last failure (empty if none) into buf. */
GRANITE_API int granite_ccz4_last_error(const void* ctx, char* buf, size_t len);
/* Waits for all work enqueued on the context's stream. */
GRANITE_API int granite_ccz4_sync(void* ctx);
GRANITE_API int granite_ccz4_abi_version(void);

/* ---- stateless operators on host buffers (drop-in for CCZ4Evolution) --- */

/* Replaces: CCZ4Evolution::computeRHS / computeRHSVacuum, ccz4.hpp:69-81,
 * ccz4.cpp:229-865 (RHS + Kreiss-Oliger). Writes interior cells of rhs;
 * ghost cells of rhs keep their values. rho[N], Si[N][3], Sij[N][6], S[N]
 * (N = cells of the block incl. ghosts) are the matter sources; pass all four
 * NULL for vacuum. precision: GRANITE_PRECISION_*. */
GRANITE_API int granite_ccz4_compute_rhs_host(void* ctx, const granite_block_desc* b, const double* u,
                                  double* rhs, const double* rho, const double* Si,
                                  const double* Sij, const double* S, int precision);

/* Replaces: CCZ4Evolution::applyDissipation, ccz4.hpp:99, ccz4.cpp:871-935.
 * rhs (interior) += KO(u). */
GRANITE_API int granite_ccz4_apply_dissipation_host(void* ctx, const granite_block_desc* b,
                                        const double* u, double* rhs);

/* Replaces: CCZ4Evolution::computeConstraints, ccz4.hpp:90-92,
 * ccz4.cpp:941-1159. ham[N], mom[N][3] over the whole block, ghosts zero. */
GRANITE_API int granite_ccz4_compute_constraints_host(void* ctx, const granite_block_desc* b,
                                          const double* u, double* ham, double* mom);

/* Same RHS on caller-owned device memory, enqueued on `stream` (a
 * cudaStream_t, NULL = the context stream). No host synchronisation. */
GRANITE_API int granite_ccz4_compute_rhs_device(void* ctx, const granite_block_desc* b, const double* u_dev,
                                    double* rhs_dev, const double* rho_dev, const double* Si_dev,
                                    const double* Sij_dev, const double* S_dev, int precision,
                                    void* stream);

/* Replaces: GRMHDEvolution::computeMatterSources, grmhd.hpp:333-338,
 * grmhd.cpp:1034-1103 (the matter sources main.cpp:300 hands to computeRHS).
 * prim[11][N]: the primitive GridBlock's flatBuffer() (PrimitiveVar order rho,
 * v^x, v^y, v^z, p, B^x, B^y, B^z, eps, T, Ye; types.hpp:149-162); rho[N],
 * Si[N][3], Sij[N][6], S[N]: written at interior cells, equal to the
 * reference's bit for bit; other cells keep their values. */
GRANITE_API int granite_ccz4_matter_sources_host(void* ctx, const granite_block_desc* b, const double* prim,
                                                 double* rho, double* Si, double* Sij, double* S);
/* Same on device memory, enqueued on `stream` (NULL = the context stream). */
GRANITE_API int granite_ccz4_matter_sources_device(void* ctx, const granite_block_desc* b, const double* prim_dev,
                                                   double* rho_dev, double* Si_dev, double* Sij_dev,
                                                   double* S_dev, void* stream);

/* ---- resident blocks ----------------------------------------------------- */
/* The hierarchy lives in one device arena per context: add every block, then
 * commit (allocates state + 2 stage buffers per block and builds the per-level
 * tile work-lists), then upload. Replaces the GridBlock storage owned by
 * AMRHierarchy::Level (amr.hpp:104-109). */

GRANITE_API int granite_ccz4_add_block(void* ctx, const granite_block_desc* b, int* block_index);
GRANITE_API int granite_ccz4_commit(void* ctx);

/* Resident matter coupling (the non-vacuum applyRHS of main.cpp:296-302):
 * before commit, granite_ccz4_enable_matter(ctx, 1) gives every block 11
 * matter-source fields (rho, S_i, S_ij, S; zero = vacuum), which every RHS of
 * rk3_step / hierarchy_step reads. granite_ccz4_upload_primitives (host
 * prim[11][N]) or _set_primitives_device (device, stream-ordered on the
 * context stream) recompute a block's sources from its primitives with
 * computeMatterSources; they stay fixed until the next call. Blocks a regrid
 * adds start in vacuum. */
GRANITE_API int granite_ccz4_enable_matter(void* ctx, int on);
GRANITE_API int granite_ccz4_upload_primitives(void* ctx, int block_index, const double* prim);
GRANITE_API int granite_ccz4_set_primitives_device(void* ctx, int block_index, const double* prim_dev);

/* Replaces the block creation of AMRHierarchy::regrid (amr.cpp:80-301), which
 * only ever adds blocks: appends n blocks (levels >= 1) to a committed
 * hierarchy. Existing blocks keep their state and their indices; each new
 * block gets indices num_blocks() .. in the order given and is filled in every
 * cell (ghosts included) by trilinear prolongation from its coarser level as
 * the reference's regrid does (amr.cpp:291-293: each coarse block in list order
 * overwrites every fine cell, so the level's last block decides). New blocks
 * are filled in ascending level order. The arena is reallocated (a device-side
 * copy of the states), work-lists and tensor maps are rebuilt, cached step
 * graphs are dropped. Which boxes to add (tracking spheres, taggers) is the
 * caller's decision; granite_ccz4_tag_count gives the reference taggers' cell
 * counts on the device. */
GRANITE_API int granite_ccz4_regrid_add(void* ctx, const granite_block_desc* blocks, int n);
/* Replaces gradientChiTagger / gradientLapseTagger (amr.cpp:653-731) as the
 * regrid uses them: the number of interior cells of `level` (state slot 0)
 * with |grad f| / (|f| + 1e-30) > threshold, f = chi (var 0) or the lapse
 * (var 18), evaluated in the reference's order. Blocks until the count is on
 * the host. */
GRANITE_API int granite_ccz4_tag_count(void* ctx, int level, int var, double threshold, long long* count);
GRANITE_API int granite_ccz4_num_blocks(const void* ctx);
/* bytes of device memory held by the arena after commit */
GRANITE_API int granite_ccz4_arena_bytes(const void* ctx, size_t* bytes);
GRANITE_API int granite_ccz4_upload_block(void* ctx, int block_index, const double* host_u);
GRANITE_API int granite_ccz4_download_block(void* ctx, int block_index, double* host_u);
/* Every block at once: hosts[i] is block i's flatBuffer() (num_blocks entries).
 * upload_all is stream-ordered and returns at once (keep the buffers until the
 * next sync); download_all returns when all blocks are on the host. One
 * synchronisation for the whole hierarchy instead of one per block; pinned
 * buffers let the copies run at full PCIe rate. */
GRANITE_API int granite_ccz4_upload_all(void* ctx, const double* const* hosts);
GRANITE_API int granite_ccz4_download_all(void* ctx, double* const* hosts);
/* download_all without the wait: the copies are queued on the context's stream
 * behind the work already enqueued and the call returns at once; the host
 * buffers hold the state after the next granite_ccz4_sync (which also reports a
 * stage whose tile wait gave up). With pinned buffers and two contexts, one
 * context's copies run on the copy engines while the other's steps run on the
 * SMs. */
GRANITE_API int granite_ccz4_download_all_async(void* ctx, double* const* hosts);

/* ---- stepping -------------------------------------------------------------- */

/* Replaces: one AMRHierarchy::subcycle(0) pass (amr.cpp:303-330) around
 * TimeIntegrator::sspRK3Step (main.cpp:86-690, spacetime part) for every
 * block of `level`, treated as independent single-level blocks: level ghost
 * fill, 3 fused RHS+KO+RK-combine+floor launches (batched over all blocks of
 * the level), outer boundary per stage, algebraic constraints on the last
 * stage, level ghost fill. bc: GRANITE_BC_*. Enqueued as one CUDA graph. */
GRANITE_API int granite_ccz4_rk3_step(void* ctx, int level, double dt, int precision, int bc);

/* Replaces: AMRHierarchy::subcycle(0, evolve, ...) recursion over all levels
 * (amr.cpp:303-350) with the RK3 step above as evolve_func
 * (main.cpp:1142-1177): level l advances by dt_coarse / 2^l, twice per parent
 * step, followed by restriction to the parent. amr_mode: GRANITE_AMR_*. */
GRANITE_API int granite_ccz4_hierarchy_step(void* ctx, double dt_coarse, int precision, int amr_mode);

/* The regrid point of AMRHierarchy::subcycle (amr.cpp:343-349): called after
 * level `level`'s step (its restriction from the finer level included) when
 * step_num = round(current_time / (dt + 1e-15)) is a multiple of the regrid
 * interval. It runs on the calling thread with the stream synchronised and may
 * call granite_ccz4_tag_count and granite_ccz4_regrid_add on the same context;
 * a non-zero return stops the step and is returned by it. */
typedef int (*granite_regrid_fn)(void* user, int level, long long step_num);

/* granite_ccz4_hierarchy_step with the reference's in-step regrid
 * (AMRHierarchy::subcycle with regrid_interval > 0, amr.cpp:303-350): `fn`
 * runs at every regrid point of every level, in the reference's order, and the
 * levels it creates join the remaining substeps of the coarse step. Not
 * captured in a graph. regrid_interval = 0 never calls fn. */
GRANITE_API int granite_ccz4_hierarchy_step_regrid(void* ctx, double dt_coarse, int precision, int amr_mode,
                                                   int regrid_interval, granite_regrid_fn fn, void* user);

/* ---- gravitational-wave extraction ------------------------------------------
 * Replaces Psi4Extractor::extract + getMode (postprocess.hpp:34-77,
 * postprocess.cpp:245-326) on one block: modes[r][q][re, im] for the nr
 * extraction radii (host array) and q over l = 2..l_max, m = -l..l
 * ((l_max + 1)^2 - 4 modes), the sphere sampled at n_theta x n_phi points as
 * GWExtractionParams describes, points within one cell of the block's faces
 * skipped. Equal to the reference to rounding (sin, cos, pow are CUDA's; the
 * sums run in a fixed tree order). The resident form reads state slot 0 of
 * block_index, the device / host forms a caller's field-major block.
 * npoints[r] (nullable) gets the number of sphere points of radius r inside
 * the block: 0 means the reference records no mode for that radius. Blocks
 * until the modes are on the host. 2 <= l_max <= 16. */
GRANITE_API int granite_ccz4_psi4_modes(void* ctx, int block_index, const double* radii, int nr, int n_theta,
                                        int n_phi, int l_max, double* modes, int* npoints);
GRANITE_API int granite_ccz4_psi4_modes_device(void* ctx, const granite_block_desc* b, const double* u_dev,
                                               const double* radii, int nr, int n_theta, int n_phi, int l_max,
                                               double* modes, int* npoints);
GRANITE_API int granite_ccz4_psi4_modes_host(void* ctx, const granite_block_desc* b, const double* u,
                                             const double* radii, int nr, int n_theta, int n_phi, int l_max,
                                             double* modes, int* npoints);

/* ---- apparent horizons ------------------------------------------------------
 * HorizonParams and the HorizonData fields the finder fills
 * (horizon_finder.hpp:17-41); spin_axis is always z there, surface points are
 * center + radii[i][j] * (sin t_i cos p_j, sin t_i sin p_j, cos t_i) with
 * t_i = pi (i + 1/2) / n, p_j = 2 pi j / (2 n), n = angular_resolution. */
typedef struct {
    int max_iterations;          /* 200 */
    double tolerance;            /* 1e-10 */
    int angular_resolution;      /* 50 theta points; 2x as many phi points */
    double initial_guess_radius; /* 1.0 */
} granite_horizon_params;

typedef struct {
    int found;      /* 1: the flow converged (otherwise the other fields are 0) */
    int iterations; /* flow iterations run */
    int id;
    double centroid[3];
    double area, irreducible_mass, spin;
    double circumference_equatorial, circumference_polar;
} granite_horizon;

GRANITE_API void granite_ccz4_default_horizon_params(granite_horizon_params* p);
/* Replaces ApparentHorizonFinder::findHorizon (horizon_finder.cpp:310-449) on
 * resident block block_index: the expansion flow from a sphere of the initial
 * radius about center, on the GPU, equal to the reference bit for bit (the
 * surface integrals are summed on the host in its order). radii (nullable,
 * n x 2n) receives the final surface, also when the flow did not converge. */
GRANITE_API int granite_ccz4_find_horizon(void* ctx, int block_index, const granite_horizon_params* p,
                                          const double* center, granite_horizon* out, double* radii);
/* The same on a caller's host block (copied to the GPU first). */
GRANITE_API int granite_ccz4_find_horizon_host(void* ctx, const granite_block_desc* b, const double* u,
                                               const granite_horizon_params* p, const double* center,
                                               granite_horizon* out, double* radii);
/* Replaces findAllHorizons (horizon_finder.cpp:452-507): candidate centres at
 * lapse minima below 0.5 (scan on the GPU, cells two in from the faces, in the
 * reference's order, at most 65536), those within 2 initial radii of an
 * earlier one dropped, then findHorizon from each; found horizons get ids
 * 0, 1, ... in order. Writes min(found, cap) to out, *n = found. */
GRANITE_API int granite_ccz4_find_all_horizons(void* ctx, int block_index, const granite_horizon_params* p,
                                               granite_horizon* out, int cap, int* n);

/* ---- checkpoint / restart --------------------------------------------------
 * Replaces HDF5Writer::writeCheckpoint / HDF5Reader::readCheckpoint
 * (hdf5_io.cpp:166-233, 392-467) for the resident state, with their data model
 * (time, step, num_blocks; per block b every field v as "block_b/var_v", the
 * block's totalSize() values) in a flat container (the HDF5 library is not
 * linked) that also stores each block's geometry, the level times and the
 * resident matter sources, so a hierarchy resumes exactly where it stopped.
 * Restart: read the header (blocks may be NULL to get num_blocks first), add
 * those blocks in that order, enable matter if has_matter, commit, then
 * granite_ccz4_checkpoint_read. A bad or mismatching file returns
 * GRANITE_ERR_INVALID and leaves the state unspecified only if the data part
 * is truncated. Blocks until the file is written / the state is on the GPU. */
GRANITE_API int granite_ccz4_checkpoint_write(void* ctx, const char* path, int step, double time);
GRANITE_API int granite_ccz4_checkpoint_header(const char* path, int* step, double* time, int* has_matter,
                                               granite_block_desc* blocks, int cap, int* num_blocks);
GRANITE_API int granite_ccz4_checkpoint_read(void* ctx, const char* path, int* step, double* time);

/* Level::current_time (amr.hpp:108-113): the sum of the level's step sizes so
 * far; a level created by a regrid starts at its parent's time. */
GRANITE_API int granite_ccz4_level_time(void* ctx, int level, double* t);

/* ---- diagnostics ----------------------------------------------------------- */

/* Replaces the constraint monitor of main.cpp:1216-1254:
 * ||H||_2 = sqrt(sum H^2 / N) and ||M||_2 = sqrt(sum |M|^2 / N) over all
 * interior points of the given level (-1 = all levels). Deterministic. */
GRANITE_API int granite_ccz4_constraint_norms(void* ctx, int level, double* h_l2, double* m_l2);

/* Compares the evolved states (slot 0) of two committed contexts of identical
 * block geometry on one device, e.g. the same hierarchy stepped in
 * GRANITE_PRECISION_FP64 and _MIXED (no counterpart in the reference). Per
 * field v over the interior cells of all blocks: max_dev[v] = max |a - b|,
 * max_abs[v] = max |a| (22 values each; NaN differences are left out of the
 * maxima); nonfinite[0], nonfinite[1] = the non-finite values in a and in b.
 * Waits for both contexts' streams. */
GRANITE_API int granite_ccz4_compare_states(void* ctx_a, void* ctx_b, double* max_dev, double* max_abs,
                                            long long* nonfinite);

/* Number of non-finite chi/alpha values met by the floors since the last call
 * (the floors repair them, main.cpp:586-608); a health signal, not an error. */
GRANITE_API int granite_ccz4_nonfinite_count(void* ctx, long long* count);

/* ---- tracing ---------------------------------------------------------------- */

/* kernel classes reported by the profiler */
#define GRANITE_KERNEL_STAGE 0       /* fused RHS + KO + RK-stage kernel */
#define GRANITE_KERNEL_GHOST 1       /* ghost fills (level fill, outer boundary) */
#define GRANITE_KERNEL_TRANSFER 2    /* prolongation, restriction, same-level copies */
#define GRANITE_KERNEL_CONSTRAINTS 3 /* constraint monitor + reduction */
#define GRANITE_KERNEL_CLASSES 4

/* While profiling is on, stepping runs without CUDA graphs and brackets every
 * launch with CUDA events on the context stream; granite_ccz4_profile_get
 * returns the summed device time and launch count of a kernel class since the
 * last reset (it synchronises the stream). No counterpart in the reference
 * (which has no timers). */
GRANITE_API int granite_ccz4_set_profiling(void* ctx, int enabled);
/* Sustained FMA rate of a device in TFLOP/s (2 flops per FMA), FP64
 * (GRANITE_PRECISION_FP64) or FP32 (GRANITE_PRECISION_MIXED), from a
 * register-only kernel at full occupancy: the compute roofline the stage
 * kernels are measured against. No counterpart in the reference. */
GRANITE_API int granite_ccz4_measure_fma_rate(int device, int precision, double* tflops);
GRANITE_API int granite_ccz4_profile_reset(void* ctx);
GRANITE_API int granite_ccz4_profile_get(void* ctx, int kernel_class, double* total_ms,
                                         long long* launches);
/* Stage-kernel variant (set before granite_ccz4_commit; no counterpart in the
 * reference): GRANITE_VARIANT_GLOBAL reads stencils from global memory through
 * L1 (32x4x1 tiles); GRANITE_VARIANT_SMEM stages every field of a 16x4x2 tile
 * and its halo through shared memory with cp.async. In a committed hierarchy the
 * GLOBAL tiles are w x 128/w points with w in {32, 16, 8} chosen per block to
 * leave the fewest idle threads. GRANITE_VARIANT_TMA (the default) runs one
 * persistent CTA per SM that streams every field of a 16x4x4 tile and its
 * 4-cell halo into a ring of shared-memory slots with tensor-map (TMA) loads;
 * blocks it cannot map (odd x extent, fewer than 16 x or 4 y/z interior cells)
 * send their level to GRANITE_VARIANT_GLOBAL. A TMA load that does not complete
 * within its wait limit makes the next granite_ccz4_sync, block download
 * (download_block / download_all) or compute_rhs_host return GRANITE_ERR_CUDA.
 * All variants compute identical FP64 results. */
#define GRANITE_VARIANT_GLOBAL 0
#define GRANITE_VARIANT_SMEM 1
#define GRANITE_VARIANT_GLOBAL_R168 2 /* GLOBAL with at most 168 registers (3 CTAs / SM) */
#define GRANITE_VARIANT_GLOBAL_R128 3 /* GLOBAL with at most 128 registers (4 CTAs / SM) */
#define GRANITE_VARIANT_TMA 4
GRANITE_API int granite_ccz4_set_kernel_variant(void* ctx, int variant);
GRANITE_API int granite_ccz4_get_kernel_variant(const void* ctx, int* variant);

/* Per-class configurations of GRANITE_VARIANT_TMA (no counterpart in the
 * reference, whose computeRHS runs one OpenMP loop per block, ccz4.cpp:267-270).
 * The TMA stage kernel exists in GRANITE_STAGE_CONFIGS configurations (see
 * granite_ccz4_stage_config_info): tiles of 16 x 4 x tile_z points, ring_slots
 * field boxes in flight, the stage input's centre values kept in shared memory
 * for the RK epilogue (shared_input), the Hessian-field loop's values in shared
 * memory (shared_hessian). Every block belongs to the block-size class whose
 * edge (GRANITE_STAGE_CLASS_EDGES) is nearest on a log scale to the cube root of
 * its interior volume; each (precision, class) has a configuration, the
 * autotuner's B200 winners by default (granite_b200/tuner.py re-tunes and
 * writes a table a caller can apply). A level's blocks of different
 * configurations run as one launch per configuration. Set before commit.
 * All configurations compute identical FP64 results. */
#define GRANITE_STAGE_CONFIGS 18
#define GRANITE_STAGE_CLASSES 6
#define GRANITE_STAGE_CLASS_EDGES 16, 24, 32, 48, 64, 96
/* cls: class index (0 .. GRANITE_STAGE_CLASSES - 1) or -1 for every class;
 * cfg: configuration or -1 for the built-in default. */
GRANITE_API int granite_ccz4_set_stage_config(void* ctx, int precision, int cls, int cfg);
GRANITE_API int granite_ccz4_get_stage_config(const void* ctx, int precision, int cls, int* cfg);
/* One configuration for every block and precision (-1: back to the per-class table). */
GRANITE_API int granite_ccz4_force_stage_config(void* ctx, int cfg);
GRANITE_API int granite_ccz4_stage_config_info(int cfg, int* tile_z, int* ring_slots, int* shared_input,
                                               int* shared_hessian);
/* The schedule of a configuration: warp_specialized = 1 when the mixed RK
 * kernels split stencil and algebra warps; ctas_per_sm = the resident CTAs per
 * SM its register allocation is sized for (3: at most 168 registers a thread);
 * items_per_barrier = field boxes consumed per CTA barrier (1 or 2);
 * x_remainder_tiles = 1 when a block whose x extent is 8 more than a multiple
 * of 16 covers its last 8 columns with 8 x 4 x 4 tiles instead of 16-wide tiles
 * half outside the block. Null outputs are skipped. */
GRANITE_API int granite_ccz4_stage_config_schedule(int cfg, int* warp_specialized, int* ctas_per_sm,
                                                   int* items_per_barrier, int* x_remainder_tiles);
GRANITE_API int granite_ccz4_block_stage_class(const granite_block_desc* b, int* cls);

/* Test switch of the wait limit above (no counterpart in the reference, which
 * has no device waits; its failure detection is the NaN scan of
 * main.cpp:525-568): the next granite_ccz4_rk3_step runs uncaptured and, in its
 * first stage launch, the first persistent CTA never issues ring item `item`
 * (item q = field q % 22 of the CTA's tile round q / 22). Nothing is in flight
 * for that item, so the CTA's bounded waits run out (about 2 s), the step's
 * state is garbage, and the next granite_ccz4_sync returns GRANITE_ERR_CUDA
 * with the wait-limit message; the sync after that returns GRANITE_OK and the
 * context keeps working. One-shot; TMA variant only. */
GRANITE_API int granite_ccz4_test_withhold_tile_load(void* ctx, int item);

/* Per-tile precision of GRANITE_PRECISION_MIXED steps (no counterpart in the
 * reference): in every RK stage of granite_ccz4_rk3_step /
 * granite_ccz4_hierarchy_step a classification kernel flags the tiles whose
 * stage input has a point with chi < chi_fp64 (or a non-finite chi); those
 * tiles are computed with the FP64 algebra (FP64 pair-difference stencils:
 * equal to GRANITE_PRECISION_FP64 to rounding, not bit for bit), every other
 * tile with the FP32 algebra. The flags come from the current chi on the
 * device, so the choice follows moving punctures and stays inside the step's
 * CUDA graph. 0 (the default) disables it; a value above every chi runs the
 * FP64 algebra on every tile. Changing it drops the cached step graphs. The
 * stateless operators (granite_ccz4_compute_rhs_*) are not affected. */
GRANITE_API int granite_ccz4_set_fp64_chi_threshold(void* ctx, double chi_fp64);
/* 1: the FP64 pass of the per-tile precision runs on a second stream of the
 * context beside the FP32 pass (they write disjoint tiles); 0 (default): after
 * it. Measured on the binary hierarchy: 67.9 vs 67.2 ms per coarse step, the
 * concurrent FP64 CTAs take SM slots the persistent FP32 pass needs. */
GRANITE_API int granite_ccz4_set_pass_overlap(void* ctx, int on);
GRANITE_API int granite_ccz4_get_fp64_chi_threshold(const void* ctx, double* chi_fp64);

/* Same-level ghost copies in GRANITE_AMR_GHOSTS (no counterpart in the
 * reference): with 1 the stage kernels write every interior value a same-level
 * neighbour holds as a ghost cell into that ghost cell of the same buffer, and
 * the fills after the stages only prolongate and apply the block-local fills;
 * 0 (the default) = the fills copy them (the same values: results are
 * identical). Levels whose interiors overlap (after a regrid) always copy.
 * Measured on the binary hierarchy: 73.4 ms per coarse step with pushes, 66.8
 * without; a 16^3 block pushes 87 % of its cells, and the stage kernel's
 * scattered ghost stores cost more than the fill kernel's copies. */
GRANITE_API int granite_ccz4_set_ghost_push(void* ctx, int on);

/* Batching (no counterpart in the reference): 1 (default) = one launch per
 * level and RK stage over all blocks, each step replayed as one CUDA graph;
 * 0 = one launch per block and stage, issued eagerly, as a per-block drop-in
 * of the reference's per-GridBlock operator calls would run. */
GRANITE_API int granite_ccz4_set_batching(void* ctx, int batched);

/* The context's cudaStream_t, for callers that order their own work or events
 * against the library's. */
GRANITE_API int granite_ccz4_get_stream(void* ctx, void** stream);

/* Kernel launches issued by this context so far (graph nodes count once per
 * replay). */
GRANITE_API int granite_ccz4_launch_count(const void* ctx, long long* count);

/* ---- allocation-free constraint norms --------------------------------------- */

/* No counterpart in the reference. ||H||_2 and ||M||_2 (the same norms as
 * granite_ccz4_constraint_norms) of ONE block whose state u_dev (GridBlock
 * layout, 22 fields) already sits in device memory, for callers that cannot
 * allocate device memory themselves: code running inside another runtime's
 * memory pool or a pre-sized arena, or code that must not call cudaMalloc /
 * cudaFree because those calls synchronise the device and would stall work in
 * flight on other streams. It needs no context and allocates nothing: its
 * scratch (one pair of partial sums per 32x4x1 tile of interior points) is a
 * fixed 1 MiB array in the library's device data, held by every GPU that loads
 * the library until the process exits.
 *   - Limit: at most 65,536 tiles, i.e. ceil(nx/32) * ceil(ny/4) * nz <= 65536
 *     (8,388,608 interior points for tile-aligned blocks); larger blocks return
 *     GRANITE_ERR_TOO_LARGE and launch nothing.
 *   - norms_dev: caller-owned device memory for 2 doubles; written by the last
 *     kernel of the call. Work is enqueued on `stream` (a cudaStream_t; NULL =
 *     the legacy default stream) of the current device; nothing is synchronised.
 *   - The first call on a device looks up the array's device address on that
 *     device (it must be the current device); make that first call before any
 *     stream capture. The address is looked up again when the device's context
 *     has changed since (after a device reset, the module can load elsewhere).
 *   - The status reflects this call's own launches only: an error left by the
 *     caller's earlier work is neither reported here nor cleared.
 *   - Every call shares the one array: calls whose kernels may overlap on the
 *     GPU (other streams, other host threads) race on it. Each call rewrites
 *     every partial it reads, so nothing needs clearing between calls. */
GRANITE_API int granite_ccz4_constraint_norms_noalloc(const granite_block_desc* b, const double* u_dev,
                                                      double* norms_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GRANITE_CCZ4_H */
