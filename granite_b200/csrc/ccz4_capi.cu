// ccz4_capi.cu -- implementation of the C ABI in include/granite_ccz4.h.
//
// Host runtime: one context = one device + one stream + one device arena for
// all resident blocks (three 22-field buffers per block: state and two RK
// stage buffers), per-level tile work-lists for the batched RHS launches,
// ghost-cell chunk lists for the fills, and a cache of CUDA graphs, one per
// (level, precision, boundary, dt) step shape.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <climits>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/granite_ccz4.h"
#include "ccz4_common.cuh"
#include "ccz4_kernels.h"

using namespace granite_b200;

namespace granite_b200 {

// Tensor map of one block buffer for the TMA stage kernel: 4-D (x, y, z,
// field) over the cells incl. ghosts, FP64, box = 16 x 4 x tz tile + 4-cell
// halo, no swizzle, zero fill outside the block. The driver's encoder is looked
// up once through the runtime (no link against libcuda).
bool encode_block_tmap(void* map128, const double* base, const DevBlock& d, int tz) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        else
            cudaGetLastError();
    });
    if (!encode || !base) return false;
    // global address 16-byte aligned, every stride a multiple of 16 bytes (x extent even)
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (d.tx & 1) != 0) return false;
    const int bz = tz + 8;
    if (d.tx < TMA_BOX_X || d.ty < TMA_BOX_Y || d.tz < bz) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)d.tx, (cuuint64_t)d.ty, (cuuint64_t)d.tz, (cuuint64_t)NV};
    const cuuint64_t strides[3] = {(cuuint64_t)d.tx * sizeof(double), (cuuint64_t)d.tx * d.ty * sizeof(double),
                                   (cuuint64_t)d.stride * sizeof(double)};
    const cuuint32_t box[4] = {(cuuint32_t)TMA_BOX_X, (cuuint32_t)TMA_BOX_Y, (cuuint32_t)bz, 1};
    const cuuint32_t estride[4] = {1, 1, 1, 1};
    const CUresult r = encode(static_cast<CUtensorMap*>(map128), CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                              const_cast<double*>(base), dims, strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace granite_b200

namespace {

// Stage configuration per (precision: FP64, MIXED) and block-size class
// (GRANITE_STAGE_CLASS_EDGES) until a caller sets its own: the autotuner's
// (granite_b200/tuner.py) uniform table on a B200, one configuration per
// precision, so a level stage stays one launch. Mixed: configuration 12
// (x-remainder tiles) has the least total over the classes, its 19-23 % gain
// on blocks 8 cells wider than a multiple of 16 outweighing 1-3 % elsewhere.
constexpr int DEFAULT_CLASS_CFG[2][GRANITE_STAGE_CLASSES] = {{0, 0, 0, 0, 0, 0}, {12, 12, 12, 12, 12, 12}};

static_assert(sizeof(CUtensorMap) == 128, "tensor maps are 128 bytes");
static_assert(alignof(CUtensorMap) >= 64, "tensor maps are 64-byte aligned");

// The global-load kernels pick their tile width per block; the others use fixed tiles.
bool adaptive_tiles(int variant) { return variant != VARIANT_SMEM && variant != VARIANT_TMA; }

struct Graph {
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
};

// Tiles of one stage-kernel configuration within a level's work-list: one launch.
struct StageGroup {
    int cfg;          // TMA configuration (TMA_CFGS), 0 for the other variants
    int first, count; // range of the level's tiles
};

struct LevelLists {
    std::vector<int> blocks;
    int variant = VARIANT_GLOBAL;  // stage kernel of this level: the context's variant, or GLOBAL
                                   // when a block cannot be mapped for TMA
    // stage-kernel tiles: per precision (0 FP64, 1 MIXED) grouped by
    // configuration (groups), each block's tiles contiguous (tile_range)
    Tile* d_tiles = nullptr;
    std::vector<Tile> h_tiles;       // host copy of d_tiles (push lists are built from it)
    std::vector<StageGroup> groups[2];
    std::vector<int> block_cfg[2];  // per block of the level: its configuration
    int ntiles = 0;
    unsigned char* d_flags = nullptr;  // per-tile precision of MIXED steps (1 = FP64 algebra)
    Tile* d_mtiles = nullptr;  // constraint-monitor tiles (variant-0 shape)
    int nmtiles = 0;
    GhostItem* d_ghost = nullptr;
    int nghost = 0;
    long long interior_points = 0;
    // per block of the level: [first, first + count) of its tiles (per precision) / ghost chunks
    std::vector<std::pair<int, int>> tile_range[2], ghost_range;
};

// Device copy of a list of transfer boxes and the chunks that cover them.
struct XferList {
    XferBox* d_boxes = nullptr;
    BoxChunk* d_chunks = nullptr;
    int nchunks = 0;
    int nboxes = 0;
};

void free_xfer(XferList& x) {
    cudaFree(x.d_boxes);
    cudaFree(x.d_chunks);
    x = XferList();
}

// Inter-level / inter-block transfer lists of one level for one AMR mode.
struct LevelXfer {
    XferList prolong;               // into this level from level-1 (ghost slabs, or whole blocks)
    XferList copy;                  // same-level ghost exchange (GRANITE_AMR_GHOSTS)
    std::vector<XferList> restrict_;  // into this level from level+1; one list per launch
    unsigned char* d_facemask = nullptr;  // faces left to the zero-gradient fill (REFERENCE)
    GhostSrc* d_src = nullptr;            // one source per ghost cell of the level (GHOSTS)
    long long nsrc = 0;
    std::vector<std::pair<long long, long long>> src_range;  // per block: first item, count
    // the ghost cells the stage stencils read (faces, and edges one cell deep for the
    // mixed derivatives; never corners): the fills of the RK stage buffers
    GhostSrc* d_src_stage = nullptr;
    long long nsrc_stage = 0;
    std::vector<std::pair<long long, long long>> src_range_stage;
    // same-level copies pushed by the stage kernels (push_ok: the level's
    // interiors do not overlap and its stage kernel is the TMA variant): the
    // push boxes, per stage tile its range of them, and the ghost sources
    // without the copies for the fills that follow a pushing stage
    bool push_ok = false;
    std::map<int, std::vector<PushBox>> push_by_src;  // host: the push boxes of each source block
    PushBox* d_push = nullptr;
    int2* d_tile_push = nullptr;
    GhostSrc* d_src_nc = nullptr;
    long long nsrc_nc = 0;
    std::vector<std::pair<long long, long long>> src_range_nc;
    GhostSrc* d_src_stage_nc = nullptr;
    long long nsrc_stage_nc = 0;
    std::vector<std::pair<long long, long long>> src_range_stage_nc;
    // the fill before a step while the pushed copies are current: no copies but
    // those of cells a restriction into the level writes
    GhostSrc* d_src_pre = nullptr;
    long long nsrc_pre = 0;
    std::vector<std::pair<long long, long long>> src_range_pre;
};

// device copy of a host vector (nullptr for an empty one)
template <typename T>
cudaError_t upload_vec(const std::vector<T>& v, T** d, cudaStream_t s) {
    *d = nullptr;
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc(d, v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

long long cells_of(const granite_block_desc& b) {
    return (long long)(b.ncells[0] + 2 * b.nghost) * (b.ncells[1] + 2 * b.nghost) * (b.ncells[2] + 2 * b.nghost);
}

}  // namespace

struct Ctx {
    granite_ccz4_params p{};
    int device = 0;
    int variant = VARIANT_TMA;     // stage-kernel variant (granite_ccz4_set_kernel_variant)
    // TMA configuration per precision and block-size class (granite_ccz4_set_stage_config);
    // forced_cfg >= 0 overrides the table for every block
    int class_cfg[2][GRANITE_STAGE_CLASSES];
    int forced_cfg = -1;
    bool batched = true;           // one launch per level and stage + CUDA graphs (else per block, eager)
    bool matter = false;           // resident matter sources (granite_ccz4_enable_matter)
    double* d_matter = nullptr;    // rho[N] | Si[N][3] | Sij[N][6] | S[N], N = matter_cells (all blocks)
    char* s_diag = nullptr;        // diagnostics scratch (Psi4 sphere points, radii, modes, counts)
    size_t s_diag_bytes = 0;
    long long matter_cells = 0;
    double fp64_chi = 0.0;         // MIXED: tiles with a point of chi below this run the FP64 algebra
    cudaStream_t stream = nullptr;
    // second stream of the per-tile precision: the FP64 pass runs beside the
    // FP32 pass (disjoint tiles), forked from and joined back to `stream`
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::string err;
    long long launches = 0;
    unsigned long long* d_nonfinite = nullptr;
    unsigned int* d_errflag = nullptr;   // set by a TMA stage kernel whose bounded wait gave up
    int test_withhold = 0;               // armed test switch (StageArgs::test_withhold) of the next rk3_step
    bool ghost_push = false;             // GRANITE_AMR_GHOSTS: stage kernels push same-level ghost copies
    bool overlap_passes = false;         // per-tile precision: FP64 pass beside the FP32 pass (second stream)
    // every level's same-level ghost copies of slot 0 equal their sources except
    // where a restriction has rewritten a source cell since (after a
    // GRANITE_AMR_GHOSTS coarse step; cleared by anything else that writes the
    // state), and, while a coarse step is being enqueued, the levels whose
    // fill after a step (or whose pushing stages) made them so in it: their
    // fills before a step copy only the cells of restricted sources
    bool copies_valid = false;
    std::vector<char> step_pushed;
    unsigned long long* d_cmp = nullptr; // granite_ccz4_compare_states results (46 words)
    CUtensorMap* d_tmaps = nullptr;      // TMA variant: per box shape, 3 maps per resident block (slots 0-2)
    CUtensorMap* s_tmap = nullptr;       // TMA variant: map of the stateless single-block input

    // stateless scratch (grow-only)
    double* s_u = nullptr;
    double* s_rhs = nullptr;
    double* s_mat = nullptr;  // rho, Si, Sij, S packed
    size_t s_cells = 0;
    DevBlock* s_desc = nullptr;
    Tile* s_tiles = nullptr;
    int s_tiles_cap = 0;
    double* s_partials = nullptr;
    int s_partials_cap = 0;
    double* s_sum = nullptr;

    // resident hierarchy
    std::vector<granite_block_desc> descs;
    std::vector<DevBlock> hblocks;
    DevBlock* d_blocks = nullptr;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    bool committed = false;
    std::vector<LevelLists> levels;
    std::vector<bool> level_ghosts_valid;
    // AMRHierarchy Level::current_time per level (amr.hpp:108-113): advanced by
    // the level's dt at every step of the level; a level a regrid creates starts
    // at its parent's time (amr.cpp:137-143)
    std::vector<double> level_time;
    std::map<std::tuple<int, int, int, unsigned long long, int>, Graph> graphs;
    // hierarchy transfer lists per AMR mode (built on first use), and graphs
    // of whole subcycled coarse steps keyed by (precision, mode, dt bits)
    std::vector<LevelXfer> xfer[2];
    bool xfer_built[2] = {false, false};
    std::map<std::tuple<int, int, unsigned long long>, Graph> hgraphs;

    // profiler: pending (class, start, stop) event pairs and per-class totals
    bool profiling = false;
    struct Pending {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double prof_ms[GRANITE_KERNEL_CLASSES] = {0, 0, 0, 0};
    long long prof_n[GRANITE_KERNEL_CLASSES] = {0, 0, 0, 0};
};

namespace {

int fail(Ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(Ctx* c, cudaError_t e, const char* where) {
    return fail(c, e == cudaErrorMemoryAllocation ? GRANITE_ERR_NOMEM : GRANITE_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call, where)                                          \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, where);   \
    } while (0)

int check_desc(Ctx* c, const granite_block_desc* b) {
    if (!b) return fail(c, GRANITE_ERR_INVALID, "null block descriptor");
    if (b->nghost != NG)
        return fail(c, GRANITE_ERR_INVALID,
                    "nghost must be 4: the upwind stencil reaches i+-4 (ccz4.cpp:109-152)");
    for (int d = 0; d < 3; ++d) {
        if (b->ncells[d] < NG) return fail(c, GRANITE_ERR_INVALID, "ncells must be >= 4 per axis");
        if (!(b->hi[d] > b->lo[d])) return fail(c, GRANITE_ERR_INVALID, "hi must exceed lo");
    }
    // cell indices within a block are 32-bit in the transfer kernels (2^31 cells
    // would be 378 GB of state, beyond any one GPU)
    if (cells_of(*b) >= (1ll << 31)) return fail(c, GRANITE_ERR_INVALID, "block too large: 2^31 cells or more");
    return GRANITE_OK;
}

DevBlock make_devblock(const granite_block_desc& b, double sigma) {
    DevBlock d{};
    for (int a = 0; a < 3; ++a) d.n[a] = b.ncells[a];
    d.tx = b.ncells[0] + 2 * NG;
    d.ty = b.ncells[1] + 2 * NG;
    d.tz = b.ncells[2] + 2 * NG;
    d.stride = (long long)d.tx * d.ty * d.tz;
    for (int a = 0; a < 3; ++a) {
        d.lo[a] = b.lo[a];
        d.dx[a] = (b.hi[a] - b.lo[a]) / static_cast<double>(b.ncells[a]);  // grid.cpp:20-22
        d.inv12h[a] = 1.0 / (12.0 * d.dx[a]);
        d.inv12h2[a] = 1.0 / (12.0 * d.dx[a] * d.dx[a]);
        d.kocf[a] = sigma / (64.0 * d.dx[a]);
        const double wts[4] = {1.0, -6.0, 15.0, -20.0};
        for (int s = 0; s < 4; ++s) d.kow[a][s] = d.kocf[a] * wts[s];
    }
    d.inv4hh[0] = 1.0 / (4.0 * d.dx[0] * d.dx[1]);
    d.inv4hh[1] = 1.0 / (4.0 * d.dx[0] * d.dx[2]);
    d.inv4hh[2] = 1.0 / (4.0 * d.dx[1] * d.dx[2]);
    d.level = b.level;
    return d;
}

// Tiles of one block. adaptive (global-load stage kernels only): pick the tile
// width w in {32, 16, 8} (128 / w rows) that leaves the fewest idle threads on
// this block's x-y face, preferring the wider tile on ties (longer coalesced rows).
// rem_mapped: the block has tensor maps of its configuration's remainder box.
void tiles_of(int block, const granite_block_desc& b, std::vector<Tile>& out, int variant, bool adaptive = false,
              int cfg = 0, bool rem_mapped = false) {
    int TX, TY, TZ;
    stage_tile_dims(variant, cfg, &TX, &TY, &TZ);
    int w = 0;
    if (adaptive) {
        long long best = -1;
        for (int cand : {32, 16, 8}) {
            const int h = 128 / cand;
            const long long cells = (long long)((b.ncells[0] + cand - 1) / cand) * cand *
                ((b.ncells[1] + h - 1) / h) * h;
            if (best < 0 || cells < best) {
                best = cells;
                w = cand;
            }
        }
        TX = w;
        TY = 128 / w;
        TZ = 1;
    }
    // TMA x-remainder tiles: a block whose x extent is TMA_REM_X more than a
    // multiple of 16 covers its last TMA_REM_X columns with TMA_REM_X x TY x 2 TZ
    // tiles (Tile::w = -TMA_REM_X), each after the full tiles of its rows
    const bool rem = variant == VARIANT_TMA && !adaptive && cfg >= 0 && cfg < NUM_TMA_CFGS && TMA_CFGS[cfg].rem &&
                     rem_mapped && b.ncells[0] % TX == TMA_REM_X;
    const int nx = rem ? b.ncells[0] - TMA_REM_X : b.ncells[0];
    for (int k = 0; k < b.ncells[2]; k += TZ)
        for (int j = 0; j < b.ncells[1]; j += TY) {
            for (int i = 0; i < nx; i += TX) out.push_back(Tile{block, i, j, k, w});
            if (rem && k % (2 * TZ) == 0) out.push_back(Tile{block, nx, j, k, -TMA_REM_X});
        }
}

// Block-size class of a block for the per-class stage configuration: the class
// edge (GRANITE_STAGE_CLASS_EDGES) nearest, on a log scale, to the cube root of
// its interior volume.
int stage_class_of(const granite_block_desc& b) {
    static const int edges[GRANITE_STAGE_CLASSES] = {GRANITE_STAGE_CLASS_EDGES};
    const double e = std::cbrt((double)b.ncells[0] * b.ncells[1] * b.ncells[2]);
    int best = 0;
    for (int q = 1; q < GRANITE_STAGE_CLASSES; ++q)
        if (std::fabs(std::log(e / edges[q])) < std::fabs(std::log(e / edges[best]))) best = q;
    return best;
}

long long ghost_count(const granite_block_desc& b) {
    return cells_of(b) - (long long)b.ncells[0] * b.ncells[1] * b.ncells[2];
}

void ghost_chunks_of(int block, const granite_block_desc& b, std::vector<GhostItem>& out) {
    const long long n = ghost_count(b);
    for (long long r = 0; r < n; r += 256) out.push_back(GhostItem{block, (int)r});
}

// TMA configuration of a block for precision index pr (0 FP64, 1 MIXED).
int block_cfg(const Ctx* c, int pr, const granite_block_desc& b) {
    if (c->forced_cfg >= 0) return c->forced_cfg;
    return c->class_cfg[pr][stage_class_of(b)];
}

StageArgs base_args(const Ctx* c) {
    StageArgs a{};
    a.chi_c = c->p.chi_blend_center;
    a.chi_w = c->p.chi_blend_width;
    a.kappa1 = c->p.kappa1;
    a.kappa2 = c->p.kappa2;
    a.eta = c->p.eta;
    a.nonfinite = c->d_nonfinite;
    a.tmaps = c->d_tmaps;
    a.errflag = c->d_errflag;
    if (c->d_matter) {  // resident matter: the context-wide arrays, block b at cell offset moff
        const long long N = c->matter_cells;
        a.rho = c->d_matter;
        a.Si = c->d_matter + N;
        a.Sij = c->d_matter + 4 * N;
        a.S = c->d_matter + 10 * N;
    }
    return a;
}

// Grow the stateless scratch to hold one block (+ matter sources).
int ensure_scratch(Ctx* c, size_t cells, int ntiles) {
    if (cells > c->s_cells) {
        cudaFree(c->s_u);
        cudaFree(c->s_rhs);
        cudaFree(c->s_mat);
        c->s_u = c->s_rhs = c->s_mat = nullptr;
        c->s_cells = 0;
        CK(cudaMalloc(&c->s_u, cells * NV * sizeof(double)), "cudaMalloc(scratch u)");
        CK(cudaMalloc(&c->s_rhs, cells * NV * sizeof(double)), "cudaMalloc(scratch rhs)");
        CK(cudaMalloc(&c->s_mat, cells * NPRIM * sizeof(double)), "cudaMalloc(scratch matter)");
        c->s_cells = cells;
    }
    if (ntiles > c->s_tiles_cap) {
        cudaFree(c->s_tiles);
        c->s_tiles = nullptr;
        CK(cudaMalloc(&c->s_tiles, ntiles * sizeof(Tile)), "cudaMalloc(tiles)");
        c->s_tiles_cap = ntiles;
    }
    if (ntiles > c->s_partials_cap) {
        cudaFree(c->s_partials);
        c->s_partials = nullptr;
        CK(cudaMalloc(&c->s_partials, 2 * (size_t)ntiles * sizeof(double)), "cudaMalloc(partials)");
        c->s_partials_cap = ntiles;
    }
    return GRANITE_OK;
}

// Stage one block into the stateless scratch: descriptor + tile list (+ the
// tensor map of its buffer for the TMA variant). *used = the variant the
// tiles were built for (TMA falls back to GLOBAL for a buffer it cannot map).
int stage_single(Ctx* c, const granite_block_desc* b, double* u_dev, int* ntiles, cudaStream_t s, int variant,
                 int* used = nullptr) {
    int r = ensure_scratch(c, (size_t)cells_of(*b), 1);
    if (r) return r;
    DevBlock d = make_devblock(*b, c->p.ko_sigma);
    d.buf[0] = u_dev ? u_dev : c->s_u;
    if (variant == VARIANT_TMA) {  // configuration 0 (the one with the store epilogue)
        CUtensorMap m;
        if (encode_block_tmap(&m, d.buf[0], d, TMA_CFGS[0].tz))
            CK(cudaMemcpyAsync(c->s_tmap, &m, sizeof(m), cudaMemcpyHostToDevice, s), "upload tensor map");
        else
            variant = VARIANT_GLOBAL;
    }
    if (used) *used = variant;
    std::vector<Tile> t;
    tiles_of(0, *b, t, variant);
    if ((r = ensure_scratch(c, (size_t)cells_of(*b), (int)t.size()))) return r;
    CK(cudaMemcpyAsync(c->s_desc, &d, sizeof(d), cudaMemcpyHostToDevice, s), "upload block descriptor");
    CK(cudaMemcpyAsync(c->s_tiles, t.data(), t.size() * sizeof(Tile), cudaMemcpyHostToDevice, s), "upload tiles");
    *ntiles = (int)t.size();
    return GRANITE_OK;
}

int check_precision(Ctx* c, int precision) {
    if (precision != GRANITE_PRECISION_FP64 && precision != GRANITE_PRECISION_MIXED)
        return fail(c, GRANITE_ERR_INVALID, "precision must be GRANITE_PRECISION_FP64 or _MIXED");
    return GRANITE_OK;
}

cudaEvent_t take_event(Ctx* c) {
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Run one launch; when profiling, bracket it with events on the context stream.
template <typename F>
cudaError_t timed(Ctx* c, int cls, F&& launch) {
    if (!c->profiling) return launch();
    cudaEvent_t a = take_event(c), b = take_event(c);
    cudaEventRecord(a, c->stream);
    cudaError_t e = launch();
    cudaEventRecord(b, c->stream);
    c->pending.push_back({cls, a, b});
    return e;
}

cudaError_t drain_profile(Ctx* c) {
    if (c->pending.empty()) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return e;
    for (auto& p : c->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.a, p.b);
        c->prof_ms[p.cls] += ms;
        c->prof_n[p.cls] += 1;
        c->event_pool.push_back(p.a);
        c->event_pool.push_back(p.b);
    }
    c->pending.clear();
    return cudaSuccess;
}

}  // namespace

extern "C" {

int granite_ccz4_set_profiling(void* h, int enabled) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    CK(drain_profile(c), "profile drain");
    c->profiling = enabled != 0;
    return GRANITE_OK;
}

int granite_ccz4_profile_reset(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    CK(drain_profile(c), "profile drain");
    for (int k = 0; k < GRANITE_KERNEL_CLASSES; ++k) {
        c->prof_ms[k] = 0.0;
        c->prof_n[k] = 0;
    }
    return GRANITE_OK;
}

int granite_ccz4_profile_get(void* h, int cls, double* ms, long long* n) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c || !ms || !n || cls < 0 || cls >= GRANITE_KERNEL_CLASSES) return GRANITE_ERR_INVALID;
    CK(drain_profile(c), "profile drain");
    *ms = c->prof_ms[cls];
    *n = c->prof_n[cls];
    return GRANITE_OK;
}

int granite_ccz4_set_batching(void* h, int batched) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    CK(drain_profile(c), "profile drain");
    c->batched = batched != 0;
    return GRANITE_OK;
}

int granite_ccz4_set_kernel_variant(void* h, int variant) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (variant < 0 || variant >= NUM_VARIANTS) return fail(c, GRANITE_ERR_INVALID, "unknown kernel variant");
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "set the kernel variant before commit");
    c->variant = variant;
    return GRANITE_OK;
}

int granite_ccz4_set_stage_config(void* h, int precision, int cls, int cfg) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "set stage configurations before commit");
    if (precision != GRANITE_PRECISION_FP64 && precision != GRANITE_PRECISION_MIXED)
        return fail(c, GRANITE_ERR_INVALID, "precision must be GRANITE_PRECISION_FP64 or _MIXED");
    if (cls < -1 || cls >= GRANITE_STAGE_CLASSES) return fail(c, GRANITE_ERR_INVALID, "unknown block-size class");
    if (cfg < -1 || cfg >= NUM_TMA_CFGS) return fail(c, GRANITE_ERR_INVALID, "unknown stage configuration");
    const int pr = precision == GRANITE_PRECISION_MIXED ? 1 : 0;
    for (int q = 0; q < GRANITE_STAGE_CLASSES; ++q)
        if (cls < 0 || q == cls) c->class_cfg[pr][q] = cfg < 0 ? DEFAULT_CLASS_CFG[pr][q] : cfg;
    return GRANITE_OK;
}

int granite_ccz4_get_stage_config(const void* h, int precision, int cls, int* cfg) {
    const Ctx* c = static_cast<const Ctx*>(h);
    if (!c || !cfg || cls < 0 || cls >= GRANITE_STAGE_CLASSES) return GRANITE_ERR_INVALID;
    if (precision != GRANITE_PRECISION_FP64 && precision != GRANITE_PRECISION_MIXED) return GRANITE_ERR_INVALID;
    *cfg = c->forced_cfg >= 0 ? c->forced_cfg : c->class_cfg[precision == GRANITE_PRECISION_MIXED ? 1 : 0][cls];
    return GRANITE_OK;
}

int granite_ccz4_force_stage_config(void* h, int cfg) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "set stage configurations before commit");
    if (cfg < -1 || cfg >= NUM_TMA_CFGS) return fail(c, GRANITE_ERR_INVALID, "unknown stage configuration");
    c->forced_cfg = cfg;
    return GRANITE_OK;
}

int granite_ccz4_stage_config_info(int cfg, int* tile_z, int* ring_slots, int* shared_input, int* shared_hessian) {
    if (cfg < 0 || cfg >= NUM_TMA_CFGS) return GRANITE_ERR_INVALID;
    if (tile_z) *tile_z = TMA_CFGS[cfg].tz;
    if (ring_slots) *ring_slots = TMA_CFGS[cfg].nbuf;
    if (shared_input) *shared_input = TMA_CFGS[cfg].tin;
    if (shared_hessian) *shared_hessian = TMA_CFGS[cfg].hs;
    return GRANITE_OK;
}

int granite_ccz4_stage_config_schedule(int cfg, int* warp_specialized, int* ctas_per_sm, int* items_per_barrier,
                                       int* x_remainder_tiles) {
    if (cfg < 0 || cfg >= NUM_TMA_CFGS) return GRANITE_ERR_INVALID;
    if (warp_specialized) *warp_specialized = TMA_CFGS[cfg].ws;
    if (ctas_per_sm) *ctas_per_sm = TMA_CFGS[cfg].minb;
    if (items_per_barrier) *items_per_barrier = TMA_CFGS[cfg].bar;
    if (x_remainder_tiles) *x_remainder_tiles = TMA_CFGS[cfg].rem;
    return GRANITE_OK;
}
static_assert(GRANITE_STAGE_CONFIGS == NUM_TMA_CFGS, "the header's configuration count");

int granite_ccz4_block_stage_class(const granite_block_desc* b, int* cls) {
    if (!b || !cls) return GRANITE_ERR_INVALID;
    for (int d = 0; d < 3; ++d)
        if (b->ncells[d] <= 0) return GRANITE_ERR_INVALID;
    *cls = stage_class_of(*b);
    return GRANITE_OK;
}

int granite_ccz4_set_fp64_chi_threshold(void* h, double chi) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!(chi >= 0.0) || !std::isfinite(chi)) return fail(c, GRANITE_ERR_INVALID, "threshold must be finite and >= 0");
    if (chi == c->fp64_chi) return GRANITE_OK;
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    // cached step graphs hold the old launch sequence
    for (auto& kv : c->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto& kv : c->hgraphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->graphs.clear();
    c->hgraphs.clear();
    c->fp64_chi = chi;
    return GRANITE_OK;
}

int granite_ccz4_get_fp64_chi_threshold(const void* h, double* chi) {
    const Ctx* c = static_cast<const Ctx*>(h);
    if (!c || !chi) return GRANITE_ERR_INVALID;
    *chi = c->fp64_chi;
    return GRANITE_OK;
}

int granite_ccz4_get_kernel_variant(const void* h, int* variant) {
    const Ctx* c = static_cast<const Ctx*>(h);
    if (!c || !variant) return GRANITE_ERR_INVALID;
    *variant = c->variant;
    return GRANITE_OK;
}

int granite_ccz4_get_stream(void* h, void** stream) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c || !stream) return GRANITE_ERR_INVALID;
    *stream = c->stream;
    return GRANITE_OK;
}

int granite_ccz4_abi_version(void) { return GRANITE_CCZ4_ABI_VERSION; }

void granite_ccz4_default_params(granite_ccz4_params* p) {
    if (!p) return;
    p->kappa1 = 0.02;
    p->kappa2 = 0.0;
    p->eta = 2.0;
    p->ko_sigma = 0.1;
    p->chi_blend_center = 0.05;
    p->chi_blend_width = 0.02;
    p->fd_order = 4;
    p->device = 0;
}

int granite_ccz4_create(const granite_ccz4_params* p, void** out) {
    if (!p || !out) return GRANITE_ERR_INVALID;
    *out = nullptr;
    if (p->fd_order != 4) return GRANITE_ERR_UNSUPPORTED;
    if (!(p->chi_blend_width != 0.0)) return GRANITE_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GRANITE_ERR_NO_DEVICE;
    }
    if (p->device < 0 || p->device >= ndev) return GRANITE_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, p->device) != cudaSuccess) return GRANITE_ERR_NO_DEVICE;
    if (prop.major != 10) return GRANITE_ERR_NO_DEVICE;  // kernels are built for sm_100a only
    Ctx* c = new Ctx();
    std::memcpy(c->class_cfg, DEFAULT_CLASS_CFG, sizeof(c->class_cfg));
    c->p = *p;
    c->device = p->device;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = configure_stage_kernels();
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_nonfinite, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(c->d_nonfinite, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_errflag, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(c->d_errflag, 0, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&c->s_tmap, sizeof(CUtensorMap));
    if (e == cudaSuccess) e = cudaMalloc(&c->s_desc, sizeof(DevBlock));
    if (e == cudaSuccess) e = cudaMalloc(&c->s_sum, 2 * sizeof(double));
    if (e != cudaSuccess) {
        granite_ccz4_destroy(c);
        return e == cudaErrorMemoryAllocation ? GRANITE_ERR_NOMEM : GRANITE_ERR_CUDA;
    }
    *out = c;
    return GRANITE_OK;
}

static void release_lists(Ctx* c);

int granite_ccz4_destroy(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& p : c->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    release_lists(c);
    cudaFree(c->arena);
    cudaFree(c->s_u);
    cudaFree(c->s_rhs);
    cudaFree(c->s_mat);
    cudaFree(c->d_matter);
    cudaFree(c->s_diag);
    cudaFree(c->s_desc);
    cudaFree(c->s_tiles);
    cudaFree(c->s_partials);
    cudaFree(c->s_sum);
    cudaFree(c->d_nonfinite);
    cudaFree(c->d_errflag);
    cudaFree(c->d_cmp);
    cudaFree(c->s_tmap);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    delete c;
    return GRANITE_OK;
}

int granite_ccz4_last_error(const void* h, char* buf, size_t len) {
    const Ctx* c = static_cast<const Ctx*>(h);
    if (!buf || len == 0) return GRANITE_ERR_INVALID;
    const std::string& m = c ? c->err : std::string("null context");
    std::snprintf(buf, len, "%s", m.c_str());
    return GRANITE_OK;
}

// Report (and clear) a bounded wait of the TMA stage kernel that gave up.
static int check_errflag(Ctx* c) {
    unsigned int v = 0;
    CK(cudaMemcpyAsync(&v, c->d_errflag, sizeof(v), cudaMemcpyDeviceToHost, c->stream), "read error flag");
    CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (v) {
        CK(cudaMemsetAsync(c->d_errflag, 0, sizeof(v), c->stream), "reset error flag");
        CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        return fail(c, GRANITE_ERR_CUDA, "stage kernel: a tensor-map tile load did not complete within its wait limit");
    }
    return GRANITE_OK;
}

int granite_ccz4_set_pass_overlap(void* h, int on) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    c->overlap_passes = on != 0;
    for (auto& kv : c->hgraphs)  // captured steps bake the choice in
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->hgraphs.clear();
    for (auto& kv : c->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->graphs.clear();
    return GRANITE_OK;
}

int granite_ccz4_set_ghost_push(void* h, int on) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    c->ghost_push = on != 0;
    c->copies_valid = false;
    for (auto& kv : c->hgraphs)  // captured steps bake the choice in
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->hgraphs.clear();
    return GRANITE_OK;
}

int granite_ccz4_test_withhold_tile_load(void* h, int item) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (item < 0) return fail(c, GRANITE_ERR_INVALID, "item must be >= 0");
    if (c->variant != VARIANT_TMA) return fail(c, GRANITE_ERR_INVALID, "the switch acts on the TMA stage kernel only");
    c->test_withhold = item + 1;
    return GRANITE_OK;
}

int granite_ccz4_sync(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    return check_errflag(c);
}

int granite_ccz4_launch_count(const void* h, long long* n) {
    const Ctx* c = static_cast<const Ctx*>(h);
    if (!c || !n) return GRANITE_ERR_INVALID;
    *n = c->launches;
    return GRANITE_OK;
}

int granite_ccz4_nonfinite_count(void* h, long long* n) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c || !n) return GRANITE_ERR_INVALID;
    unsigned long long v = 0;
    CK(cudaMemcpyAsync(&v, c->d_nonfinite, sizeof(v), cudaMemcpyDeviceToHost, c->stream), "read nonfinite");
    CK(cudaMemsetAsync(c->d_nonfinite, 0, sizeof(v), c->stream), "reset nonfinite");
    CK(cudaStreamSynchronize(c->stream), "sync");
    *n = (long long)v;
    return GRANITE_OK;
}

// ---------------------------------------------------------------------------
// stateless operators
// ---------------------------------------------------------------------------

int granite_ccz4_compute_rhs_device(void* h, const granite_block_desc* b, const double* u_dev, double* rhs_dev,
                                    const double* rho, const double* Si, const double* Sij, const double* S,
                                    int precision, void* stream) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if ((r = check_precision(c, precision))) return r;
    if (!u_dev || !rhs_dev) return fail(c, GRANITE_ERR_INVALID, "null device buffer");
    const int nm = (rho != nullptr) + (Si != nullptr) + (Sij != nullptr) + (S != nullptr);
    if (nm != 0 && nm != 4) return fail(c, GRANITE_ERR_INVALID, "matter sources: pass all four or none");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    int nt = 0, variant = VARIANT_GLOBAL;
    if ((r = stage_single(c, b, const_cast<double*>(u_dev), &nt, s, c->variant, &variant))) return r;
    StageArgs a = base_args(c);
    a.in_sel = 0;
    a.rhs = rhs_dev;
    a.rho = rho;
    a.Si = Si;
    a.Sij = Sij;
    a.S = S;
    a.tmaps = c->s_tmap;  // block 0, slot 0
    CK(launch_stage(variant, 0, precision, EPI_STORE, c->s_desc, c->s_tiles, nt, a, s), "launch RHS");
    c->launches += 1;
    return GRANITE_OK;
}

int granite_ccz4_matter_sources_device(void* h, const granite_block_desc* b, const double* prim_dev, double* rho_dev,
                                      double* Si_dev, double* Sij_dev, double* S_dev, void* stream) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!prim_dev || !rho_dev || !Si_dev || !Sij_dev || !S_dev) return fail(c, GRANITE_ERR_INVALID, "null buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const MatterOut o{rho_dev, Si_dev, Sij_dev, S_dev, 3, 1, 6, 1};
    CK(launch_matter_sources(make_devblock(*b, c->p.ko_sigma), prim_dev, o,
                             stream ? static_cast<cudaStream_t>(stream) : c->stream),
       "launch matter sources");
    c->launches += 1;
    return GRANITE_OK;
}

int granite_ccz4_matter_sources_host(void* h, const granite_block_desc* b, const double* prim, double* rho,
                                    double* Si, double* Sij, double* S) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!prim || !rho || !Si || !Sij || !S) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)cells_of(*b);
    if ((r = ensure_scratch(c, N, 1))) return r;
    cudaStream_t s = c->stream;
    double* m = c->s_mat;  // rho | Si (3N) | Sij (6N) | S: the caller's arrays, in/out
    CK(cudaMemcpyAsync(c->s_u, prim, N * NPRIM * sizeof(double), cudaMemcpyHostToDevice, s), "H2D prim");
    CK(cudaMemcpyAsync(m, rho, N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D rho");
    CK(cudaMemcpyAsync(m + N, Si, 3 * N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D Si");
    CK(cudaMemcpyAsync(m + 4 * N, Sij, 6 * N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D Sij");
    CK(cudaMemcpyAsync(m + 10 * N, S, N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D S");
    r = granite_ccz4_matter_sources_device(c, b, c->s_u, m, m + N, m + 4 * N, m + 10 * N, s);
    if (r) return r;
    CK(cudaMemcpyAsync(rho, m, N * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H rho");
    CK(cudaMemcpyAsync(Si, m + N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H Si");
    CK(cudaMemcpyAsync(Sij, m + 4 * N, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H Sij");
    CK(cudaMemcpyAsync(S, m + 10 * N, N * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H S");
    CK(cudaStreamSynchronize(s), "sync");
    return GRANITE_OK;
}

int granite_ccz4_compute_rhs_host(void* h, const granite_block_desc* b, const double* u, double* rhs,
                                  const double* rho, const double* Si, const double* Sij, const double* S,
                                  int precision) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!u || !rhs) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    const int nm = (rho != nullptr) + (Si != nullptr) + (Sij != nullptr) + (S != nullptr);
    if (nm != 0 && nm != 4) return fail(c, GRANITE_ERR_INVALID, "matter sources: pass all four or none");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)cells_of(*b);
    std::vector<Tile> t;
    tiles_of(0, *b, t, VARIANT_GLOBAL);
    if ((r = ensure_scratch(c, N, (int)t.size()))) return r;
    cudaStream_t s = c->stream;
    CK(cudaMemcpyAsync(c->s_u, u, N * NV * sizeof(double), cudaMemcpyHostToDevice, s), "H2D u");
    CK(cudaMemcpyAsync(c->s_rhs, rhs, N * NV * sizeof(double), cudaMemcpyHostToDevice, s), "H2D rhs");
    const double *drho = nullptr, *dSi = nullptr, *dSij = nullptr, *dS = nullptr;
    if (nm == 4) {
        double* m = c->s_mat;
        CK(cudaMemcpyAsync(m, rho, N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D rho");
        CK(cudaMemcpyAsync(m + N, Si, 3 * N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D Si");
        CK(cudaMemcpyAsync(m + 4 * N, Sij, 6 * N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D Sij");
        CK(cudaMemcpyAsync(m + 10 * N, S, N * sizeof(double), cudaMemcpyHostToDevice, s), "H2D S");
        drho = m;
        dSi = m + N;
        dSij = m + 4 * N;
        dS = m + 10 * N;
    }
    r = granite_ccz4_compute_rhs_device(c, b, c->s_u, c->s_rhs, drho, dSi, dSij, dS, precision, s);
    if (r) return r;
    CK(cudaMemcpyAsync(rhs, c->s_rhs, N * NV * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H rhs");
    CK(cudaStreamSynchronize(s), "sync");
    return check_errflag(c);
}

int granite_ccz4_apply_dissipation_host(void* h, const granite_block_desc* b, const double* u, double* rhs) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!u || !rhs) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    if (!(c->p.ko_sigma > 0.0)) return GRANITE_OK;  // ccz4.cpp:873
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)cells_of(*b);
    cudaStream_t s = c->stream;
    int nt = 0;
    if ((r = stage_single(c, b, nullptr, &nt, s, VARIANT_GLOBAL))) return r;
    CK(cudaMemcpyAsync(c->s_u, u, N * NV * sizeof(double), cudaMemcpyHostToDevice, s), "H2D u");
    CK(cudaMemcpyAsync(c->s_rhs, rhs, N * NV * sizeof(double), cudaMemcpyHostToDevice, s), "H2D rhs");
    CK(launch_dissipation(c->s_desc, 0, c->s_rhs, nt, c->s_tiles, s), "launch KO");
    c->launches += 1;
    CK(cudaMemcpyAsync(rhs, c->s_rhs, N * NV * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H rhs");
    CK(cudaStreamSynchronize(s), "sync");
    return GRANITE_OK;
}

int granite_ccz4_compute_constraints_host(void* h, const granite_block_desc* b, const double* u, double* ham,
                                          double* mom) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!u || !ham || !mom) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)cells_of(*b);
    cudaStream_t s = c->stream;
    int nt = 0;
    if ((r = stage_single(c, b, nullptr, &nt, s, VARIANT_GLOBAL))) return r;
    CK(cudaMemcpyAsync(c->s_u, u, N * NV * sizeof(double), cudaMemcpyHostToDevice, s), "H2D u");
    // ham in s_rhs[0:N], mom in s_rhs[N:4N]; ghosts zero (ccz4.cpp:945-946)
    CK(cudaMemsetAsync(c->s_rhs, 0, 4 * N * sizeof(double), s), "memset");
    CK(launch_constraints(c->s_desc, c->s_tiles, nt, 0, c->s_rhs, c->s_rhs + N, nullptr, s), "launch constraints");
    c->launches += 1;
    CK(cudaMemcpyAsync(ham, c->s_rhs, N * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H ham");
    CK(cudaMemcpyAsync(mom, c->s_rhs + N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H mom");
    CK(cudaStreamSynchronize(s), "sync");
    return GRANITE_OK;
}

// ---------------------------------------------------------------------------
// resident blocks
// ---------------------------------------------------------------------------

int granite_ccz4_add_block(void* h, const granite_block_desc* b, int* idx) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "add_block after commit");
    int r = check_desc(c, b);
    if (r) return r;
    if (b->level < 0 || b->level > 31) return fail(c, GRANITE_ERR_INVALID, "level out of range");
    c->descs.push_back(*b);
    if (idx) *idx = (int)c->descs.size() - 1;
    return GRANITE_OK;
}

int granite_ccz4_num_blocks(const void* h) {
    const Ctx* c = static_cast<const Ctx*>(h);
    return c ? (int)c->descs.size() : GRANITE_ERR_INVALID;
}

int granite_ccz4_arena_bytes(const void* h, size_t* bytes) {
    const Ctx* c = static_cast<const Ctx*>(h);
    if (!c || !bytes) return GRANITE_ERR_INVALID;
    *bytes = c->arena_bytes;
    return GRANITE_OK;
}

namespace {
cudaError_t upload_xfer(const std::vector<XferBox>& boxes, XferList& out, cudaStream_t s);
}

// Arena layout of a block list: 3 buffers per block, each 256-byte aligned.
// Block i's cells start at cell offset moff in the matter arrays (block order).
static int alloc_arena(Ctx* c, const std::vector<granite_block_desc>& descs, char** arena, size_t* bytes,
                       std::vector<DevBlock>& hb) {
    std::vector<size_t> off(descs.size());
    size_t total = 0;
    for (size_t i = 0; i < descs.size(); ++i) {
        off[i] = total;
        const size_t one = ((size_t)cells_of(descs[i]) * NV * sizeof(double) + 255) / 256 * 256;
        total += 3 * one;
    }
    CK(cudaMalloc(arena, total), "cudaMalloc(arena)");
    *bytes = total;
    hb.resize(descs.size());
    long long moff = 0;
    for (size_t i = 0; i < descs.size(); ++i) {
        DevBlock d = make_devblock(descs[i], c->p.ko_sigma);
        const size_t one = ((size_t)cells_of(descs[i]) * NV * sizeof(double) + 255) / 256 * 256;
        for (int sl = 0; sl < 3; ++sl) d.buf[sl] = reinterpret_cast<double*>(*arena + off[i] + sl * one);
        d.moff = c->matter ? (int)moff : 0;  // the total is checked against INT_MAX when matter is on
        moff += cells_of(descs[i]);
        hb[i] = d;
    }
    return GRANITE_OK;
}

// Resident matter arrays for n cells (zero = vacuum); the first `keep` cells of
// each of the four arrays are copied from the current ones.
static int realloc_matter(Ctx* c, long long n, long long keep) {
    if (n > INT_MAX) return fail(c, GRANITE_ERR_UNSUPPORTED, "resident matter: more than 2^31 cells in all blocks");
    double* m = nullptr;
    CK(cudaMalloc(&m, (size_t)n * NPRIM * sizeof(double)), "cudaMalloc(matter)");
    cudaError_t e = cudaMemsetAsync(m, 0, (size_t)n * NPRIM * sizeof(double), c->stream);
    const long long N = c->matter_cells;
    const int width[4] = {1, 3, 6, 1}, at[4] = {0, 1, 4, 10};  // rho, Si, Sij, S
    for (int q = 0; q < 4 && e == cudaSuccess && keep > 0; ++q)
        e = cudaMemcpyAsync(m + at[q] * n, c->d_matter + at[q] * N, (size_t)keep * width[q] * sizeof(double),
                            cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaFree(m);
        return cuda_fail(c, e, "matter arrays");
    }
    cudaFree(c->d_matter);
    c->d_matter = m;
    c->matter_cells = n;
    return GRANITE_OK;
}

static long long total_cells(const std::vector<granite_block_desc>& descs) {
    long long n = 0;
    for (const auto& d : descs) n += cells_of(d);
    return n;
}

// Everything derived from the block list (not the arena): block table, tensor
// maps, per-level work-lists, transfer lists and the cached step graphs.
static void release_lists(Ctx* c) {
    for (auto& kv : c->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto& kv : c->hgraphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    c->graphs.clear();
    c->hgraphs.clear();
    for (auto& L : c->levels) {
        cudaFree(L.d_tiles);
        cudaFree(L.d_flags);
        cudaFree(L.d_mtiles);
        cudaFree(L.d_ghost);
    }
    c->levels.clear();
    for (int m = 0; m < 2; ++m) {
        for (auto& X : c->xfer[m]) {
            free_xfer(X.prolong);
            free_xfer(X.copy);
            for (auto& r : X.restrict_) free_xfer(r);
            cudaFree(X.d_facemask);
            cudaFree(X.d_src);
            cudaFree(X.d_src_stage);
            cudaFree(X.d_push);
            cudaFree(X.d_tile_push);
            cudaFree(X.d_src_nc);
            cudaFree(X.d_src_stage_nc);
            cudaFree(X.d_src_pre);
        }
        c->xfer[m].clear();
        c->xfer_built[m] = false;
    }
    cudaFree(c->d_blocks);
    c->d_blocks = nullptr;
    cudaFree(c->d_tmaps);
    c->d_tmaps = nullptr;
}

// Block table, tensor maps and per-level work-lists of c->descs / c->hblocks.
static int build_lists(Ctx* c) {
    CK(upload_vec(c->hblocks, &c->d_blocks, c->stream), "upload block table");
    int maxlev = 0;
    for (const auto& d : c->descs) maxlev = std::max(maxlev, d.level);
    // TMA variant: one tensor map per (box shape, block, slot); a block that
    // cannot be mapped in the tile shapes (tz = 4 and 2) sends its whole level
    // to the global-load kernel; a block without the tz = 8 shape (less than 8
    // cells deep) only goes without the remainder tiles of tz = 4 configurations
    const size_t nb = c->descs.size();
    std::vector<char> mapped(nb, 0);
    std::vector<std::array<char, TMA_SHAPES>> shape_ok(nb);
    if (c->variant == VARIANT_TMA) {
        std::vector<CUtensorMap> maps(TMA_SHAPES * 3 * nb);
        for (size_t i = 0; i < nb; ++i) {
            for (int sh = 0; sh < TMA_SHAPES; ++sh) {
                bool ok = true;
                for (int sl = 0; sl < 3; ++sl)
                    ok = ok && encode_block_tmap(&maps[(sh * nb + i) * 3 + sl], c->hblocks[i].buf[sl], c->hblocks[i],
                                                 TMA_SHAPE_TZ[sh]);
                shape_ok[i][sh] = ok;
            }
            mapped[i] = shape_ok[i][tma_shape_for_tz(4)] && shape_ok[i][tma_shape_for_tz(2)];
        }
        CK(upload_vec(maps, &c->d_tmaps, c->stream), "upload tensor maps");
    }
    c->levels.assign(maxlev + 1, LevelLists());
    c->level_ghosts_valid.assign(maxlev + 1, false);
    for (int L = 0; L <= maxlev; ++L) {
        std::vector<Tile> tiles, mtiles;
        std::vector<GhostItem> ghosts;
        LevelLists& ll = c->levels[L];
        ll.variant = c->variant;
        for (size_t i = 0; i < c->descs.size(); ++i)
            if (c->descs[i].level == L && c->variant == VARIANT_TMA && !mapped[i]) ll.variant = VARIANT_GLOBAL;
        for (size_t i = 0; i < c->descs.size(); ++i)
            if (c->descs[i].level == L) ll.blocks.push_back((int)i);
        // per precision: stage tiles grouped by configuration (one launch per
        // group), each block's tiles contiguous
        for (int pr = 0; pr < 2; ++pr) {
            for (int i : ll.blocks) ll.block_cfg[pr].push_back(ll.variant == VARIANT_TMA ? block_cfg(c, pr, c->descs[i]) : 0);
            ll.tile_range[pr].assign(ll.blocks.size(), {0, 0});
            for (int cfg = 0; cfg < NUM_TMA_CFGS; ++cfg) {
                const int g0 = (int)tiles.size();
                for (size_t q = 0; q < ll.blocks.size(); ++q) {
                    if (ll.block_cfg[pr][q] != cfg) continue;
                    const int t0 = (int)tiles.size();
                    const int rs = ll.variant == VARIANT_TMA ? tma_rem_shape_of(cfg) : -1;
                    tiles_of(ll.blocks[q], c->descs[ll.blocks[q]], tiles, ll.variant, adaptive_tiles(ll.variant), cfg,
                             rs >= 0 && shape_ok[ll.blocks[q]][rs]);
                    ll.tile_range[pr][q] = {t0, (int)tiles.size() - t0};
                }
                if ((int)tiles.size() > g0) ll.groups[pr].push_back({cfg, g0, (int)tiles.size() - g0});
            }
        }
        for (size_t q = 0; q < ll.blocks.size(); ++q) {
            const int i = ll.blocks[q];
            const int g0 = (int)ghosts.size();
            tiles_of(i, c->descs[i], mtiles, VARIANT_GLOBAL);
            ghost_chunks_of(i, c->descs[i], ghosts);
            ll.ghost_range.push_back({g0, (int)ghosts.size() - g0});
            ll.interior_points += (long long)c->descs[i].ncells[0] * c->descs[i].ncells[1] * c->descs[i].ncells[2];
        }
        CK(upload_vec(tiles, &ll.d_tiles, c->stream), "upload tiles");
        ll.h_tiles = tiles;
        CK(upload_vec(mtiles, &ll.d_mtiles, c->stream), "upload monitor tiles");
        ll.nmtiles = (int)mtiles.size();
        CK(upload_vec(ghosts, &ll.d_ghost, c->stream), "upload ghost chunks");
        ll.ntiles = (int)tiles.size();
        CK(cudaMalloc(&ll.d_flags, std::max<size_t>(1, ll.ntiles)), "cudaMalloc(tile precision flags)");
        ll.nghost = (int)ghosts.size();
    }
    int maxt = 0;
    for (auto& L : c->levels) maxt = std::max(maxt, std::max(L.ntiles, L.nmtiles));
    return ensure_scratch(c, 1, std::max(1, maxt));
}

int granite_ccz4_commit(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "already committed");
    if (c->descs.empty()) return fail(c, GRANITE_ERR_INVALID, "no blocks");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    int r = alloc_arena(c, c->descs, &c->arena, &c->arena_bytes, c->hblocks);
    if (r) return r;
    CK(cudaMemsetAsync(c->arena, 0, c->arena_bytes, c->stream), "memset arena");
    if (c->matter && (r = realloc_matter(c, total_cells(c->descs), 0))) return r;
    if ((r = build_lists(c))) return r;
    c->level_time.assign(c->levels.size(), 0.0);
    c->committed = true;
    return GRANITE_OK;
}

int granite_ccz4_enable_matter(void* h, int on) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "enable matter before commit");
    c->matter = on != 0;
    return GRANITE_OK;
}

int granite_ccz4_set_primitives_device(void* h, int i, const double* prim_dev) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed || !c->matter) return fail(c, GRANITE_ERR_INVALID, "enable matter and commit first");
    if (i < 0 || i >= (int)c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "block index out of range");
    if (!prim_dev) return fail(c, GRANITE_ERR_INVALID, "null buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const DevBlock& d = c->hblocks[i];
    double* m = c->d_matter;
    const long long N = c->matter_cells, o0 = d.moff;
    const MatterOut o{m + o0, m + N + 3 * o0, m + 4 * N + 6 * o0, m + 10 * N + o0, 3, 1, 6, 1};
    CK(launch_matter_sources(d, prim_dev, o, c->stream), "launch matter sources");
    c->launches += 1;
    return GRANITE_OK;
}

int granite_ccz4_upload_primitives(void* h, int i, const double* prim) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed || !c->matter) return fail(c, GRANITE_ERR_INVALID, "enable matter and commit first");
    if (i < 0 || i >= (int)c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "block index out of range");
    if (!prim) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)c->hblocks[i].stride;
    int r = ensure_scratch(c, N, 1);
    if (r) return r;
    CK(cudaMemcpyAsync(c->s_u, prim, N * NPRIM * sizeof(double), cudaMemcpyHostToDevice, c->stream), "H2D prim");
    return granite_ccz4_set_primitives_device(c, i, c->s_u);
}

int granite_ccz4_tag_count(void* h, int level, int var, double threshold, long long* count) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c || !count) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before tagging");
    if (level < 0 || level >= (int)c->levels.size()) return fail(c, GRANITE_ERR_INVALID, "level out of range");
    if (var != CHI && var != ALPHA) return fail(c, GRANITE_ERR_INVALID, "taggers exist for chi (0) and the lapse (18)");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const LevelLists& L = c->levels[level];
    unsigned long long* d = reinterpret_cast<unsigned long long*>(c->s_sum);  // 16 bytes of scratch
    unsigned long long v = 0;
    CK(cudaMemsetAsync(d, 0, sizeof(v), c->stream), "memset tag count");
    CK(launch_tag_count(c->d_blocks, L.d_mtiles, L.nmtiles, var, threshold, d, c->stream), "launch tagger");
    CK(cudaMemcpyAsync(&v, d, sizeof(v), cudaMemcpyDeviceToHost, c->stream), "read tag count");
    CK(cudaStreamSynchronize(c->stream), "sync");
    c->launches += 1;
    *count = (long long)v;
    return GRANITE_OK;
}

int granite_ccz4_regrid_add(void* h, const granite_block_desc* b, int n) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before regrid");
    if (n < 0 || (n > 0 && !b)) return fail(c, GRANITE_ERR_INVALID, "bad block list");
    if (n == 0) return GRANITE_OK;
    c->copies_valid = false;  // new blocks: their neighbours' ghost copies are not current
    c->step_pushed.clear();
    std::vector<granite_block_desc> descs = c->descs;
    std::vector<int> count(64, 0);
    for (const auto& d : descs) ++count[d.level];
    for (int i = 0; i < n; ++i) {
        int r = check_desc(c, &b[i]);
        if (r) return r;
        if (b[i].level < 1 || b[i].level > 31) return fail(c, GRANITE_ERR_INVALID, "regrid adds blocks on levels >= 1");
        descs.push_back(b[i]);
    }
    // every new block needs a coarser level to be filled from (checked in ascending level order)
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b[x].level < b[y].level; });
    for (int i : order) {
        if (count[b[i].level - 1] == 0) return fail(c, GRANITE_ERR_INVALID, "regrid: no block on the coarser level");
        ++count[b[i].level];
    }
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(drain_profile(c), "profile drain");
    CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    char* arena = nullptr;
    size_t bytes = 0;
    std::vector<DevBlock> hb;
    int r = alloc_arena(c, descs, &arena, &bytes, hb);
    if (r) return r;
    // existing blocks keep their state
    cudaError_t e = cudaMemsetAsync(arena, 0, bytes, c->stream);
    const size_t nold = c->descs.size();
    for (size_t i = 0; i < nold && e == cudaSuccess; ++i)
        e = cudaMemcpyAsync(hb[i].buf[0], c->hblocks[i].buf[0], (size_t)hb[i].stride * NV * sizeof(double),
                            cudaMemcpyDeviceToDevice, c->stream);
    DevBlock* d_hb = nullptr;
    if (e == cudaSuccess) e = upload_vec(hb, &d_hb, c->stream);
    // new blocks: trilinear prolongation of every cell (ghosts included) from the
    // coarser level; the reference prolongates from each coarse block in list order
    // and each writes every fine cell, so the level's last block decides
    // (amr.cpp:291-293 with prolongate, amr.cpp:484-564)
    // (new blocks are filled in ascending level order, so a new coarse block is
    // filled before the finer ones that read it)
    for (int i : order) {
        if (e != cudaSuccess) break;
        const int f = (int)nold + i, L = b[i].level;
        int last = -1;
        for (size_t j = 0; j < descs.size(); ++j)
            if (descs[j].level == L - 1) last = (int)j;
        XferBox x{};
        x.dst = f;
        x.src = last;
        for (int d = 0; d < 3; ++d) x.n[d] = b[i].ncells[d] + 2 * NG;
        XferList xl;
        e = upload_xfer(std::vector<XferBox>{x}, xl, c->stream);
        if (e == cudaSuccess) e = launch_xfer(XFER_PROLONG, d_hb, xl.d_boxes, xl.d_chunks, xl.nchunks, 0, 0, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        free_xfer(xl);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_hb);
    if (e != cudaSuccess) {
        cudaFree(arena);
        return cuda_fail(c, e, "regrid");
    }
    if (c->d_matter) {  // old blocks keep their sources (same offsets), new blocks start in vacuum
        if ((r = realloc_matter(c, total_cells(descs), c->matter_cells))) {
            cudaFree(arena);
            return r;
        }
    }
    release_lists(c);
    cudaFree(c->arena);
    c->arena = arena;
    c->arena_bytes = bytes;
    c->descs = std::move(descs);
    c->hblocks = std::move(hb);
    c->launches += n;
    if ((r = build_lists(c))) return r;
    for (size_t L = c->level_time.size(); L < c->levels.size(); ++L) c->level_time.push_back(c->level_time[L - 1]);
    return GRANITE_OK;
}

static int check_block(Ctx* c, int i) {
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before upload/download");
    if (i < 0 || i >= (int)c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "block index out of range");
    return GRANITE_OK;
}

int granite_ccz4_upload_block(void* h, int i, const double* host) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_block(c, i);
    if (r) return r;
    if (!host) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(c->hblocks[i].buf[0], host, (size_t)c->hblocks[i].stride * NV * sizeof(double),
                       cudaMemcpyHostToDevice, c->stream),
       "H2D block");
    c->level_ghosts_valid[c->descs[i].level] = false;
    c->copies_valid = false;  // the state changed outside a pushing coarse step
    return GRANITE_OK;
}

int granite_ccz4_upload_all(void* h, const double* const* hosts) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before upload/download");
    if (!hosts) return fail(c, GRANITE_ERR_INVALID, "null host buffer list");
    for (size_t i = 0; i < c->descs.size(); ++i)
        if (!hosts[i]) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    for (size_t i = 0; i < c->descs.size(); ++i)
        CK(cudaMemcpyAsync(c->hblocks[i].buf[0], hosts[i], (size_t)c->hblocks[i].stride * NV * sizeof(double),
                           cudaMemcpyHostToDevice, c->stream),
           "H2D block");
    for (size_t L = 0; L < c->level_ghosts_valid.size(); ++L) c->level_ghosts_valid[L] = false;
    c->copies_valid = false;  // the state changed outside a pushing coarse step
    return GRANITE_OK;
}

int granite_ccz4_download_all_async(void* h, double* const* hosts) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before upload/download");
    if (!hosts) return fail(c, GRANITE_ERR_INVALID, "null host buffer list");
    for (size_t i = 0; i < c->descs.size(); ++i)
        if (!hosts[i]) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    for (size_t i = 0; i < c->descs.size(); ++i)
        CK(cudaMemcpyAsync(hosts[i], c->hblocks[i].buf[0], (size_t)c->hblocks[i].stride * NV * sizeof(double),
                           cudaMemcpyDeviceToHost, c->stream),
           "D2H block");
    return GRANITE_OK;
}

int granite_ccz4_download_all(void* h, double* const* hosts) {
    int r = granite_ccz4_download_all_async(h, hosts);
    if (r) return r;
    Ctx* c = static_cast<Ctx*>(h);
    CK(cudaStreamSynchronize(c->stream), "sync");
    return check_errflag(c);  // a stage whose tile wait gave up has left no valid state
}

int granite_ccz4_download_block(void* h, int i, double* host) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_block(c, i);
    if (r) return r;
    if (!host) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(host, c->hblocks[i].buf[0], (size_t)c->hblocks[i].stride * NV * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream),
       "D2H block");
    CK(cudaStreamSynchronize(c->stream), "sync");
    return check_errflag(c);
}

// ---------------------------------------------------------------------------
// stepping
// ---------------------------------------------------------------------------

// One stage over tiles [first, first + count) of a level: one launch, or with
// per-tile precision (MIXED and a positive chi threshold) a classification of
// the tiles from the stage input's chi (flag 1: a point below the threshold),
// then the FP32 kernel over the unflagged tiles and the FP64 kernel over the
// flagged ones. The two passes write disjoint tiles, so the in-place last
// stage is safe and no tile is computed twice.
static cudaError_t stage_range(Ctx* c, LevelLists& L, int cfg, int precision, const StageArgs& a0, int first,
                               int count, long long* n) {
    const Tile* tiles = L.d_tiles + first;
    StageArgs a = a0;
    if (L.variant == VARIANT_TMA) {  // the tensor maps of this configuration's box shape(s)
        a.tmaps = c->d_tmaps + (size_t)tma_shape_of(cfg) * 3 * c->descs.size();
        a.tmaps_rem = TMA_CFGS[cfg].rem ? c->d_tmaps + (size_t)tma_rem_shape_of(cfg) * 3 * c->descs.size() : nullptr;
    }
    if (a.tile_push) a.tile_push += first;  // indexed like the launch's tiles
    // (the TMA kernel keeps a CTA's selected tiles in shared memory: bounded count)
    const bool split = precision == GRANITE_PRECISION_MIXED && c->fp64_chi > 0.0 &&
        (L.variant != VARIANT_TMA || (long long)count <= (long long)tma_grid(cfg) * TMA_SEL_CAP);
    if (!split) {
        ++*n;
        return launch_stage(L.variant, cfg, precision, EPI_RK, c->d_blocks, tiles, count, a, c->stream);
    }
    unsigned char* flags = L.d_flags + first;
    cudaError_t e = launch_classify(L.variant, cfg, c->d_blocks, tiles, 0, count, a.in_sel, c->fp64_chi, flags,
                                    c->stream);
    if (e != cudaSuccess) return e;
    StageArgs b = a;
    b.tile_prec = flags;
    *n += 3;
    // The two passes write disjoint tiles: the FP64 pass (few tiles, few CTAs
    // with work) runs on the second stream beside the FP32 pass and fills the
    // SMs its tail leaves idle. Under the profiler (every launch bracketed by
    // events on the main stream) they run one after the other.
    StageArgs b64 = b;
    b64.want_prec = 1;
    b.want_prec = 0;
    if (c->profiling || !c->overlap_passes) {
        if ((e = launch_stage(L.variant, cfg, PM_MIXED, EPI_RK, c->d_blocks, tiles, count, b, c->stream))) return e;
        return launch_stage(L.variant, cfg, PM_FP64F, EPI_RK, c->d_blocks, tiles, count, b64, c->stream);
    }
    if ((e = cudaEventRecord(c->ev_fork, c->stream))) return e;
    if ((e = cudaStreamWaitEvent(c->stream2, c->ev_fork, 0))) return e;
    if ((e = launch_stage(L.variant, cfg, PM_FP64F, EPI_RK, c->d_blocks, tiles, count, b64, c->stream2))) return e;
    if ((e = launch_stage(L.variant, cfg, PM_MIXED, EPI_RK, c->d_blocks, tiles, count, b, c->stream))) return e;
    if ((e = cudaEventRecord(c->ev_join, c->stream2))) return e;
    return cudaStreamWaitEvent(c->stream, c->ev_join, 0);
}

// The fused stage kernel over one level: the whole work-list at once, or
// (unbatched) block by block.
static cudaError_t level_stage(Ctx* c, LevelLists& L, int precision, const StageArgs& a, long long* n) {
    const int pr = precision == GRANITE_PRECISION_MIXED ? 1 : 0;
    if (c->batched) {
        for (const auto& g : L.groups[pr]) {
            cudaError_t e = timed(c, GRANITE_KERNEL_STAGE,
                                  [&] { return stage_range(c, L, g.cfg, precision, a, g.first, g.count, n); });
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    for (size_t q = 0; q < L.tile_range[pr].size(); ++q) {
        const auto& r = L.tile_range[pr][q];
        cudaError_t e = timed(c, GRANITE_KERNEL_STAGE, [&] {
            return stage_range(c, L, L.block_cfg[pr][q], precision, a, r.first, r.second, n);
        });
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// A block-local ghost fill over one level (batched or per block).
static cudaError_t level_ghost(Ctx* c, LevelLists& L, int mode, int slot, const unsigned char* mask, long long* n) {
    if (c->batched) {
        ++*n;
        return timed(c, GRANITE_KERNEL_GHOST, [&] {
            return launch_ghost_fill(mode, c->d_blocks, L.d_ghost, L.nghost, slot, mask, c->stream);
        });
    }
    for (const auto& r : L.ghost_range) {
        ++*n;
        cudaError_t e = timed(c, GRANITE_KERNEL_GHOST, [&] {
            return launch_ghost_fill(mode, c->d_blocks, L.d_ghost + r.first, r.second, slot, mask, c->stream);
        });
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static cudaError_t enqueue_level_step(Ctx* c, int level, double dt, int precision, int bc, bool prefill,
                                      long long* nl) {
    LevelLists& L = c->levels[level];
    const int level_mode = (bc == GRANITE_BC_PERIODIC) ? GHOST_PERIODIC : GHOST_ZERO_GRADIENT;
    const int outer_mode = (bc == GRANITE_BC_PERIODIC) ? GHOST_PERIODIC : GHOST_SOMMERFELD;
    cudaError_t e;
    long long n = 0;
    // amr.cpp:319 level fill before the step (only when the state changed since the last one)
    if (prefill && (e = level_ghost(c, L, level_mode, 0, nullptr, &n))) return e;
    StageArgs a = base_args(c);
    // stage 1: u1 = u + dt L(u)                       main.cpp:673
    a.in_sel = 0; a.n_sel = 0; a.out_sel = 1; a.final_stage = 0;
    a.a1 = 1.0; a.a2 = 0.0; a.a3dt = 1.0 * dt;
    a.test_withhold = c->test_withhold;  // one-shot test switch (eager steps only)
    c->test_withhold = 0;
    e = level_stage(c, L, precision, a, &n);
    a.test_withhold = 0;
    if (e) return e;
    if ((e = level_ghost(c, L, outer_mode, 1, nullptr, &n))) return e;
    // stage 2: u2 = 3/4 u + 1/4 u1 + 1/4 dt L(u1)      main.cpp:679
    a.in_sel = 1; a.n_sel = 0; a.out_sel = 2;
    a.a1 = 0.75; a.a2 = 0.25; a.a3dt = 0.25 * dt;
    if ((e = level_stage(c, L, precision, a, &n))) return e;
    if ((e = level_ghost(c, L, outer_mode, 2, nullptr, &n))) return e;
    // stage 3: u = 1/3 u + 2/3 u2 + 2/3 dt L(u2), floors, det/trace   main.cpp:685-687
    a.in_sel = 2; a.n_sel = 0; a.out_sel = 0; a.final_stage = 1;
    a.a1 = 1.0 / 3.0; a.a2 = 2.0 / 3.0; a.a3dt = (2.0 / 3.0) * dt;
    if ((e = level_stage(c, L, precision, a, &n))) return e;
    // main.cpp:689 outer BC on u is overwritten by the level fill of amr.cpp:329,
    // so only the level fill runs.
    if ((e = level_ghost(c, L, level_mode, 0, nullptr, &n))) return e;
    *nl = n;
    return cudaSuccess;
}

int granite_ccz4_rk3_step(void* h, int level, double dt, int precision, int bc) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before stepping");
    int r = check_precision(c, precision);
    if (r) return r;
    if (level < 0 || level >= (int)c->levels.size() || c->levels[level].ntiles == 0)
        return fail(c, GRANITE_ERR_INVALID, "level has no blocks");
    if (bc != GRANITE_BC_REFERENCE && bc != GRANITE_BC_PERIODIC) return fail(c, GRANITE_ERR_INVALID, "bad bc");
    if (!std::isfinite(dt)) return fail(c, GRANITE_ERR_INVALID, "dt must be finite");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    c->copies_valid = false;  // a level step fills its ghosts block by block
    const bool prefill = !c->level_ghosts_valid[level];
    if (c->profiling || !c->batched || c->test_withhold) {  // (an armed test switch is never captured)
        long long nl = 0;
        cudaError_t e = enqueue_level_step(c, level, dt, precision, bc, prefill, &nl);
        if (e != cudaSuccess) return cuda_fail(c, e, "enqueue step");
        c->launches += nl;
        c->level_ghosts_valid[level] = true;
        return GRANITE_OK;
    }
    unsigned long long dtbits;
    std::memcpy(&dtbits, &dt, sizeof(dt));
    auto key = std::make_tuple(level, precision, bc, dtbits, (int)prefill);
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) {
        Graph g;
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        long long nl = 0;
        cudaError_t e = enqueue_level_step(c, level, dt, precision, bc, prefill, &nl);
        cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
        if (e != cudaSuccess) return cuda_fail(c, e, "enqueue step");
        if (e2 != cudaSuccess) return cuda_fail(c, e2, "end capture");
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
        g.launches = nl;
        it = c->graphs.emplace(key, g).first;
    }
    CK(cudaGraphLaunch(it->second.exec, c->stream), "graph launch");
    c->launches += it->second.launches;
    c->level_ghosts_valid[level] = true;
    return GRANITE_OK;
}

// ---------------------------------------------------------------------------
// Berger-Oliger hierarchy (amr.cpp:303-350)
// ---------------------------------------------------------------------------

namespace {

struct Interval {
    int lo, hi;  // [lo, hi)
    bool empty() const { return hi <= lo; }
};
Interval meet(Interval a, Interval b) { return {std::max(a.lo, b.lo), std::min(a.hi, b.hi)}; }

// Reference cell centre, grid.hpp:92-94.
double xref(const granite_block_desc& b, int d, int idx) {
    const double dx = (b.hi[d] - b.lo[d]) / static_cast<double>(b.ncells[d]);
    return b.lo[d] + (static_cast<double>(idx) - b.nghost + 0.5) * dx;
}

cudaError_t upload_xfer(const std::vector<XferBox>& boxes, XferList& out, cudaStream_t s) {
    std::vector<BoxChunk> chunks;
    for (int b = 0; b < (int)boxes.size(); ++b) {
        const long long n = (long long)boxes[b].n[0] * boxes[b].n[1] * boxes[b].n[2];
        for (long long r = 0; r < n; r += XFER_CHUNK) chunks.push_back(BoxChunk{b, (int)r});
    }
    cudaError_t e = upload_vec(boxes, &out.d_boxes, s);
    if (e != cudaSuccess) return e;
    e = upload_vec(chunks, &out.d_chunks, s);
    out.nboxes = (int)boxes.size();
    out.nchunks = (int)chunks.size();
    return e;
}

// Global cell index of every block's first interior cell on its level's grid
// (origin: the lower corner of level 0), for the aligned-grid transfers of
// GRANITE_AMR_GHOSTS. Fails when a level's blocks do not share one spacing, a
// level is not twice as fine as its parent, or a block is off the grid.
int level_grid(Ctx* c, std::vector<std::array<int, 3>>& G) {
    const int nb = (int)c->descs.size();
    G.assign(nb, {0, 0, 0});
    double X0[3] = {1e300, 1e300, 1e300};
    for (int i : c->levels[0].blocks)
        for (int d = 0; d < 3; ++d) X0[d] = std::min(X0[d], c->descs[i].lo[d]);
    std::vector<std::array<double, 3>> dxl(c->levels.size());
    for (size_t L = 0; L < c->levels.size(); ++L) {
        const auto& first = c->hblocks[c->levels[L].blocks[0]];
        for (int d = 0; d < 3; ++d) dxl[L][d] = first.dx[d];
        for (int i : c->levels[L].blocks)
            for (int d = 0; d < 3; ++d) {
                if (std::fabs(c->hblocks[i].dx[d] - dxl[L][d]) > 1e-12 * dxl[L][d])
                    return fail(c, GRANITE_ERR_UNSUPPORTED, "blocks of one level must share one cell spacing");
                const double g = (c->descs[i].lo[d] - X0[d]) / dxl[L][d];
                const double gr = std::round(g);
                if (std::fabs(g - gr) > 1e-6)
                    return fail(c, GRANITE_ERR_UNSUPPORTED, "block corner is not on its level's cell grid");
                G[i][d] = (int)gr;
            }
        if (L > 0)
            for (int d = 0; d < 3; ++d)
                if (std::fabs(dxl[L - 1][d] - 2.0 * dxl[L][d]) > 1e-12 * dxl[L - 1][d])
                    return fail(c, GRANITE_ERR_UNSUPPORTED, "refinement ratio must be 2");
    }
    return GRANITE_OK;
}

// Transfer lists for GRANITE_AMR_GHOSTS: ghost slabs of every fine block filled
// from the coarse blocks covering them, then overwritten by same-level
// neighbours where one covers the cell; coarse cells whose 2x2x2 children lie
// in a fine interior are restricted.
int build_ghosts_mode(Ctx* c) {
    std::vector<std::array<int, 3>> G;
    int r = level_grid(c, G);
    if (r) return r;
    auto& X = c->xfer[GRANITE_AMR_GHOSTS];
    X.assign(c->levels.size(), LevelXfer());
    std::vector<std::vector<GhostSrc>> full_src(c->levels.size());    // host copies of the ghost sources
    std::vector<std::vector<XferBox>> restricted(c->levels.size());   // restriction boxes into each level
    for (size_t L = 0; L < c->levels.size(); ++L) {
        const auto& blocks = c->levels[L].blocks;
        // same-level copies
        std::vector<XferBox> copies;
        for (int a : blocks)
            for (int b : blocks) {
                if (a == b) continue;
                XferBox x{};
                bool ok = true;
                for (int d = 0; d < 3; ++d) {
                    const Interval full{G[a][d] - NG, G[a][d] + c->descs[a].ncells[d] + NG};
                    const Interval inb{G[b][d], G[b][d] + c->descs[b].ncells[d]};
                    const Interval m = meet(full, inb);
                    if (m.empty()) {
                        ok = false;
                        break;
                    }
                    x.d0[d] = m.lo - (G[a][d] - NG);
                    x.s0[d] = m.lo - (G[b][d] - NG);
                    x.n[d] = m.hi - m.lo;
                }
                if (!ok) continue;
                x.dst = a;
                x.src = b;
                copies.push_back(x);
            }
        CK(upload_xfer(copies, X[L].copy, c->stream), "upload copy boxes");
        // prolongation into the six ghost slabs of each fine block
        std::vector<XferBox> pro;
        for (int f : (L > 0 ? blocks : std::vector<int>())) {
            const auto& fd = c->descs[f];
            Interval full[3], in[3];
            for (int d = 0; d < 3; ++d) {
                full[d] = {G[f][d] - NG, G[f][d] + fd.ncells[d] + NG};
                in[d] = {G[f][d], G[f][d] + fd.ncells[d]};
            }
            const Interval lo_s[3] = {{full[0].lo, in[0].lo}, {full[1].lo, in[1].lo}, {full[2].lo, in[2].lo}};
            const Interval hi_s[3] = {{in[0].hi, full[0].hi}, {in[1].hi, full[1].hi}, {in[2].hi, full[2].hi}};
            // slabs: z-lo, z-hi (full x, y), y-lo, y-hi (interior z), x-lo, x-hi (interior y, z)
            const Interval slabs[6][3] = {{full[0], full[1], lo_s[2]}, {full[0], full[1], hi_s[2]},
                                          {full[0], lo_s[1], in[2]},   {full[0], hi_s[1], in[2]},
                                          {lo_s[0], in[1], in[2]},     {hi_s[0], in[1], in[2]}};
            for (int cb : c->levels[L - 1].blocks) {
                Interval cov[3];
                for (int d = 0; d < 3; ++d)
                    cov[d] = {2 * G[cb][d], 2 * (G[cb][d] + c->descs[cb].ncells[d])};
                for (auto& sl : slabs) {
                    XferBox x{};
                    bool ok = true;
                    for (int d = 0; d < 3; ++d) {
                        const Interval m = meet(sl[d], cov[d]);
                        if (m.empty()) {
                            ok = false;
                            break;
                        }
                        x.d0[d] = m.lo - (G[f][d] - NG);
                        x.n[d] = m.hi - m.lo;
                    }
                    if (!ok) continue;
                    x.dst = f;
                    x.src = cb;
                    pro.push_back(x);
                }
            }
        }
        CK(upload_xfer(pro, X[L].prolong, c->stream), "upload prolongation boxes");
        // one source per ghost cell: same-level neighbour over coarse block over own fill
        {
            std::vector<GhostSrc> items, sitems;
            X[L].src_range.clear();
            X[L].src_range_stage.clear();
            for (int f : blocks) {
                const long long first = (long long)items.size();
                const auto& fd = c->descs[f];
                const int T0 = fd.ncells[0] + 2 * NG, T1 = fd.ncells[1] + 2 * NG, T2 = fd.ncells[2] + 2 * NG;
                std::vector<std::pair<int, int>> src((size_t)T0 * T1 * T2, {-1, -1});
                auto each = [&](const XferBox& x, auto&& fn) {
                    for (int k = 0; k < x.n[2]; ++k)
                        for (int j = 0; j < x.n[1]; ++j)
                            for (int i = 0; i < x.n[0]; ++i)
                                fn(x.d0[0] + i + T0 * (x.d0[1] + j + T1 * (x.d0[2] + k)), i, j, k);
                };
                for (const auto& x : pro)
                    if (x.dst == f) each(x, [&](int cell, int, int, int) { src[cell] = {x.src, -1}; });
                for (const auto& x : copies)
                    if (x.dst == f) {
                        const auto& sd = c->descs[x.src];
                        const int S0 = sd.ncells[0] + 2 * NG, S1 = sd.ncells[1] + 2 * NG;
                        each(x, [&](int cell, int i, int j, int k) {
                            src[cell] = {x.src, x.s0[0] + i + S0 * (x.s0[1] + j + S1 * (x.s0[2] + k))};
                        });
                    }
                for (int k = 0; k < T2; ++k)
                    for (int j = 0; j < T1; ++j)
                        for (int i = 0; i < T0; ++i) {
                            const bool interior = i >= NG && i < T0 - NG && j >= NG && j < T1 - NG && k >= NG &&
                                k < T2 - NG;
                            if (interior) continue;
                            const int cell = i + T0 * (j + T1 * k);
                            items.push_back(GhostSrc{f, cell, src[cell].first, src[cell].second});
                        }
                // copies, then prolongations, then local fills (each in cell order): warps
                // take one branch of the kernel and their stores stay coalesced
                auto kind = [](const GhostSrc& g) { return g.src_block < 0 ? 2 : (g.src_cell < 0 ? 1 : 0); };
                std::stable_sort(items.begin() + first, items.end(),
                                 [&](const GhostSrc& a, const GhostSrc& b) { return kind(a) < kind(b); });
                X[L].src_range.push_back({first, (long long)items.size() - first});
                // the subset the stencils of a stage read: depth into the ghost layer per axis
                const long long sfirst = (long long)sitems.size();
                auto depth = [](int a, int T) { return a < NG ? NG - a : (a >= T - NG ? a - (T - NG) + 1 : 0); };
                for (long long q = first; q < (long long)items.size(); ++q) {
                    const int cell = items[q].dst_cell;
                    const int di = depth(cell % T0, T0), dj = depth((cell / T0) % T1, T1), dk = depth(cell / (T0 * T1), T2);
                    const int outside = (di > 0) + (dj > 0) + (dk > 0);
                    if (outside == 1 || (outside == 2 && std::max(di, std::max(dj, dk)) == 1)) sitems.push_back(items[q]);
                }
                X[L].src_range_stage.push_back({sfirst, (long long)sitems.size() - sfirst});
            }
            CK(upload_vec(items, &X[L].d_src, c->stream), "upload ghost sources");
            X[L].nsrc = (long long)items.size();
            full_src[L] = items;
            CK(upload_vec(sitems, &X[L].d_src_stage, c->stream), "upload stage ghost sources");
            X[L].nsrc_stage = (long long)sitems.size();
            // the same lists without the same-level copies (for the fills after a pushing stage)
            auto nocopy = [](const std::vector<GhostSrc>& all, const std::vector<std::pair<long long, long long>>& rg,
                             std::vector<GhostSrc>& out, std::vector<std::pair<long long, long long>>& orange) {
                for (const auto& r : rg) {
                    const long long f = (long long)out.size();
                    for (long long q = r.first; q < r.first + r.second; ++q)
                        if (!(all[q].src_block >= 0 && all[q].src_cell >= 0)) out.push_back(all[q]);
                    orange.push_back({f, (long long)out.size() - f});
                }
            };
            std::vector<GhostSrc> nc, snc;
            X[L].src_range_nc.clear();
            X[L].src_range_stage_nc.clear();
            nocopy(items, X[L].src_range, nc, X[L].src_range_nc);
            nocopy(sitems, X[L].src_range_stage, snc, X[L].src_range_stage_nc);
            CK(upload_vec(nc, &X[L].d_src_nc, c->stream), "upload ghost sources without copies");
            X[L].nsrc_nc = (long long)nc.size();
            CK(upload_vec(snc, &X[L].d_src_stage_nc, c->stream), "upload stage ghost sources without copies");
            X[L].nsrc_stage_nc = (long long)snc.size();
        }
        // push boxes: every copy box (a <- b) seen from b's interior, and per
        // stage tile of the level the boxes of its block that meet the tile.
        // Only where no two interiors of the level overlap (then every ghost
        // cell has at most one same-level source, the one the fill would copy).
        {
            bool ovl = false;
            for (size_t p = 0; p < blocks.size() && !ovl; ++p)
                for (size_t q = p + 1; q < blocks.size() && !ovl; ++q) {
                    bool all = true;
                    for (int d = 0; d < 3 && all; ++d)
                        all = !meet({G[blocks[p]][d], G[blocks[p]][d] + c->descs[blocks[p]].ncells[d]},
                                    {G[blocks[q]][d], G[blocks[q]][d] + c->descs[blocks[q]].ncells[d]})
                                   .empty();
                    ovl = all;
                }
            LevelLists& ll = c->levels[L];
            X[L].push_ok = !ovl && ll.variant == VARIANT_TMA && !ll.h_tiles.empty();
            if (X[L].push_ok) {
                std::map<int, std::vector<PushBox>>& by_src = X[L].push_by_src;
                by_src.clear();
                for (const XferBox& x : copies) {
                    const DevBlock& D = c->hblocks[x.dst];
                    PushBox pb{};
                    for (int sl = 0; sl < 3; ++sl) pb.buf[sl] = D.buf[sl];
                    pb.stride = D.stride;
                    pb.tx = D.tx;
                    pb.txy = D.tx * D.ty;
                    int off[3];
                    for (int d = 0; d < 3; ++d) {
                        pb.lo[d] = x.s0[d] - NG;
                        pb.hi[d] = pb.lo[d] + x.n[d];
                        off[d] = x.d0[d] + NG - x.s0[d];  // destination cell index - source interior index
                    }
                    pb.base = off[0] + (long long)pb.tx * off[1] + (long long)pb.txy * off[2];
                    by_src[x.src].push_back(pb);
                }
                std::vector<PushBox> plist;
                std::vector<int2> tp(ll.h_tiles.size(), make_int2(0, 0));
                for (int pr = 0; pr < 2; ++pr)
                    for (const StageGroup& g : ll.groups[pr]) {
                        int TX, TY, TZ;
                        stage_tile_dims(ll.variant, g.cfg, &TX, &TY, &TZ);
                        const int tdim[3] = {TX, TY, TZ};
                        for (int t = g.first; t < g.first + g.count; ++t) {
                            const Tile& tl = ll.h_tiles[t];
                            const int t0[3] = {tl.i0, tl.j0, tl.k0};
                            const int rdim[3] = {TMA_REM_X, TY, 2 * TZ};  // x-remainder tiles
                            const int* tdim_t = tl.w < 0 ? rdim : tdim;
                            const int first = (int)plist.size();
                            auto it = by_src.find(tl.block);
                            if (it != by_src.end())
                                for (const PushBox& pb : it->second) {
                                    bool hit = true;
                                    for (int d = 0; d < 3 && hit; ++d) hit = pb.lo[d] < t0[d] + tdim_t[d] && pb.hi[d] > t0[d];
                                    if (hit) plist.push_back(pb);
                                }
                            tp[t] = make_int2(first, (int)plist.size() - first);
                        }
                    }
                CK(upload_vec(plist, &X[L].d_push, c->stream), "upload push boxes");
                CK(upload_vec(tp, &X[L].d_tile_push, c->stream), "upload tile push ranges");
                if (!X[L].d_push) X[L].push_ok = false;  // nothing to push on this level
            }
        }
        // restriction into level L-1 from level L: one launch for the level, or,
        // where fine interiors overlap (a regrid adds blocks beside the old ones),
        // one launch per fine block in list order so that the last one holding a
        // coarse cell's children decides it, as in the reference (amr.cpp:339-341)
        if (L == 0) continue;
        bool overlap = false;
        for (size_t p = 0; p < blocks.size() && !overlap; ++p)
            for (size_t q = p + 1; q < blocks.size() && !overlap; ++q) {
                bool all = true;
                for (int d = 0; d < 3 && all; ++d)
                    all = !meet({G[blocks[p]][d], G[blocks[p]][d] + c->descs[blocks[p]].ncells[d]},
                                {G[blocks[q]][d], G[blocks[q]][d] + c->descs[blocks[q]].ncells[d]})
                               .empty();
                overlap = all;
            }
        std::vector<std::vector<XferBox>> waves(overlap ? blocks.size() : 1);
        for (int cb : c->levels[L - 1].blocks)
            for (size_t fi = 0; fi < blocks.size(); ++fi) {
                const int f = blocks[fi];
                std::vector<XferBox>& res = waves[overlap ? fi : 0];
                XferBox x{};
                bool ok = true;
                for (int d = 0; d < 3; ++d) {
                    const int F0 = G[f][d], nf = c->descs[f].ncells[d];
                    // coarse I with children 2I, 2I+1 inside [F0, F0 + nf) (F0 >= 0)
                    const Interval ci{(F0 + 1) / 2, (F0 + nf) / 2};
                    const Interval m = meet(ci, {G[cb][d], G[cb][d] + c->descs[cb].ncells[d]});
                    if (m.empty()) {
                        ok = false;
                        break;
                    }
                    x.d0[d] = m.lo - (G[cb][d] - NG);
                    x.s0[d] = 2 * m.lo - (F0 - NG);
                    x.n[d] = m.hi - m.lo;
                }
                if (!ok) continue;
                x.dst = cb;
                x.src = f;
                res.push_back(x);
            }
        for (const auto& res : waves) {
            X[L - 1].restrict_.emplace_back();
            CK(upload_xfer(res, X[L - 1].restrict_.back(), c->stream), "upload restriction boxes");
            for (const XferBox& x : res) restricted[L - 1].push_back(x);
        }
    }
    // The fill before a level step when the same-level copies are current (the
    // fill after the level's previous step, or its pushing stages, made them
    // so): the copies whose source cell a restriction into the level can have
    // changed since, and every non-copy ghost cell. (The restriction itself
    // does not push: like the reference, it leaves the neighbours' copies of
    // the cells it writes stale until this fill.) Built for every level.
    for (size_t L = 0; L < c->levels.size(); ++L) {
        std::map<int, std::vector<char>> mask;  // per block of the level: cells some restriction writes
        for (const XferBox& x : restricted[L]) {
            const auto& d = c->descs[x.dst];
            const int T0 = d.ncells[0] + 2 * NG, T1 = d.ncells[1] + 2 * NG, T2 = d.ncells[2] + 2 * NG;
            auto& m = mask[x.dst];
            if (m.empty()) m.assign((size_t)T0 * T1 * T2, 0);
            for (int k = 0; k < x.n[2]; ++k)
                for (int j = 0; j < x.n[1]; ++j)
                    for (int i = 0; i < x.n[0]; ++i)
                        m[(size_t)(x.d0[0] + i) + (size_t)T0 * ((x.d0[1] + j) + (size_t)T1 * (x.d0[2] + k))] = 1;
        }
        std::vector<GhostSrc> pre;
        X[L].src_range_pre.clear();
        for (const auto& r : X[L].src_range) {
            const long long f = (long long)pre.size();
            for (long long q = r.first; q < r.first + r.second; ++q) {
                const GhostSrc& g = full_src[L][q];
                const bool copy = g.src_block >= 0 && g.src_cell >= 0;
                auto it = copy ? mask.find(g.src_block) : mask.end();
                if (!copy || (it != mask.end() && it->second[g.src_cell])) pre.push_back(g);
            }
            X[L].src_range_pre.push_back({f, (long long)pre.size() - f});
        }
        CK(upload_vec(pre, &X[L].d_src_pre, c->stream), "upload prefill ghost sources");
        X[L].nsrc_pre = (long long)pre.size();
    }
    c->xfer_built[GRANITE_AMR_GHOSTS] = true;
    return GRANITE_OK;
}

// Transfer lists for GRANITE_AMR_REFERENCE, literally amr.cpp: every fine block
// is overwritten in all its cells by prolongation from each coarse block in
// turn (the last one wins, amr.cpp:313-318,438), faces no coarse block covers
// get the zero-gradient fill (amr.cpp:420-480), and restriction runs fine block
// by fine block (amr.cpp:339-341,566-626).
int build_reference_mode(Ctx* c) {
    auto& X = c->xfer[GRANITE_AMR_REFERENCE];
    X.assign(c->levels.size(), LevelXfer());
    for (size_t L = 0; L < c->levels.size(); ++L) {
        const auto& blocks = c->levels[L].blocks;
        std::vector<unsigned char> mask(c->descs.size(), 0x3F);
        if (L > 0) {
            const int last = c->levels[L - 1].blocks.back();
            std::vector<XferBox> pro;
            for (int f : blocks) {
                const auto& fd = c->descs[f];
                XferBox x{};
                x.dst = f;
                x.src = last;
                for (int d = 0; d < 3; ++d) x.n[d] = fd.ncells[d] + 2 * NG;
                pro.push_back(x);
                unsigned char m = 0;
                for (int d = 0; d < 3; ++d) {
                    const double dxf = (fd.hi[d] - fd.lo[d]) / static_cast<double>(fd.ncells[d]);
                    const double fine_lo = xref(fd, d, fd.nghost), fine_hi = xref(fd, d, fd.nghost + fd.ncells[d] - 1);
                    bool flo = false, fhi = false;
                    for (int cb : c->levels[L - 1].blocks) {
                        const auto& cd = c->descs[cb];
                        if (xref(cd, d, cd.nghost) <= fine_lo + 0.5 * dxf) flo = true;
                        if (xref(cd, d, cd.nghost + cd.ncells[d] - 1) >= fine_hi - 0.5 * dxf) fhi = true;
                    }
                    if (!flo) m |= (unsigned char)(1u << (2 * d));
                    if (!fhi) m |= (unsigned char)(1u << (2 * d + 1));
                }
                mask[f] = m;
            }
            CK(upload_xfer(pro, X[L].prolong, c->stream), "upload prolongation boxes");
            // restriction into level L-1, one launch per fine block in order
            for (int f : blocks) {
                const auto& fd = c->descs[f];
                std::vector<XferBox> res;
                for (int cb : c->levels[L - 1].blocks) {
                    const auto& cd = c->descs[cb];
                    XferBox x{};
                    bool ok = true;
                    for (int d = 0; d < 3; ++d) {
                        const double dxf = (fd.hi[d] - fd.lo[d]) / static_cast<double>(fd.ncells[d]);
                        const double fx0 = xref(fd, d, 0);
                        int first = -1, last = -1, base0 = 0;
                        for (int ci = cd.nghost; ci < cd.nghost + cd.ncells[d]; ++ci) {
                            const int fb = (int)std::round((xref(cd, d, ci) - fx0) / dxf) - 1;
                            const bool in = fb >= fd.nghost && fb + 2 <= fd.nghost + fd.ncells[d] + fd.nghost;
                            if (!in) continue;
                            if (first < 0) {
                                first = ci;
                                base0 = fb;
                            } else if (ci != last + 1 || fb != base0 + 2 * (ci - first)) {
                                return fail(c, GRANITE_ERR_UNSUPPORTED,
                                            "restriction needs ratio-2 aligned blocks");
                            }
                            last = ci;
                        }
                        if (first < 0) {
                            ok = false;
                            break;
                        }
                        x.d0[d] = first;
                        x.s0[d] = base0;
                        x.n[d] = last - first + 1;
                    }
                    if (!ok) continue;
                    x.dst = cb;
                    x.src = f;
                    res.push_back(x);
                }
                X[L - 1].restrict_.emplace_back();
                CK(upload_xfer(res, X[L - 1].restrict_.back(), c->stream), "upload restriction boxes");
            }
        }
        CK(upload_vec(mask, &X[L].d_facemask, c->stream), "upload face masks");
    }
    c->xfer_built[GRANITE_AMR_REFERENCE] = true;
    return GRANITE_OK;
}

cudaError_t xfer(Ctx* c, int kind, const XferList& x, int dst_sel, int src_sel) {
    if (x.nchunks == 0) return cudaSuccess;
    return timed(c, GRANITE_KERNEL_TRANSFER, [&] {
        return launch_xfer(kind, c->d_blocks, x.d_boxes, x.d_chunks, x.nchunks, dst_sel, src_sel, c->stream);
    });
}

// Ghost fill of one level's buffer slot. level_fill: the fill around a step
// (zero-gradient base); otherwise a stage fill (1/r falloff base).
// pushed: the fill after a stage that pushed the same-level copies (no copies);
// prefill_fresh: the fill before a step while the pushed copies are current
// (only the copies of cells restrictions write).
cudaError_t fill_level(Ctx* c, int L, int slot, bool level_fill, int mode, long long* n, bool pushed = false,
                       bool prefill_fresh = false) {
    LevelLists& ll = c->levels[L];
    const LevelXfer& X = c->xfer[mode][L];
    cudaError_t e;
    if (mode == GRANITE_AMR_REFERENCE) {
        if (level_fill) {
            if (L > 0) {  // fillGhostZones: prolongate into all cells, then the uncovered faces
                if ((e = xfer(c, XFER_PROLONG, X.prolong, slot, 0))) return e;
                ++*n;
            }
            const int gm = L > 0 ? GHOST_ZERO_GRADIENT_MASKED : GHOST_ZERO_GRADIENT;
            return level_ghost(c, ll, gm, slot, X.d_facemask, n);
        }
        // applyOuterBC on every block (main.cpp:351-521)
        return level_ghost(c, ll, GHOST_SOMMERFELD, slot, nullptr, n);
    }
    // GRANITE_AMR_GHOSTS: every ghost cell once, from a same-level neighbour if one
    // covers it, else from the coarse level, else from the block's own fill. The
    // state (slot 0) gets every ghost cell (finer levels prolong from it, callers
    // read it); an RK stage buffer only the cells the stage stencils read.
    // after a stage that pushed the same-level copies, the lists without them
    const int local = level_fill ? GHOST_ZERO_GRADIENT : GHOST_SOMMERFELD;
    const bool all = slot == 0;
    const GhostSrc* src = all ? (prefill_fresh ? X.d_src_pre : pushed ? X.d_src_nc : X.d_src)
                              : (pushed ? X.d_src_stage_nc : X.d_src_stage);
    const long long nsrc = all ? (prefill_fresh ? X.nsrc_pre : pushed ? X.nsrc_nc : X.nsrc)
                               : (pushed ? X.nsrc_stage_nc : X.nsrc_stage);
    const auto& ranges = all ? (prefill_fresh ? X.src_range_pre : pushed ? X.src_range_nc : X.src_range)
                             : (pushed ? X.src_range_stage_nc : X.src_range_stage);
    if (c->batched) {
        if (nsrc == 0) return cudaSuccess;
        ++*n;
        return timed(c, GRANITE_KERNEL_GHOST, [&] {
            return launch_ghost_sources(c->d_blocks, src, nsrc, slot, local, c->stream);
        });
    }
    for (const auto& r : ranges) {
        if (r.second == 0) continue;
        ++*n;
        if ((e = timed(c, GRANITE_KERNEL_GHOST, [&] {
                 return launch_ghost_sources(c->d_blocks, src + r.first, r.second, slot, local, c->stream);
             })))
            return e;
    }
    return cudaSuccess;
}

// Whether the stage kernels of level L push the same-level ghost copies in mode.
bool pushes(const Ctx* c, int L, int mode) {
    return mode == GRANITE_AMR_GHOSTS && c->ghost_push && c->xfer_built[mode] && c->xfer[mode][L].push_ok;
}

cudaError_t stage(Ctx* c, int L, int precision, int in, int out, double a1, double a2, double a3dt, int final_stage,
                  long long* n, bool push = false) {
    LevelLists& ll = c->levels[L];
    StageArgs a = base_args(c);
    if (push) {
        a.push = c->xfer[GRANITE_AMR_GHOSTS][L].d_push;
        a.tile_push = c->xfer[GRANITE_AMR_GHOSTS][L].d_tile_push;
    }
    a.in_sel = in;
    a.n_sel = 0;
    a.out_sel = out;
    a.final_stage = final_stage;
    a.a1 = a1;
    a.a2 = a2;
    a.a3dt = a3dt;
    return level_stage(c, ll, precision, a, n);
}

int ensure_xfer(Ctx* c, int mode) {
    if (c->xfer_built[mode]) return GRANITE_OK;
    return mode == GRANITE_AMR_GHOSTS ? build_ghosts_mode(c) : build_reference_mode(c);
}

// The regrid step of subcycle (amr.cpp:343-349): after level L's step, with
// step_num = round(current_time / (dt + 1e-15)) a multiple of the interval,
// the caller's regrid runs on the host (it may add blocks through
// granite_ccz4_regrid_add, which rebuilds every list; subcycle re-reads them).
struct RegridHook {
    int interval;
    granite_regrid_fn fn;
    void* user;
    int status;  // first non-zero status of fn or of a list rebuild
};

// AMRHierarchy::subcycle(L) with the RK3 step as evolve_func, amr.cpp:303-350.
// With a hook, nothing is captured: the level times advance here and the hook
// runs at the reference's regrid points.
// skip_prefill: the level's state and every cell its fill reads are what the
// fill at the end of its previous step saw (the second substep of the finest
// level in GRANITE_AMR_GHOSTS: nothing restricts into it, its parent does not
// change between the two substeps), so the fill before this step would write
// the values already there.
cudaError_t subcycle(Ctx* c, int L, double dt, int precision, int mode, long long* n, RegridHook* hook = nullptr,
                     bool skip_prefill = false) {
    cudaError_t e;
    if (hook && (hook->status = ensure_xfer(c, mode))) return cudaErrorInvalidValue;
    const LevelXfer& X = c->xfer[mode][L];
    if (skip_prefill) {
    } else if (mode == GRANITE_AMR_REFERENCE && L > 0) {  // amr.cpp:313-318 (the fill below repeats it exactly)
        if ((e = xfer(c, XFER_PROLONG, X.prolong, 0, 0))) return e;
        ++*n;
        if ((e = level_ghost(c, c->levels[L], GHOST_ZERO_GRADIENT_MASKED, 0, X.d_facemask, n))) return e;
    } else {
        // amr.cpp:319; once the fill after this level's last step (or its pushing
        // stages) made the same-level copies current, only those whose source a
        // restriction rewrote since are stale: between that fill and this one
        // the level's state changed only by restrictions into it
        const bool fresh = mode == GRANITE_AMR_GHOSTS &&
                           (c->copies_valid || (L < (int)c->step_pushed.size() && c->step_pushed[L]));
        if ((e = fill_level(c, L, 0, true, mode, n, false, fresh))) return e;
    }
    // TimeIntegrator::sspRK3Step, main.cpp:673-689 (in GRANITE_AMR_GHOSTS the
    // stages write the same-level ghost copies themselves; the fills add the rest)
    const bool push = pushes(c, L, mode);
    if ((e = stage(c, L, precision, 0, 1, 1.0, 0.0, 1.0 * dt, 0, n, push))) return e;
    if ((e = fill_level(c, L, 1, false, mode, n, push))) return e;
    if ((e = stage(c, L, precision, 1, 2, 0.75, 0.25, 0.25 * dt, 0, n, push))) return e;
    if ((e = fill_level(c, L, 2, false, mode, n, push))) return e;
    if ((e = stage(c, L, precision, 2, 0, 1.0 / 3.0, 2.0 / 3.0, (2.0 / 3.0) * dt, 1, n, push))) return e;
    if ((e = fill_level(c, L, 0, true, mode, n, push))) return e;  // amr.cpp:329
    if (mode == GRANITE_AMR_GHOSTS && L < (int)c->step_pushed.size()) c->step_pushed[L] = 1;
    if (hook) c->level_time[L] += dt;                         // amr.cpp:326
    if (L + 1 < (int)c->levels.size()) {
        for (int r = 0; r < 2; ++r) {  // amr.cpp:334-336, :393-397
            // (with a regrid hook the level list may change between the substeps: always fill)
            const bool skip = r == 1 && !hook && mode == GRANITE_AMR_GHOSTS && L + 2 == (int)c->levels.size();
            if ((e = subcycle(c, L + 1, dt / 2.0, precision, mode, n, hook, skip))) return e;
        }
        if (hook && (hook->status = ensure_xfer(c, mode))) return cudaErrorInvalidValue;  // a regrid rebuilt them
        for (const XferList& rl : c->xfer[mode][L].restrict_) {                            // amr.cpp:339-341
            if ((e = xfer(c, XFER_RESTRICT, rl, 0, 0))) return e;
            ++*n;
        }
    }
    if (hook && hook->interval > 0) {
        const long long step_num = std::llround(c->level_time[L] / (dt + 1e-15));
        if (step_num % hook->interval == 0) {
            if ((e = cudaStreamSynchronize(c->stream))) return e;
            if ((hook->status = hook->fn(hook->user, L, step_num))) {
                fail(c, hook->status, "regrid callback returned " + std::to_string(hook->status));
                return cudaErrorInvalidValue;
            }
        }
    }
    return cudaSuccess;
}

}  // namespace

static int check_hierarchy_step(Ctx* c, double dt_coarse, int precision, int amr_mode) {
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit before stepping");
    int r = check_precision(c, precision);
    if (r) return r;
    if (amr_mode != GRANITE_AMR_REFERENCE && amr_mode != GRANITE_AMR_GHOSTS)
        return fail(c, GRANITE_ERR_INVALID, "amr_mode must be GRANITE_AMR_REFERENCE or GRANITE_AMR_GHOSTS");
    if (!std::isfinite(dt_coarse)) return fail(c, GRANITE_ERR_INVALID, "dt must be finite");
    for (auto& L : c->levels)
        if (L.blocks.empty()) return fail(c, GRANITE_ERR_INVALID, "hierarchy levels must be contiguous from 0");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    return ensure_xfer(c, amr_mode);
}

// Level times of one coarse step without the hook: level L takes 2^L steps of
// dt / 2^L (the same additions the hook path makes).
static void advance_level_times(Ctx* c, double dt_coarse) {
    double dt = dt_coarse;
    for (size_t L = 0; L < c->level_time.size(); ++L, dt /= 2.0)
        for (long long s = 0; s < (1LL << L); ++s) c->level_time[L] += dt;
}

int granite_ccz4_hierarchy_step(void* h, double dt_coarse, int precision, int amr_mode) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_hierarchy_step(c, dt_coarse, precision, amr_mode);
    if (r) return r;
    for (size_t L = 0; L < c->level_ghosts_valid.size(); ++L) c->level_ghosts_valid[L] = false;
    const bool valid_at_start = c->copies_valid && amr_mode == GRANITE_AMR_GHOSTS;
    c->step_pushed.assign(c->levels.size(), 0);
    auto finish = [&]() {  // after a GRANITE_AMR_GHOSTS coarse step only copies of restricted cells are stale
        c->copies_valid = amr_mode == GRANITE_AMR_GHOSTS;
        c->step_pushed.clear();
    };
    if (c->profiling || !c->batched) {
        long long n = 0;
        cudaError_t e = subcycle(c, 0, dt_coarse, precision, amr_mode, &n);
        if (e != cudaSuccess) return cuda_fail(c, e, "hierarchy step");
        c->launches += n;
        advance_level_times(c, dt_coarse);
        finish();
        return GRANITE_OK;
    }
    unsigned long long dtbits;
    std::memcpy(&dtbits, &dt_coarse, sizeof(dt_coarse));
    auto key = std::make_tuple(precision, amr_mode + (valid_at_start ? 2 : 0), dtbits);
    auto it = c->hgraphs.find(key);
    if (it == c->hgraphs.end()) {
        Graph g;
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        long long n = 0;
        cudaError_t e = subcycle(c, 0, dt_coarse, precision, amr_mode, &n);
        cudaError_t e2 = cudaStreamEndCapture(c->stream, &graph);
        if (e != cudaSuccess) return cuda_fail(c, e, "enqueue hierarchy step");
        if (e2 != cudaSuccess) return cuda_fail(c, e2, "end capture");
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
        g.launches = n;
        it = c->hgraphs.emplace(key, g).first;
    }
    CK(cudaGraphLaunch(it->second.exec, c->stream), "graph launch");
    c->launches += it->second.launches;
    advance_level_times(c, dt_coarse);
    finish();
    return GRANITE_OK;
}

int granite_ccz4_hierarchy_step_regrid(void* h, double dt_coarse, int precision, int amr_mode, int regrid_interval,
                                       granite_regrid_fn fn, void* user) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (regrid_interval < 0 || (regrid_interval > 0 && !fn))
        return fail(c, GRANITE_ERR_INVALID, "regrid_interval >= 0, with a callback when > 0");
    int r = check_hierarchy_step(c, dt_coarse, precision, amr_mode);
    if (r) return r;
    for (size_t L = 0; L < c->level_ghosts_valid.size(); ++L) c->level_ghosts_valid[L] = false;
    c->copies_valid = false;  // the state changed outside a pushing coarse step
    RegridHook hook{regrid_interval, fn, user, 0};
    long long n = 0;
    cudaError_t e = subcycle(c, 0, dt_coarse, precision, amr_mode, &n, &hook);
    c->launches += n;
    if (hook.status) return hook.status;  // the message is the callback's or the rebuild's
    if (e != cudaSuccess) return cuda_fail(c, e, "hierarchy step with regrid");
    return GRANITE_OK;
}

int granite_ccz4_level_time(void* h, int level, double* t) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c || !t) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit first");
    if (level < 0 || level >= (int)c->level_time.size()) return fail(c, GRANITE_ERR_INVALID, "bad level");
    *t = c->level_time[level];
    return GRANITE_OK;
}

int granite_ccz4_constraint_norms(void* h, int level, double* h_l2, double* m_l2) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit first");
    if (!h_l2 || !m_l2) return fail(c, GRANITE_ERR_INVALID, "null output");
    if (level < -1 || level >= (int)c->levels.size()) return fail(c, GRANITE_ERR_INVALID, "bad level");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    double sh = 0.0, sm = 0.0;
    long long npts = 0;
    for (int L = 0; L < (int)c->levels.size(); ++L) {
        if (level >= 0 && L != level) continue;
        LevelLists& ll = c->levels[L];
        if (ll.ntiles == 0) continue;
        CK(launch_constraints(c->d_blocks, ll.d_mtiles, ll.nmtiles, 0, nullptr, nullptr, c->s_partials, c->stream),
           "launch constraints");
        CK(launch_sum_partials(c->s_partials, ll.nmtiles, c->s_sum, c->stream), "launch sum");
        c->launches += 2;
        double hs[2];
        CK(cudaMemcpyAsync(hs, c->s_sum, sizeof(hs), cudaMemcpyDeviceToHost, c->stream), "D2H sums");
        CK(cudaStreamSynchronize(c->stream), "sync");
        sh += hs[0];
        sm += hs[1];
        npts += ll.interior_points;
    }
    if (npts == 0) return fail(c, GRANITE_ERR_INVALID, "no points");
    *h_l2 = std::sqrt(sh / (double)npts);
    *m_l2 = std::sqrt(sm / (double)npts);
    return GRANITE_OK;
}

int granite_ccz4_compare_states(void* ha, void* hb, double* max_dev, double* max_abs, long long* nonfinite) {
    Ctx* c = static_cast<Ctx*>(ha);
    Ctx* o = static_cast<Ctx*>(hb);
    if (!c || !o) return GRANITE_ERR_INVALID;
    if (!max_dev || !max_abs || !nonfinite) return fail(c, GRANITE_ERR_INVALID, "null output");
    if (!c->committed || !o->committed) return fail(c, GRANITE_ERR_INVALID, "commit both contexts first");
    if (c->device != o->device) return fail(c, GRANITE_ERR_INVALID, "contexts on different devices");
    if (c->descs.size() != o->descs.size()) return fail(c, GRANITE_ERR_INVALID, "different block counts");
    for (size_t i = 0; i < c->descs.size(); ++i)
        for (int d = 0; d < 3; ++d)
            if (c->descs[i].ncells[d] != o->descs[i].ncells[d])
                return fail(c, GRANITE_ERR_INVALID, "different block geometry");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    if (!c->d_cmp) CK(cudaMalloc(&c->d_cmp, (2 * NV + 2) * sizeof(unsigned long long)), "cudaMalloc(compare)");
    CK(cudaStreamSynchronize(o->stream), "cudaStreamSynchronize");  // the other context's steps have landed
    CK(launch_compare_states(c->d_blocks, o->d_blocks, (int)c->descs.size(), c->d_cmp, c->stream),
       "launch compare");
    ++c->launches;
    unsigned long long r[2 * NV + 2];
    CK(cudaMemcpyAsync(r, c->d_cmp, sizeof(r), cudaMemcpyDeviceToHost, c->stream), "D2H compare");
    CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    for (int v = 0; v < NV; ++v) {
        std::memcpy(&max_dev[v], &r[v], sizeof(double));
        std::memcpy(&max_abs[v], &r[NV + v], sizeof(double));
    }
    nonfinite[0] = (long long)r[2 * NV];
    nonfinite[1] = (long long)r[2 * NV + 1];
    return GRANITE_OK;
}

// ---------------------------------------------------------------------------
// Checkpoint / restart of the resident state
//
// The data model of HDF5Writer::writeCheckpoint (hdf5_io.cpp:166-233): root
// attributes time, step, num_blocks, then per block b the totalSize() values of
// every field v ("block_b/var_v"), in block order and field order. The
// container is a flat little-endian file (the HDF5 library is not linked):
//   "GRNB200\0", u32 version, u32 data offset,
//   i32 step, i32 num_blocks, i32 num_vars, i32 num_levels, i32 has_matter, i32 0,
//   f64 time, f64 level_time[num_levels], granite_block_desc blocks[num_blocks],
//   zero padding to the data offset (a multiple of 4096),
//   block_b/var_v for every b, v (f64), then, with matter, rho[N], Si[N][3],
//   Sij[N][6], S[N] (N = the cells of all blocks).
// Unlike the reference's reader (hdf5_io.cpp:392-467, which rebuilds every block
// with the level-0 geometry), the block geometry is stored, so a hierarchy
// resumes as it was.
// ---------------------------------------------------------------------------
namespace {

constexpr char CK_MAGIC[8] = {'G', 'R', 'N', 'B', '2', '0', '0', '\0'};
constexpr uint32_t CK_VERSION = 1;
constexpr size_t CK_CHUNK = size_t(64) << 20;  // pinned staging per transfer

struct CkHeader {
    char magic[8];
    uint32_t version, data_offset;
    int32_t step, num_blocks, num_vars, num_levels, has_matter, zero;
    double time;
};
static_assert(sizeof(CkHeader) == 48, "checkpoint header layout");
static_assert(sizeof(granite_block_desc) == 72, "block descriptor layout");

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

int read_header(Ctx* c, FILE* f, CkHeader& h, std::vector<double>& lt, std::vector<granite_block_desc>& d) {
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, CK_MAGIC, 8) != 0)
        return fail(c, GRANITE_ERR_INVALID, "not a granite_b200 checkpoint");
    if (h.version != CK_VERSION) return fail(c, GRANITE_ERR_UNSUPPORTED, "checkpoint version");
    if (h.num_vars != NV || h.num_blocks < 0 || h.num_levels < 0 || h.num_levels > 64)
        return fail(c, GRANITE_ERR_INVALID, "checkpoint header");
    lt.resize(h.num_levels);
    d.resize(h.num_blocks);
    if ((h.num_levels && std::fread(lt.data(), sizeof(double), lt.size(), f) != lt.size()) ||
        (h.num_blocks && std::fread(d.data(), sizeof(granite_block_desc), d.size(), f) != d.size()))
        return fail(c, GRANITE_ERR_INVALID, "truncated checkpoint header");
    return GRANITE_OK;
}

// Device <-> file through one pinned staging buffer, CK_CHUNK bytes at a time.
int stream_out(Ctx* c, FILE* f, const char* dev, size_t bytes, char* pin) {
    for (size_t o = 0; o < bytes; o += CK_CHUNK) {
        const size_t n = std::min(CK_CHUNK, bytes - o);
        CK(cudaMemcpyAsync(pin, dev + o, n, cudaMemcpyDeviceToHost, c->stream), "D2H checkpoint");
        CK(cudaStreamSynchronize(c->stream), "sync");
        if (std::fwrite(pin, 1, n, f) != n) return fail(c, GRANITE_ERR_INVALID, "checkpoint write failed");
    }
    return GRANITE_OK;
}

int stream_in(Ctx* c, FILE* f, char* dev, size_t bytes, char* pin) {
    for (size_t o = 0; o < bytes; o += CK_CHUNK) {
        const size_t n = std::min(CK_CHUNK, bytes - o);
        if (std::fread(pin, 1, n, f) != n) return fail(c, GRANITE_ERR_INVALID, "truncated checkpoint data");
        CK(cudaMemcpyAsync(dev + o, pin, n, cudaMemcpyHostToDevice, c->stream), "H2D checkpoint");
        CK(cudaStreamSynchronize(c->stream), "sync");
    }
    return GRANITE_OK;
}

struct Pinned {
    char* p = nullptr;
    ~Pinned() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

int granite_ccz4_checkpoint_header(const char* path, int* step, double* time, int* has_matter,
                                   granite_block_desc* blocks, int cap, int* num_blocks) {
    if (!path || !num_blocks) return GRANITE_ERR_INVALID;
    File f;
    if (!(f.f = std::fopen(path, "rb"))) return GRANITE_ERR_INVALID;
    CkHeader h;
    std::vector<double> lt;
    std::vector<granite_block_desc> d;
    int r = read_header(nullptr, f.f, h, lt, d);
    if (r) return r;
    *num_blocks = h.num_blocks;
    if (step) *step = h.step;
    if (time) *time = h.time;
    if (has_matter) *has_matter = h.has_matter;
    if (blocks) {
        if (cap < h.num_blocks) return GRANITE_ERR_TOO_LARGE;
        std::copy(d.begin(), d.end(), blocks);
    }
    return GRANITE_OK;
}

int granite_ccz4_checkpoint_write(void* hc, const char* path, int step, double time) {
    Ctx* c = static_cast<Ctx*>(hc);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit first");
    if (!path) return fail(c, GRANITE_ERR_INVALID, "null path");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(c->stream), "sync");
    CkHeader h{};
    std::memcpy(h.magic, CK_MAGIC, 8);
    h.version = CK_VERSION;
    h.step = step;
    h.num_blocks = (int)c->descs.size();
    h.num_vars = NV;
    h.num_levels = (int)c->level_time.size();
    h.has_matter = c->d_matter ? 1 : 0;
    h.time = time;
    const size_t head = sizeof(h) + c->level_time.size() * sizeof(double) + c->descs.size() * sizeof(granite_block_desc);
    h.data_offset = (uint32_t)((head + 4095) / 4096 * 4096);
    if ((head + 4095) / 4096 * 4096 > UINT32_MAX) return fail(c, GRANITE_ERR_TOO_LARGE, "checkpoint header");
    File f;
    if (!(f.f = std::fopen(path, "wb"))) return fail(c, GRANITE_ERR_INVALID, std::string("cannot create ") + path);
    std::vector<char> pad(h.data_offset - head, 0);
    if (std::fwrite(&h, sizeof(h), 1, f.f) != 1 ||
        (!c->level_time.empty() &&
         std::fwrite(c->level_time.data(), sizeof(double), c->level_time.size(), f.f) != c->level_time.size()) ||
        std::fwrite(c->descs.data(), sizeof(granite_block_desc), c->descs.size(), f.f) != c->descs.size() ||
        (!pad.empty() && std::fwrite(pad.data(), 1, pad.size(), f.f) != pad.size()))
        return fail(c, GRANITE_ERR_INVALID, "checkpoint write failed");
    Pinned pin;
    CK(cudaMallocHost(&pin.p, CK_CHUNK), "cudaMallocHost(checkpoint staging)");
    int r;
    for (size_t i = 0; i < c->descs.size(); ++i)  // block_b/var_v: slot 0 is field-major already
        if ((r = stream_out(c, f.f, reinterpret_cast<const char*>(c->hblocks[i].buf[0]),
                            (size_t)c->hblocks[i].stride * NV * sizeof(double), pin.p)))
            return r;
    if (c->d_matter &&
        (r = stream_out(c, f.f, reinterpret_cast<const char*>(c->d_matter),
                        (size_t)c->matter_cells * NPRIM * sizeof(double), pin.p)))
        return r;
    if (std::fflush(f.f) != 0) return fail(c, GRANITE_ERR_INVALID, "checkpoint write failed");
    return GRANITE_OK;
}

int granite_ccz4_checkpoint_read(void* hc, const char* path, int* step, double* time) {
    Ctx* c = static_cast<Ctx*>(hc);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "add the checkpoint's blocks and commit first");
    if (!path) return fail(c, GRANITE_ERR_INVALID, "null path");
    File f;
    if (!(f.f = std::fopen(path, "rb"))) return fail(c, GRANITE_ERR_INVALID, std::string("cannot open ") + path);
    CkHeader h;
    std::vector<double> lt;
    std::vector<granite_block_desc> d;
    int r = read_header(c, f.f, h, lt, d);
    if (r) return r;
    if (d.size() != c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "checkpoint: block count differs");
    for (size_t i = 0; i < d.size(); ++i) {
        const granite_block_desc &a = d[i], &b = c->descs[i];
        bool same = a.nghost == b.nghost && a.level == b.level;
        for (int k = 0; k < 3; ++k) same = same && a.ncells[k] == b.ncells[k] && a.lo[k] == b.lo[k] && a.hi[k] == b.hi[k];
        if (!same) return fail(c, GRANITE_ERR_INVALID, "checkpoint: block " + std::to_string(i) + " geometry differs");
    }
    if ((h.has_matter != 0) != (c->d_matter != nullptr))
        return fail(c, GRANITE_ERR_INVALID, "checkpoint: matter sources present in one of file and context only");
    if (lt.size() != c->level_time.size()) return fail(c, GRANITE_ERR_INVALID, "checkpoint: level count differs");
    if (std::fseek(f.f, (long)h.data_offset, SEEK_SET) != 0) return fail(c, GRANITE_ERR_INVALID, "checkpoint seek");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(c->stream), "sync");
    Pinned pin;
    CK(cudaMallocHost(&pin.p, CK_CHUNK), "cudaMallocHost(checkpoint staging)");
    for (size_t i = 0; i < c->descs.size(); ++i)
        if ((r = stream_in(c, f.f, reinterpret_cast<char*>(c->hblocks[i].buf[0]),
                           (size_t)c->hblocks[i].stride * NV * sizeof(double), pin.p)))
            return r;
    if (c->d_matter && (r = stream_in(c, f.f, reinterpret_cast<char*>(c->d_matter),
                                      (size_t)c->matter_cells * NPRIM * sizeof(double), pin.p)))
        return r;
    c->level_time = lt;
    for (size_t L = 0; L < c->level_ghosts_valid.size(); ++L) c->level_ghosts_valid[L] = false;
    c->copies_valid = false;  // the state changed outside a pushing coarse step
    if (step) *step = h.step;
    if (time) *time = h.time;
    return GRANITE_OK;
}

// ---------------------------------------------------------------------------
// Psi4 extraction (Psi4Extractor::extract, postprocess.cpp:245-314)
// ---------------------------------------------------------------------------
namespace {

int psi4_run(Ctx* c, const DevBlock& B, const double* u, const double hi[3], const double* radii, int nr, int n_theta,
             int n_phi, int l_max, double* modes, int* npoints) {
    if (!radii || !modes || nr <= 0 || n_theta <= 0 || n_phi <= 0 || l_max < 2 || l_max > 16)
        return fail(c, GRANITE_ERR_INVALID, "psi4: radii, nr > 0, n_theta, n_phi > 0, 2 <= l_max <= 16");
    const long long npts = (long long)nr * n_theta * n_phi;
    if (npts > (1LL << 28)) return fail(c, GRANITE_ERR_TOO_LARGE, "psi4: more than 2^28 sphere points");
    const int nm = (l_max + 1) * (l_max + 1) - 4;
    const size_t b_r = ((size_t)nr * sizeof(double) + 255) / 256 * 256,
                 b_modes = ((size_t)nr * nm * sizeof(double2) + 255) / 256 * 256,
                 b_cnt = ((size_t)nr * sizeof(unsigned int) + 255) / 256 * 256, b_pts = (size_t)npts * sizeof(double2);
    const size_t need = b_r + b_modes + b_cnt + b_pts;
    if (need > c->s_diag_bytes) {
        cudaFree(c->s_diag);
        c->s_diag = nullptr;
        c->s_diag_bytes = 0;
        CK(cudaMalloc(&c->s_diag, need), "cudaMalloc(psi4 scratch)");
        c->s_diag_bytes = need;
    }
    double* d_r = reinterpret_cast<double*>(c->s_diag);
    double2* d_modes = reinterpret_cast<double2*>(c->s_diag + b_r);
    unsigned int* d_cnt = reinterpret_cast<unsigned int*>(c->s_diag + b_r + b_modes);
    double2* d_pts = reinterpret_cast<double2*>(c->s_diag + b_r + b_modes + b_cnt);
    CK(cudaMemcpyAsync(d_r, radii, (size_t)nr * sizeof(double), cudaMemcpyHostToDevice, c->stream), "H2D radii");
    CK(launch_psi4_modes(B, u, hi, d_r, nr, n_theta, n_phi, l_max, d_pts, d_modes, d_cnt, c->stream), "launch psi4");
    CK(cudaMemcpyAsync(modes, d_modes, (size_t)nr * nm * sizeof(double2), cudaMemcpyDeviceToHost, c->stream),
       "D2H modes");
    std::vector<unsigned int> cnt(nr);
    CK(cudaMemcpyAsync(cnt.data(), d_cnt, (size_t)nr * sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream),
       "D2H counts");
    CK(cudaStreamSynchronize(c->stream), "sync");
    if (npoints)
        for (int r = 0; r < nr; ++r) npoints[r] = (int)cnt[r];
    c->launches += 2;
    return GRANITE_OK;
}

}  // namespace

int granite_ccz4_psi4_modes(void* h, int block_index, const double* radii, int nr, int n_theta, int n_phi, int l_max,
                            double* modes, int* npoints) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit first");
    if (block_index < 0 || block_index >= (int)c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "bad block");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const DevBlock& B = c->hblocks[block_index];
    return psi4_run(c, B, B.buf[0], c->descs[block_index].hi, radii, nr, n_theta, n_phi, l_max, modes, npoints);
}

int granite_ccz4_psi4_modes_device(void* h, const granite_block_desc* b, const double* u_dev, const double* radii,
                                   int nr, int n_theta, int n_phi, int l_max, double* modes, int* npoints) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!u_dev) return fail(c, GRANITE_ERR_INVALID, "null device buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    return psi4_run(c, make_devblock(*b, c->p.ko_sigma), u_dev, b->hi, radii, nr, n_theta, n_phi, l_max, modes,
                    npoints);
}

int granite_ccz4_psi4_modes_host(void* h, const granite_block_desc* b, const double* u, const double* radii, int nr,
                                 int n_theta, int n_phi, int l_max, double* modes, int* npoints) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!u) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)cells_of(*b);
    if ((r = ensure_scratch(c, N, 1))) return r;
    CK(cudaMemcpyAsync(c->s_u, u, N * NV * sizeof(double), cudaMemcpyHostToDevice, c->stream), "H2D u");
    return granite_ccz4_psi4_modes_device(c, b, c->s_u, radii, nr, n_theta, n_phi, l_max, modes, npoints);
}

// ---------------------------------------------------------------------------
// Apparent horizons (ApparentHorizonFinder, horizon_finder.cpp:310-507)
// ---------------------------------------------------------------------------
namespace {

constexpr double HZ_PI = 3.14159265358979323846;  // constants::PI
constexpr int HZ_CHUNK = 16;                      // flow iterations per launch
constexpr unsigned int HZ_MAX_CANDIDATES = 65536;

// the next 256-byte aligned piece of `bytes` bytes of a scratch area
char* carve(char*& p, size_t bytes) {
    char* r = p;
    p += (bytes + 255) / 256 * 256;
    return r;
}

int diag_scratch(Ctx* c, size_t need) {
    if (need > c->s_diag_bytes) {
        cudaFree(c->s_diag);
        c->s_diag = nullptr;
        c->s_diag_bytes = 0;
        CK(cudaMalloc(&c->s_diag, need), "cudaMalloc(diagnostics scratch)");
        c->s_diag_bytes = need;
    }
    return GRANITE_OK;
}

int horizon_run(Ctx* c, const DevBlock& B, const double* u, const granite_horizon_params* p, const double* center,
                granite_horizon* out, double* radii_out) {
    if (!p || !center || !out) return fail(c, GRANITE_ERR_INVALID, "horizon: null argument");
    if (p->angular_resolution <= 0 || p->angular_resolution > 2048 || p->max_iterations < 0)
        return fail(c, GRANITE_ERR_INVALID, "horizon: 0 < angular_resolution <= 2048, max_iterations >= 0");
    const int nth = p->angular_resolution, nph = 2 * nth, N = nth * nph;
    HorizonArgs a;
    for (int d = 0; d < 3; ++d) a.center[d] = center[d];
    const double h_grid = B.dx[0];
    a.flow_step = 0.05 * h_grid;
    a.rmin = 1.0e-6 * h_grid;
    a.dth = HZ_PI / nth;
    a.dph = 2.0 * HZ_PI / nph;
    a.nth = nth;
    a.nph = nph;
    // angular tables from the host libm, as buildAngularGrid + std::sin / std::cos
    std::vector<double> tab(2 * nth + 2 * nph);
    for (int i = 0; i < nth; ++i) {
        const double th = HZ_PI * (i + 0.5) / nth;
        tab[i] = std::sin(th);
        tab[nth + i] = std::cos(th);
    }
    for (int j = 0; j < nph; ++j) {
        const double ph = 2.0 * HZ_PI * j / nph;
        tab[2 * nth + j] = std::sin(ph);
        tab[2 * nth + nph + j] = std::cos(ph);
    }
    // five pieces, each rounded up to 256 bytes by carve()
    const size_t need = 5 * 256 + (tab.size() + (size_t)N + (size_t)HZ_CHUNK * N + 3 * (size_t)N + HZ_CHUNK) * 8;
    int r = diag_scratch(c, need);
    if (r) return r;
    char* q = c->s_diag;
    double* d_tab = reinterpret_cast<double*>(carve(q, tab.size() * 8));
    double* d_h = reinterpret_cast<double*>(carve(q, (size_t)N * 8));
    double* d_hist = reinterpret_cast<double*>(carve(q, (size_t)HZ_CHUNK * N * 8));
    double* d_terms = reinterpret_cast<double*>(carve(q, 3 * (size_t)N * 8));
    unsigned long long* d_itmax = reinterpret_cast<unsigned long long*>(carve(q, HZ_CHUNK * 8));
    std::vector<double> h(N, p->initial_guess_radius);
    CK(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, c->stream), "H2D tables");
    CK(cudaMemcpyAsync(d_h, h.data(), (size_t)N * 8, cudaMemcpyHostToDevice, c->stream), "H2D radii");
    int converged = -1, done = 0;
    while (done < p->max_iterations && converged < 0) {
        const int it = std::min(HZ_CHUNK, p->max_iterations - done);
        CK(launch_horizon_flow(B, u, a, d_tab, d_h, it, d_hist, d_itmax, c->stream), "launch horizon flow");
        unsigned long long mx[HZ_CHUNK];
        CK(cudaMemcpyAsync(mx, d_itmax, it * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream),
           "D2H flow maxima");
        CK(cudaStreamSynchronize(c->stream), "sync");
        c->launches += 1;
        for (int k = 0; k < it && converged < 0; ++k) {
            double v;
            std::memcpy(&v, &mx[k], 8);
            if (v < p->tolerance) {  // the radii of this iteration are the result
                converged = done + k + 1;
                CK(cudaMemcpyAsync(d_h, d_hist + (size_t)k * N, (size_t)N * 8, cudaMemcpyDeviceToDevice, c->stream),
                   "converged radii");
            }
        }
        done += it;
    }
    *out = granite_horizon{};
    out->iterations = converged > 0 ? converged : done;
    for (int d = 0; d < 3; ++d) out->centroid[d] = center[d];
    CK(cudaMemcpyAsync(h.data(), d_h, (size_t)N * 8, cudaMemcpyDeviceToHost, c->stream), "D2H radii");
    CK(cudaStreamSynchronize(c->stream), "sync");
    if (radii_out) std::copy(h.begin(), h.end(), radii_out);
    if (converged < 0) {
        for (int d = 0; d < 3; ++d) out->centroid[d] = 0.0;
        return GRANITE_OK;
    }
    std::vector<double> terms(3 * (size_t)N);
    CK(launch_horizon_surface(B, u, a, d_tab, d_h, d_terms, c->stream), "launch horizon surface");
    CK(cudaMemcpyAsync(terms.data(), d_terms, terms.size() * 8, cudaMemcpyDeviceToHost, c->stream), "D2H terms");
    CK(cudaStreamSynchronize(c->stream), "sync");
    c->launches += 1;
    double area = 0.0, jz = 0.0;  // sums in the reference's point order
    for (int k = 0; k < N; ++k)
        if (terms[3 * k + 2] != 0.0) {
            area += terms[3 * k];
            jz += terms[3 * k + 1];
        }
    out->found = 1;
    out->area = area;
    out->irreducible_mass = std::sqrt(area / (16.0 * HZ_PI));
    double ceq = 0.0, cpol = 0.0;
    for (int j = 0; j < nph; ++j) ceq += h[(size_t)(nth / 2) * nph + j] * a.dph;
    for (int i = 0; i < nth; ++i) cpol += h[(size_t)i * nph] * a.dth;
    out->circumference_equatorial = ceq;
    out->circumference_polar = 2.0 * cpol;
    const double m = out->irreducible_mass;
    const double spin = m > 1.0e-12 ? jz / (m * m) : 0.0;
    out->spin = std::clamp(spin, -1.0, 1.0);
    return GRANITE_OK;
}

}  // namespace

void granite_ccz4_default_horizon_params(granite_horizon_params* p) {
    if (!p) return;
    p->max_iterations = 200;
    p->tolerance = 1.0e-10;
    p->angular_resolution = 50;
    p->initial_guess_radius = 1.0;
}

int granite_ccz4_find_horizon(void* h, int block_index, const granite_horizon_params* p, const double* center,
                              granite_horizon* out, double* radii) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit first");
    if (block_index < 0 || block_index >= (int)c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "bad block");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const DevBlock& B = c->hblocks[block_index];
    return horizon_run(c, B, B.buf[0], p, center, out, radii);
}

int granite_ccz4_find_horizon_host(void* h, const granite_block_desc* b, const double* u,
                                   const granite_horizon_params* p, const double* center, granite_horizon* out,
                                   double* radii) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    int r = check_desc(c, b);
    if (r) return r;
    if (!u) return fail(c, GRANITE_ERR_INVALID, "null host buffer");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t N = (size_t)cells_of(*b);
    if ((r = ensure_scratch(c, N, 1))) return r;
    CK(cudaMemcpyAsync(c->s_u, u, N * NV * sizeof(double), cudaMemcpyHostToDevice, c->stream), "H2D u");
    DevBlock B = make_devblock(*b, c->p.ko_sigma);
    B.buf[0] = c->s_u;
    return horizon_run(c, B, c->s_u, p, center, out, radii);
}

int granite_ccz4_find_all_horizons(void* h, int block_index, const granite_horizon_params* p, granite_horizon* out,
                                   int cap, int* n) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (!c->committed) return fail(c, GRANITE_ERR_INVALID, "commit first");
    if (block_index < 0 || block_index >= (int)c->descs.size()) return fail(c, GRANITE_ERR_INVALID, "bad block");
    if (!p || !n || cap < 0 || (cap > 0 && !out)) return fail(c, GRANITE_ERR_INVALID, "horizon: null argument");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const DevBlock& B = c->hblocks[block_index];
    const granite_block_desc& d = c->descs[block_index];
    // candidate scan: indices, then count, in a scratch of their own (the flow reuses the diagnostics scratch)
    long long* d_idx = nullptr;
    CK(cudaMalloc(&d_idx, HZ_MAX_CANDIDATES * sizeof(long long) + 256), "cudaMalloc(candidates)");
    unsigned int* d_cnt = reinterpret_cast<unsigned int*>(d_idx + HZ_MAX_CANDIDATES);
    cudaError_t e = launch_lapse_minima(B, B.buf[0], d_idx, d_cnt, HZ_MAX_CANDIDATES, c->stream);
    unsigned int cnt = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    std::vector<long long> idx(std::min(cnt, HZ_MAX_CANDIDATES));
    if (e == cudaSuccess && !idx.empty())
        e = cudaMemcpy(idx.data(), d_idx, idx.size() * sizeof(long long), cudaMemcpyDeviceToHost);
    cudaFree(d_idx);
    if (e != cudaSuccess) return cuda_fail(c, e, "lapse minima");
    if (cnt > HZ_MAX_CANDIDATES) return fail(c, GRANITE_ERR_TOO_LARGE, "horizon: more than 65536 lapse minima");
    c->launches += 1;
    std::sort(idx.begin(), idx.end());  // the reference's k, j, i scan order
    const double min_sep = 2.0 * p->initial_guess_radius;
    std::vector<std::array<double, 3>> uniq;
    for (long long ci : idx) {
        const int i = (int)(ci % B.tx), j = (int)((ci / B.tx) % B.ty), k = (int)(ci / ((long long)B.tx * B.ty));
        const std::array<double, 3> x = {xref(d, 0, i), xref(d, 1, j), xref(d, 2, k)};
        bool dup = false;
        for (const auto& w : uniq) {
            const double d2 = (x[0] - w[0]) * (x[0] - w[0]) + (x[1] - w[1]) * (x[1] - w[1]) +
                (x[2] - w[2]) * (x[2] - w[2]);
            if (d2 < min_sep * min_sep) {
                dup = true;
                break;
            }
        }
        if (!dup) uniq.push_back(x);
    }
    int found = 0;
    for (const auto& ctr : uniq) {
        granite_horizon hz;
        int r = horizon_run(c, B, B.buf[0], p, ctr.data(), &hz, nullptr);
        if (r) return r;
        if (!hz.found) continue;
        hz.id = found;
        if (found < cap) out[found] = hz;
        ++found;
    }
    *n = found;
    return GRANITE_OK;
}

}  // extern "C"
