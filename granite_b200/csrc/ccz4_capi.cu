// ccz4_capi.cu -- implementation of the C ABI in include/granite_ccz4.h.
//
// Host runtime: one context = one device + one stream + one device arena for
// all resident blocks (three 22-field buffers per block: state and two RK
// stage buffers), per-level tile work-lists for the batched RHS launches,
// ghost-cell chunk lists for the fills, and a cache of CUDA graphs, one per
// (level, precision, boundary, dt) step shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/granite_ccz4.h"
#include "ccz4_common.cuh"
#include "ccz4_kernels.h"

using namespace granite_b200;

namespace {

struct Graph {
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;
};

struct LevelLists {
    std::vector<int> blocks;
    Tile* d_tiles = nullptr;   // stage-kernel tiles (shape of the context's variant)
    int ntiles = 0;
    Tile* d_mtiles = nullptr;  // constraint-monitor tiles (variant-0 shape)
    int nmtiles = 0;
    GhostItem* d_ghost = nullptr;
    int nghost = 0;
    long long interior_points = 0;
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
    int variant = VARIANT_SMEM;  // stage-kernel variant (granite_ccz4_set_kernel_variant)
    cudaStream_t stream = nullptr;
    std::string err;
    long long launches = 0;
    unsigned long long* d_nonfinite = nullptr;

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
    std::map<std::tuple<int, int, int, unsigned long long, int>, Graph> graphs;

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
    if (cells_of(*b) * NV > (1ll << 40)) return fail(c, GRANITE_ERR_INVALID, "block too large");
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

void tiles_of(int block, const granite_block_desc& b, std::vector<Tile>& out, int variant) {
    int TX, TY, TZ;
    stage_tile_dims(variant, &TX, &TY, &TZ);
    for (int k = 0; k < b.ncells[2]; k += TZ)
        for (int j = 0; j < b.ncells[1]; j += TY)
            for (int i = 0; i < b.ncells[0]; i += TX) out.push_back(Tile{block, i, j, k});
}

long long ghost_count(const granite_block_desc& b) {
    return cells_of(b) - (long long)b.ncells[0] * b.ncells[1] * b.ncells[2];
}

void ghost_chunks_of(int block, const granite_block_desc& b, std::vector<GhostItem>& out) {
    const long long n = ghost_count(b);
    for (long long r = 0; r < n; r += 256) out.push_back(GhostItem{block, (int)r});
}

StageArgs base_args(const Ctx* c) {
    StageArgs a{};
    a.ko_on = c->p.ko_sigma > 0.0 ? 1 : 0;
    a.chi_c = c->p.chi_blend_center;
    a.chi_w = c->p.chi_blend_width;
    a.kappa1 = c->p.kappa1;
    a.kappa2 = c->p.kappa2;
    a.eta = c->p.eta;
    a.nonfinite = c->d_nonfinite;
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
        CK(cudaMalloc(&c->s_mat, cells * 11 * sizeof(double)), "cudaMalloc(scratch matter)");
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

// Stage one block into the stateless scratch: descriptor + tile list.
int stage_single(Ctx* c, const granite_block_desc* b, double* u_dev, int* ntiles, cudaStream_t s, int variant) {
    std::vector<Tile> t;
    tiles_of(0, *b, t, variant);
    int r = ensure_scratch(c, (size_t)cells_of(*b), (int)t.size());
    if (r) return r;
    DevBlock d = make_devblock(*b, c->p.ko_sigma);
    d.buf[0] = u_dev ? u_dev : c->s_u;
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

int granite_ccz4_set_kernel_variant(void* h, int variant) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (variant < 0 || variant >= NUM_VARIANTS) return fail(c, GRANITE_ERR_INVALID, "unknown kernel variant");
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "set the kernel variant before commit");
    c->variant = variant;
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
    c->p = *p;
    c->device = p->device;
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = configure_stage_kernels();
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_nonfinite, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(c->d_nonfinite, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&c->s_desc, sizeof(DevBlock));
    if (e == cudaSuccess) e = cudaMalloc(&c->s_sum, 2 * sizeof(double));
    if (e != cudaSuccess) {
        granite_ccz4_destroy(c);
        return e == cudaErrorMemoryAllocation ? GRANITE_ERR_NOMEM : GRANITE_ERR_CUDA;
    }
    *out = c;
    return GRANITE_OK;
}

int granite_ccz4_destroy(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto& kv : c->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto& p : c->pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : c->event_pool) cudaEventDestroy(e);
    for (auto& L : c->levels) {
        cudaFree(L.d_tiles);
        cudaFree(L.d_mtiles);
        cudaFree(L.d_ghost);
    }
    cudaFree(c->d_blocks);
    cudaFree(c->arena);
    cudaFree(c->s_u);
    cudaFree(c->s_rhs);
    cudaFree(c->s_mat);
    cudaFree(c->s_desc);
    cudaFree(c->s_tiles);
    cudaFree(c->s_partials);
    cudaFree(c->s_sum);
    cudaFree(c->d_nonfinite);
    if (c->stream) cudaStreamDestroy(c->stream);
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

int granite_ccz4_sync(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    CK(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    return GRANITE_OK;
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
    int nt = 0;
    if ((r = stage_single(c, b, const_cast<double*>(u_dev), &nt, s, c->variant))) return r;
    StageArgs a = base_args(c);
    a.in_sel = 0;
    a.rhs = rhs_dev;
    a.rho = rho;
    a.Si = Si;
    a.Sij = Sij;
    a.S = S;
    CK(launch_stage(c->variant, precision, EPI_STORE, c->s_desc, c->s_tiles, nt, a, s), "launch RHS");
    c->launches += 1;
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
    return GRANITE_OK;
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

int granite_ccz4_commit(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    if (c->committed) return fail(c, GRANITE_ERR_INVALID, "already committed");
    if (c->descs.empty()) return fail(c, GRANITE_ERR_INVALID, "no blocks");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    // arena: 3 buffers per block, each 256-byte aligned
    std::vector<size_t> off(c->descs.size());
    size_t total = 0;
    for (size_t i = 0; i < c->descs.size(); ++i) {
        off[i] = total;
        const size_t one = ((size_t)cells_of(c->descs[i]) * NV * sizeof(double) + 255) / 256 * 256;
        total += 3 * one;
    }
    CK(cudaMalloc(&c->arena, total), "cudaMalloc(arena)");
    c->arena_bytes = total;
    int maxlev = 0;
    c->hblocks.resize(c->descs.size());
    for (size_t i = 0; i < c->descs.size(); ++i) {
        DevBlock d = make_devblock(c->descs[i], c->p.ko_sigma);
        const size_t one = ((size_t)cells_of(c->descs[i]) * NV * sizeof(double) + 255) / 256 * 256;
        for (int sl = 0; sl < 3; ++sl) d.buf[sl] = reinterpret_cast<double*>(c->arena + off[i] + sl * one);
        c->hblocks[i] = d;
        maxlev = std::max(maxlev, c->descs[i].level);
    }
    CK(cudaMemsetAsync(c->arena, 0, total, c->stream), "memset arena");
    CK(upload_vec(c->hblocks, &c->d_blocks, c->stream), "upload block table");
    c->levels.assign(maxlev + 1, LevelLists());
    c->level_ghosts_valid.assign(maxlev + 1, false);
    for (int L = 0; L <= maxlev; ++L) {
        std::vector<Tile> tiles, mtiles;
        std::vector<GhostItem> ghosts;
        LevelLists& ll = c->levels[L];
        for (size_t i = 0; i < c->descs.size(); ++i) {
            if (c->descs[i].level != L) continue;
            ll.blocks.push_back((int)i);
            tiles_of((int)i, c->descs[i], tiles, c->variant);
            tiles_of((int)i, c->descs[i], mtiles, VARIANT_GLOBAL);
            ghost_chunks_of((int)i, c->descs[i], ghosts);
            ll.interior_points += (long long)c->descs[i].ncells[0] * c->descs[i].ncells[1] * c->descs[i].ncells[2];
        }
        CK(upload_vec(tiles, &ll.d_tiles, c->stream), "upload tiles");
        CK(upload_vec(mtiles, &ll.d_mtiles, c->stream), "upload monitor tiles");
        ll.nmtiles = (int)mtiles.size();
        CK(upload_vec(ghosts, &ll.d_ghost, c->stream), "upload ghost chunks");
        ll.ntiles = (int)tiles.size();
        ll.nghost = (int)ghosts.size();
    }
    int maxt = 0;
    for (auto& L : c->levels) maxt = std::max(maxt, std::max(L.ntiles, L.nmtiles));
    int r = ensure_scratch(c, 1, std::max(1, maxt));
    if (r) return r;
    c->committed = true;
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
    return GRANITE_OK;
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
    return GRANITE_OK;
}

// ---------------------------------------------------------------------------
// stepping
// ---------------------------------------------------------------------------

static cudaError_t enqueue_level_step(Ctx* c, int level, double dt, int precision, int bc, bool prefill,
                                      long long* nl) {
    LevelLists& L = c->levels[level];
    const int level_mode = (bc == GRANITE_BC_PERIODIC) ? GHOST_PERIODIC : GHOST_ZERO_GRADIENT;
    const int outer_mode = (bc == GRANITE_BC_PERIODIC) ? GHOST_PERIODIC : GHOST_SOMMERFELD;
    cudaStream_t s = c->stream;
    cudaError_t e;
    long long n = 0;
    // amr.cpp:319 level fill before the step (only when the state changed since the last one)
    if (prefill) {
        if ((e = timed(c, GRANITE_KERNEL_GHOST, [&] { return launch_ghost_fill(level_mode, c->d_blocks, L.d_ghost, L.nghost, 0, s); }))) return e;
        ++n;
    }
    StageArgs a = base_args(c);
    // stage 1: u1 = u + dt L(u)                       main.cpp:673
    a.in_sel = 0; a.n_sel = 0; a.out_sel = 1; a.final_stage = 0;
    a.a1 = 1.0; a.a2 = 0.0; a.a3dt = 1.0 * dt;
    if ((e = timed(c, GRANITE_KERNEL_STAGE, [&] { return launch_stage(c->variant, precision, EPI_RK, c->d_blocks, L.d_tiles, L.ntiles, a, s); }))) return e;
    if ((e = timed(c, GRANITE_KERNEL_GHOST, [&] { return launch_ghost_fill(outer_mode, c->d_blocks, L.d_ghost, L.nghost, 1, s); }))) return e;
    // stage 2: u2 = 3/4 u + 1/4 u1 + 1/4 dt L(u1)      main.cpp:679
    a.in_sel = 1; a.n_sel = 0; a.out_sel = 2;
    a.a1 = 0.75; a.a2 = 0.25; a.a3dt = 0.25 * dt;
    if ((e = timed(c, GRANITE_KERNEL_STAGE, [&] { return launch_stage(c->variant, precision, EPI_RK, c->d_blocks, L.d_tiles, L.ntiles, a, s); }))) return e;
    if ((e = timed(c, GRANITE_KERNEL_GHOST, [&] { return launch_ghost_fill(outer_mode, c->d_blocks, L.d_ghost, L.nghost, 2, s); }))) return e;
    // stage 3: u = 1/3 u + 2/3 u2 + 2/3 dt L(u2), floors, det/trace   main.cpp:685-687
    a.in_sel = 2; a.n_sel = 0; a.out_sel = 0; a.final_stage = 1;
    a.a1 = 1.0 / 3.0; a.a2 = 2.0 / 3.0; a.a3dt = (2.0 / 3.0) * dt;
    if ((e = timed(c, GRANITE_KERNEL_STAGE, [&] { return launch_stage(c->variant, precision, EPI_RK, c->d_blocks, L.d_tiles, L.ntiles, a, s); }))) return e;
    // main.cpp:689 outer BC on u is overwritten by the level fill of amr.cpp:329,
    // so only the level fill runs.
    if ((e = timed(c, GRANITE_KERNEL_GHOST, [&] { return launch_ghost_fill(level_mode, c->d_blocks, L.d_ghost, L.nghost, 0, s); }))) return e;
    n += 6;
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
    const bool prefill = !c->level_ghosts_valid[level];
    if (c->profiling) {
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

int granite_ccz4_hierarchy_step(void* h, double dt_coarse, int precision, int amr_mode) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return GRANITE_ERR_INVALID;
    (void)dt_coarse;
    (void)precision;
    (void)amr_mode;
    return fail(c, GRANITE_ERR_UNSUPPORTED, "hierarchy_step: not built yet");
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

}  // extern "C"
