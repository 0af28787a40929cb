// ccz4_rhs.cu -- fused CCZ4 RHS + Kreiss-Oliger + SSP-RK3 stage kernels
// (global-load and cp.async variants), the per-tile precision classifier, the
// stage-kernel launchers and the standalone KO kernel.
//
// One thread per interior point; one CTA per tile of a block; the launch walks
// a work-list of tiles over every block of an AMR level, so blocks of uneven
// size share one launch per RK stage. The per-point body is ccz4_point
// (ccz4_point.cuh); the TMA-ring variant is in ccz4_stage_tma.cuh, instantiated
// per tuning configuration in ccz4_tma_cfg<k>.cu.
//
// Per-tile precision: a launch can be restricted to the tiles of a flag array
// (classify_tiles_kernel marks the tiles with a point of chi below a threshold,
// near a puncture): the FP64 kernel takes those tiles and the FP32 kernel the
// others, both walking the tile list in its spatial order.
//
// Control flow: the per-point body is one straight-line sequence (the KO term
// is always evaluated -- its weights sigma/(64 dx) w_s are zero when KO is off
// -- and the upwind side is a select, not a branch), so the compiler can
// schedule the stencil loads of later fields across earlier ones.
#include "ccz4_common.cuh"
#include "ccz4_kernels.h"
#include "ccz4_point.cuh"
#include "ccz4_stencil.cuh"

namespace granite_b200 {

namespace {

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Tile staging geometry: a TX x TY x TZ tile of points plus the cells its
// stencils touch (the tile grown by 1 in every direction for the mixed
// derivatives, and arms of 3 more cells along each axis for the +-4 reach),
// laid out in shared memory as a (TX+8) x (TY+8) x (TZ+8) box.
template <int TX, int TY, int TZ>
struct TileGeom {
    static constexpr int BX = TX + 8, BY = TY + 8, BZ = TZ + 8;
    static constexpr int BOX = BX * BY * BZ;
    static constexpr int N_CORE = (TX + 2) * (TY + 2) * (TZ + 2);
    static constexpr int N_XARM = 6 * TY * TZ, N_YARM = 6 * TX * TZ, N_ZARM = 6 * TX * TY;
    static constexpr int NLOAD = N_CORE + N_XARM + N_YARM + N_ZARM;
    // cell q of the load list -> offset (rx, ry, rz) from the tile origin
    __device__ static void cell(int q, int& rx, int& ry, int& rz) {
        constexpr int ARM[6] = {-4, -3, -2, 1, 2, 3};
        if (q < N_CORE) {
            rx = q % (TX + 2) - 1;
            ry = (q / (TX + 2)) % (TY + 2) - 1;
            rz = q / ((TX + 2) * (TY + 2)) - 1;
            return;
        }
        q -= N_CORE;
        if (q < N_XARM) {
            const int a = q % 6;
            rx = a < 3 ? ARM[a] : TX + ARM[a];
            ry = (q / 6) % TY;
            rz = q / (6 * TY);
            return;
        }
        q -= N_XARM;
        if (q < N_YARM) {
            const int a = (q / TX) % 6;
            rx = q % TX;
            ry = a < 3 ? ARM[a] : TY + ARM[a];
            rz = q / (6 * TX);
            return;
        }
        q -= N_YARM;
        const int a = q / (TX * TY);
        rx = q % TX;
        ry = (q / TX) % TY;
        rz = a < 3 ? ARM[a] : TZ + ARM[a];
    }
};

// Stencils read from a CTA-staged shared-memory tile. Fields are copied in
// FIELD_ORDER with cp.async into NBUF rotating buffers, NBUF-1 fields ahead of
// the one being differentiated, so the copies of the next fields overlap the
// algebra of the current one. Every thread of the CTA must call der() for
// every field in order (the calls carry the CTA barrier).
template <int TX, int TY, int TZ, int NBUF>
struct SmemSource {
    static constexpr bool HS = false, UNROLL = false;
    using G = TileGeom<TX, TY, TZ>;
    const DevBlock& B;
    const double* __restrict__ u;  // stencil buffer (global)
    double* sm;                    // NBUF x BOX doubles
    const int2* table;             // NLOAD x {smem offset or -1, global offset from the tile origin}
    long long origin;              // global cell index of the tile origin
    int lin;                       // shared offset of this thread's point in a box
    int next;                      // index in FIELD_ORDER of the next field to consume

    __device__ __forceinline__ void issue(int k) {
        if (k < NV) {
            double* dst = sm + (k % NBUF) * G::BOX;
            const double* src = u + (long long)FIELD_ORDER[k] * B.stride + origin;
            for (int q = threadIdx.x; q < G::NLOAD; q += TX * TY * TZ) {
                const int2 e = table[q];
                if (e.x >= 0) cp_async8(dst + e.x, src + e.y);
            }
        }
        cp_async_commit();
    }
    __device__ __forceinline__ void start() {
        for (int k = 0; k < NBUF - 1; ++k) issue(k);
    }
    template <bool HESS, bool EXACT, typename P>
    __device__ __forceinline__ FieldDer<P> der(int /*v*/, const double beta[3], P w) {
        cp_async_wait<NBUF - 2>();
        __syncthreads();
        issue(next + NBUF - 1);
        const long long off[3] = {1, G::BX, G::BX * G::BY};
        const SharedLoad L{sm + (next % NBUF) * G::BOX + lin};
        ++next;
        return field_der_l<P, HESS, true, SharedLoad, EXACT>(B, L, off, beta, w);
    }
};

}  // namespace

// Variants 0, 2, 3: stencils from global memory, one thread per point; MINB
// resident CTAs per SM requested from the register allocator (1: up to 255
// registers, 3: up to 168, 4: up to 128).
template <int PM, int EPI, int TX, int TY, int TZ, int MINB>
__global__ void __launch_bounds__(TX* TY* TZ, MINB)
    ccz4_stage_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, StageArgs A) {
    if (!tile_selected(A.tile_prec, A.want_prec, blockIdx.x)) return;
    const Tile t = tiles[blockIdx.x];
    const DevBlock& B = blocks[t.block];
    // 128 threads over a w x (128 / w) tile; w matches the block width (x fastest)
    const int tid = threadIdx.x + TX * (threadIdx.y + TY * threadIdx.z);
    const int w = t.w > 0 ? t.w : TX;
    const int i = t.i0 + tid % w, j = t.j0 + tid / w, k = t.k0;
    if (i >= B.n[0] || j >= B.n[1] || k >= B.n[2]) return;
    const long long c = cell_index(B, i + NG, j + NG, k + NG);
    const double* __restrict__ uin = B.buf[A.in_sel];
    GlobalSource S{B, uin, c};
    AlgebraT<PM> L[NV];
    point_pm<PM>(B, uin, c, A, S, L);
    stage_epilogue<EPI>(B, A, c, L);
}

// Variant 1: every field of the tile (with its stencil halo) staged through
// shared memory by cp.async, NBUF-1 fields ahead of the computation.
template <int PM, int EPI, int TX, int TY, int TZ, int NBUF>
__global__ void __launch_bounds__(TX* TY* TZ, 2)
    ccz4_stage_smem_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, StageArgs A) {
    using G = TileGeom<TX, TY, TZ>;
    constexpr int NT = TX * TY * TZ;
    extern __shared__ __align__(16) double smem[];
    int2* table = reinterpret_cast<int2*>(smem + NBUF * G::BOX);
    if (!tile_selected(A.tile_prec, A.want_prec, blockIdx.x)) return;
    const Tile t = tiles[blockIdx.x];
    const DevBlock& B = blocks[t.block];
    const int tid = threadIdx.x;
    const int lx = tid % TX, ly = (tid / TX) % TY, lz = tid / (TX * TY);
    const int i = t.i0 + lx, j = t.j0 + ly, k = t.k0 + lz;
    const bool valid = i < B.n[0] && j < B.n[1] && k < B.n[2];
    // load list of this tile: shared offset (or -1 outside the block) and global offset
    const int gi0 = t.i0 + NG, gj0 = t.j0 + NG, gk0 = t.k0 + NG;
    const int row = B.tx, plane = B.tx * B.ty;
    for (int q = tid; q < G::NLOAD; q += NT) {
        int rx, ry, rz;
        G::cell(q, rx, ry, rz);
        const bool in = gi0 + rx < B.tx && gj0 + ry < B.ty && gk0 + rz < B.tz;
        table[q] = make_int2(in ? (rx + 4) + G::BX * ((ry + 4) + G::BY * (rz + 4)) : -1, rx + row * ry + plane * rz);
    }
    __syncthreads();
    const double* __restrict__ uin = B.buf[A.in_sel];
    SmemSource<TX, TY, TZ, NBUF> S{B, uin, smem, table, cell_index(B, gi0, gj0, gk0),
                                      (lx + 4) + G::BX * ((ly + 4) + G::BY * (lz + 4)), 0};
    S.start();
    // pointwise loads of threads outside the block use a valid cell; their results are dropped
    const int ic = i < B.n[0] ? i : B.n[0] - 1, jc = j < B.n[1] ? j : B.n[1] - 1, kc = k < B.n[2] ? k : B.n[2] - 1;
    const long long c = cell_index(B, ic + NG, jc + NG, kc + NG);
    AlgebraT<PM> L[NV];
    point_pm<PM>(B, uin, c, A, S, L);
    if (!valid) return;  // no barrier follows the last field
    stage_epilogue<EPI>(B, A, c, L);
}

// Per-tile precision flags: flag[ti] = 1 (FP64 algebra) when a point of tile ti
// has chi below chi_fp64 in buffer slot `sel` (or a non-finite chi), else 0.
// One warp per tile, CLASSIFY_WARPS tiles per CTA (a CTA per tile made the
// launch block-scheduling bound: ~16 k CTAs of one load per thread).
constexpr int CLASSIFY_WARPS = 8;
__global__ void __launch_bounds__(32 * CLASSIFY_WARPS)
    classify_tiles_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int first, int ntiles,
                          int sel, int tx, int ty, int tz, double chi_fp64, unsigned char* __restrict__ flag) {
    const int lane = threadIdx.x % 32;
    const int tl = blockIdx.x * CLASSIFY_WARPS + (int)threadIdx.x / 32;
    if (tl >= ntiles) return;  // whole warps
    const int ti = first + tl;
    const Tile t = tiles[ti];
    const DevBlock& B = blocks[t.block];
    // global-load tiles: w x 128/w x 1; TMA x-remainder tiles (w < 0): -w x ty x 2 tz
    const int w = t.w > 0 ? t.w : (t.w < 0 ? -t.w : tx), h = t.w > 0 ? 128 / t.w : ty,
              d = t.w > 0 ? 1 : (t.w < 0 ? 2 * tz : tz);
    const double* chi = B.buf[sel] + (long long)CHI * B.stride;
    bool low = false;
#pragma unroll 4
    for (int p = lane; p < w * h * d; p += 32) {
        const int i = t.i0 + p % w, j = t.j0 + (p / w) % h, k = t.k0 + p / (w * h);
        if (i < B.n[0] && j < B.n[1] && k < B.n[2])
            low |= !(__ldg(chi + cell_index(B, i + NG, j + NG, k + NG)) >= chi_fp64);
    }
    low = __any_sync(0xffffffffu, low);
    if (lane == 0) flag[ti] = low ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
constexpr int V0_TX = 32, V0_TY = 4, V0_TZ = 1;
constexpr int V1_TX = 16, V1_TY = 4, V1_TZ = 2, V1_NBUF = 3;

int stage_tile_dims(int variant, int cfg, int* tx, int* ty, int* tz) {
    if (variant == VARIANT_TMA) {
        if (cfg < 0 || cfg >= NUM_TMA_CFGS) return -1;
        *tx = 16;
        *ty = 4;
        *tz = TMA_CFGS[cfg].tz;
    } else if (variant == 1) {
        *tx = V1_TX;
        *ty = V1_TY;
        *tz = V1_TZ;
    } else {
        *tx = V0_TX;
        *ty = V0_TY;
        *tz = V0_TZ;
    }
    return 0;
}

template <int PM, int EPI>
static cudaError_t launch_smem(const DevBlock* blocks, const Tile* tiles, int ntiles, const StageArgs& args,
                               cudaStream_t stream) {
    using G = TileGeom<V1_TX, V1_TY, V1_TZ>;
    constexpr size_t bytes = V1_NBUF * G::BOX * sizeof(double) + G::NLOAD * sizeof(int2);
    auto k = ccz4_stage_smem_kernel<PM, EPI, V1_TX, V1_TY, V1_TZ, V1_NBUF>;
    k<<<ntiles, V1_TX * V1_TY * V1_TZ, bytes, stream>>>(blocks, tiles, args);
    return cudaGetLastError();
}

template <int PM, int EPI>
static cudaError_t configure_smem() {
    using G = TileGeom<V1_TX, V1_TY, V1_TZ>;
    constexpr size_t bytes = V1_NBUF * G::BOX * sizeof(double) + G::NLOAD * sizeof(int2);
    return cudaFuncSetAttribute(ccz4_stage_smem_kernel<PM, EPI, V1_TX, V1_TY, V1_TZ, V1_NBUF>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// The TMA configurations, one translation unit each (ccz4_tma_cfg<k>.cu).
using TmaConfigure = cudaError_t (*)(int nsm, int grids[3][2][2]);
using TmaLaunch = cudaError_t (*)(int pm, int epi, bool sel, const DevBlock* blocks, const Tile* tiles, int ntiles,
                                  const StageArgs& args, cudaStream_t stream, int grid);
cudaError_t configure_tma_cfg0(int, int[3][2][2]);
cudaError_t configure_tma_cfg1(int, int[3][2][2]);
cudaError_t configure_tma_cfg2(int, int[3][2][2]);
cudaError_t configure_tma_cfg3(int, int[3][2][2]);
cudaError_t configure_tma_cfg4(int, int[3][2][2]);
cudaError_t configure_tma_cfg5(int, int[3][2][2]);
cudaError_t configure_tma_cfg6(int, int[3][2][2]);
cudaError_t configure_tma_cfg7(int, int[3][2][2]);
cudaError_t configure_tma_cfg8(int, int[3][2][2]);
cudaError_t configure_tma_cfg9(int, int[3][2][2]);
cudaError_t configure_tma_cfg10(int, int[3][2][2]);
cudaError_t configure_tma_cfg11(int, int[3][2][2]);
cudaError_t configure_tma_cfg12(int, int[3][2][2]);
cudaError_t configure_tma_cfg13(int, int[3][2][2]);
cudaError_t configure_tma_cfg14(int, int[3][2][2]);
cudaError_t configure_tma_cfg15(int, int[3][2][2]);
cudaError_t configure_tma_cfg16(int, int[3][2][2]);
cudaError_t configure_tma_cfg17(int, int[3][2][2]);
cudaError_t launch_tma_cfg0(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg1(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg2(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg3(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg4(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg5(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg6(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg7(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg8(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg9(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg10(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg11(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg12(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg13(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg14(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg15(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg16(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
cudaError_t launch_tma_cfg17(int, int, bool, const DevBlock*, const Tile*, int, const StageArgs&, cudaStream_t, int);
static_assert(NUM_TMA_CFGS == 18, "one configure / launch pair per TMA configuration");
static const TmaConfigure g_tma_configure[NUM_TMA_CFGS] = {
    configure_tma_cfg0, configure_tma_cfg1, configure_tma_cfg2, configure_tma_cfg3, configure_tma_cfg4, configure_tma_cfg5,
    configure_tma_cfg6, configure_tma_cfg7, configure_tma_cfg8, configure_tma_cfg9, configure_tma_cfg10,
    configure_tma_cfg11, configure_tma_cfg12, configure_tma_cfg13, configure_tma_cfg14, configure_tma_cfg15,
    configure_tma_cfg16, configure_tma_cfg17};
static const TmaLaunch g_tma_launch[NUM_TMA_CFGS] = {
    launch_tma_cfg0, launch_tma_cfg1, launch_tma_cfg2, launch_tma_cfg3, launch_tma_cfg4, launch_tma_cfg5,
    launch_tma_cfg6, launch_tma_cfg7, launch_tma_cfg8, launch_tma_cfg9, launch_tma_cfg10, launch_tma_cfg11,
    launch_tma_cfg12, launch_tma_cfg13, launch_tma_cfg14, launch_tma_cfg15, launch_tma_cfg16, launch_tma_cfg17};

// Persistent grid of each TMA configuration on each device: SMs x resident CTAs.
constexpr int MAX_DEVICES = 64;
static int g_tma_grid[MAX_DEVICES][NUM_TMA_CFGS][3][2][2];  // [device][cfg][precision mode][epi][sel]

int tma_grid(int cfg) {
    int dev = 0;
    if (cfg < 0 || cfg >= NUM_TMA_CFGS) return 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return 0;
    // the smaller of the two per-tile passes' resident grids (the FP64 pass may
    // fit fewer CTAs per SM)
    const int a = g_tma_grid[dev][cfg][PM_MIXED][EPI_RK][1], b = g_tma_grid[dev][cfg][PM_FP64F][EPI_RK][1];
    return a < b ? a : b;
}

static cudaError_t launch_tma(int cfg, int pm, int epi, const DevBlock* blocks, const Tile* tiles, int ntiles,
                              const StageArgs& args, cudaStream_t stream) {
    if (!args.tmaps || cfg < 0 || cfg >= NUM_TMA_CFGS || pm < 0 || pm > 2) return cudaErrorInvalidValue;
    if (TMA_CFGS[cfg].rem && !args.tmaps_rem) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const bool sel = args.tile_prec != nullptr;  // per-tile precision passes (RK epilogue)
    if (sel && epi != EPI_RK) return cudaErrorInvalidValue;
    int cap = (dev >= 0 && dev < MAX_DEVICES) ? g_tma_grid[dev][cfg][pm][epi][sel ? 1 : 0] : 0;
    if (cap <= 0) return cudaErrorInvalidConfiguration;  // not instantiated, or configure_stage_kernels() not run
    // The FP64 pass of the per-tile precision takes few tiles, clustered near the
    // punctures: TMA_FP64_SPREAD times the resident grid spreads them over more
    // CTAs (a CTA without selected tiles exits after its scan), so fewer CTAs run
    // two or more of them one after the other.
    if (pm == PM_FP64F && sel) cap *= TMA_FP64_SPREAD;
    return g_tma_launch[cfg](pm, epi, sel, blocks, tiles, ntiles, args, stream, ntiles < cap ? ntiles : cap);
}

// Opt the shared-memory variants into more than 48 KB of dynamic shared memory
// on the current device and size the persistent grids (called once per context
// at creation).
cudaError_t configure_stage_kernels() {
    cudaError_t e;
    if ((e = configure_smem<PM_FP64, EPI_STORE>())) return e;
    if ((e = configure_smem<PM_FP64, EPI_RK>())) return e;
    if ((e = configure_smem<PM_MIXED, EPI_STORE>())) return e;
    if ((e = configure_smem<PM_MIXED, EPI_RK>())) return e;
    if ((e = configure_smem<PM_FP64F, EPI_RK>())) return e;
    int dev = 0, nsm = 0;
    if ((e = cudaGetDevice(&dev))) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev))) return e;
    for (int k = 0; k < NUM_TMA_CFGS; ++k)
        if ((e = g_tma_configure[k](nsm, g_tma_grid[dev][k]))) return e;
    return cudaSuccess;
}

template <int PM, int EPI, int MINB>
static cudaError_t launch_global(const DevBlock* blocks, const Tile* tiles, int ntiles, const StageArgs& args,
                                 cudaStream_t stream) {
    ccz4_stage_kernel<PM, EPI, V0_TX, V0_TY, V0_TZ, MINB>
        <<<ntiles, dim3(V0_TX, V0_TY, V0_TZ), 0, stream>>>(blocks, tiles, args);
    return cudaGetLastError();
}

// Precision mode x epilogue -> one instantiation of a launcher L<PM, EPI>.
template <template <int, int> class L>
static cudaError_t dispatch(int pm, int epi, const DevBlock* blocks, const Tile* tiles, int ntiles,
                            const StageArgs& args, cudaStream_t stream) {
    if (pm == PM_FP64)
        return epi == EPI_STORE ? L<PM_FP64, EPI_STORE>::run(blocks, tiles, ntiles, args, stream)
                                : L<PM_FP64, EPI_RK>::run(blocks, tiles, ntiles, args, stream);
    if (pm == PM_MIXED)
        return epi == EPI_STORE ? L<PM_MIXED, EPI_STORE>::run(blocks, tiles, ntiles, args, stream)
                                : L<PM_MIXED, EPI_RK>::run(blocks, tiles, ntiles, args, stream);
    if (pm == PM_FP64F && epi == EPI_RK) return L<PM_FP64F, EPI_RK>::run(blocks, tiles, ntiles, args, stream);
    return cudaErrorInvalidValue;
}

template <int PM, int EPI>
struct RunSmem {
    static cudaError_t run(const DevBlock* b, const Tile* t, int n, const StageArgs& a, cudaStream_t s) {
        return launch_smem<PM, EPI>(b, t, n, a, s);
    }
};
template <int MINB>
struct RunGlobal {
    template <int PM, int EPI>
    struct L {
        static cudaError_t run(const DevBlock* b, const Tile* t, int n, const StageArgs& a, cudaStream_t s) {
            return launch_global<PM, EPI, MINB>(b, t, n, a, s);
        }
    };
};

cudaError_t launch_classify(int variant, int cfg, const DevBlock* blocks, const Tile* tiles, int first, int ntiles,
                            int sel, double chi_fp64, unsigned char* flag, cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    int tx, ty, tz;
    if (stage_tile_dims(variant, cfg, &tx, &ty, &tz)) return cudaErrorInvalidValue;
    classify_tiles_kernel<<<(ntiles + CLASSIFY_WARPS - 1) / CLASSIFY_WARPS, 32 * CLASSIFY_WARPS, 0, stream>>>(
        blocks, tiles, first, ntiles, sel, tx, ty, tz, chi_fp64, flag);
    return cudaGetLastError();
}

cudaError_t launch_stage(int variant, int cfg, int precision, int epi, const DevBlock* blocks, const Tile* tiles,
                         int ntiles, const StageArgs& args, cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    switch (variant) {
        case VARIANT_TMA: return launch_tma(cfg, precision, epi, blocks, tiles, ntiles, args, stream);
        case VARIANT_SMEM: return dispatch<RunSmem>(precision, epi, blocks, tiles, ntiles, args, stream);
        case VARIANT_GLOBAL_R168:
            return dispatch<RunGlobal<3>::L>(precision, epi, blocks, tiles, ntiles, args, stream);
        case VARIANT_GLOBAL_R128:
            return dispatch<RunGlobal<4>::L>(precision, epi, blocks, tiles, ntiles, args, stream);
        default: return dispatch<RunGlobal<1>::L>(precision, epi, blocks, tiles, ntiles, args, stream);
    }
}


// KO dissipation alone (CCZ4Evolution::applyDissipation, ccz4.cpp:871-935):
// rhs += sum_d sum_s (cf_d w_s) u(x + s e_d) in the reference's order, without
// contraction, so the drop-in reproduces the host loop bit for bit.
__global__ void __launch_bounds__(128)
    ko_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int in_sel, double* rhs) {
    const Tile t = tiles[blockIdx.x];
    const DevBlock& B = blocks[t.block];
    const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y, k = t.k0 + threadIdx.z;
    if (i >= B.n[0] || j >= B.n[1] || k >= B.n[2]) return;
    const long long c = cell_index(B, i + NG, j + NG, k + NG);
    const long long off[3] = {1, B.tx, (long long)B.tx * B.ty};
    const double wts[7] = {1.0, -6.0, 15.0, -20.0, 15.0, -6.0, 1.0};
    const double* u = B.buf[in_sel];
    for (int v = 0; v < NV; ++v) {
        const double* f = u + (long long)v * B.stride + c;
        double diss = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int s = 0; s < 7; ++s) diss = __dadd_rn(diss, __dmul_rn(__dmul_rn(B.kocf[d], wts[s]), __ldg(f + (s - 3) * off[d])));
        double* r = rhs + (long long)v * B.stride + c;
        *r = __dadd_rn(*r, diss);
    }
}

cudaError_t launch_dissipation(const DevBlock* block, int in_sel, double* rhs, int ntiles, const Tile* tiles,
                               cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    ko_kernel<<<ntiles, dim3(V0_TX, V0_TY, V0_TZ), 0, stream>>>(block, tiles, in_sel, rhs);
    return cudaGetLastError();
}

}  // namespace granite_b200
