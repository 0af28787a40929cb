// ccz4_rhs.cu -- fused CCZ4 RHS + Kreiss-Oliger + SSP-RK3 stage kernel.
//
// One thread per interior point; one CTA per tile of a block; the launch walks
// a work-list of tiles over every block of an AMR level, so blocks of uneven
// size share one launch per RK stage.
//
// Physics: CCZ4Evolution::computeRHS (ccz4.cpp:251-865) plus applyDissipation
// (ccz4.cpp:871-935). The algebra is regrouped (first-kind Christoffels reused
// in the Ricci tensor, mixed-index A and Christoffel contractions computed
// once) but every term of the reference is kept with the same coefficients,
// regularisers and blend, so results agree with the reference to rounding.
//
// Epilogues:
//   EPI_STORE   rhs = L(u)                         (computeRHS drop-in)
//   EPI_RK      out = a1 u^n + a2 u_in + a3dt L(u_in), chi/alpha floors, and on
//               the last stage the det/trace constraints (main.cpp:306-335,
//               588-671), all pointwise, so the RK combine never re-reads memory.
//
// Precision: P = double gives the plain FP64 kernel. P = float gives the mixed
// form: every stencil is evaluated as FP64 pair differences (f[+k] - f[-k],
// f[+k] + f[-k] - 2 f[0] ...), rounded to FP32 only after the cancellation,
// then the Christoffel/Ricci/gauge/KO algebra runs in FP32. chi, the inverse
// conformal metric, the 1/chi factors, the evolved state and the RK3 combine
// stay FP64. Per-tile precision: a launch can be restricted to the tiles of a
// flag array (classify_tiles_kernel marks the tiles with a point of chi below a
// threshold, near a puncture): the FP64 kernel takes those tiles and the FP32
// kernel the others, both walking the tile list in its spatial order.
//
// Control flow: the per-point body is one straight-line sequence (the KO term
// is always evaluated -- its weights sigma/(64 dx) w_s are zero when KO is off
// -- and the upwind side is a select, not a branch), so the compiler can
// schedule the stencil loads of later fields across earlier ones.
#include "ccz4_common.cuh"
#include "ccz4_kernels.h"
#include "ccz4_stencil.cuh"

namespace granite_b200 {

namespace {

constexpr double PI_D = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Sources of per-field stencil results. ccz4_point asks for the fields in one
// fixed order (FIELD_ORDER); a source may rely on that order.
// ---------------------------------------------------------------------------
__device__ constexpr int FIELD_ORDER[NV] = {GXX, GXY, GXZ, GYY, GYZ, GZZ, GHX, GHY, GHZ, CHI, ALPHA,
                                            BETAX, BETAY, BETAZ, KTR, THETA, AXX, AXY, AXZ, AYY, AYZ, AZZ};

// Per-tile precision: a launch with tile_prec set covers only the tiles whose
// flag equals want (1 = FP64 algebra, 0 = FP32), in list order.
__device__ __forceinline__ bool tile_selected(const unsigned char* prec, int want, int ti) {
    return !prec || prec[ti] == want;
}

// Stencils read straight from global memory (through L1). Every source
// evaluates the stencils of one field in the precision of the caller's algebra
// (P = double or float, deduced from the blend weight w).
struct GlobalSource {
    const DevBlock& B;
    const double* __restrict__ u;
    long long c;
    template <bool HESS, bool EXACT, typename P>
    __device__ __forceinline__ FieldDer<P> der(int v, const double beta[3], P w) {
        const long long off[3] = {1, B.tx, (long long)B.tx * B.ty};
        return field_der_l<P, HESS, true, GlobalLoad, EXACT>(B, GlobalLoad{u + (long long)v * B.stride + c}, off,
                                                             beta, w);
    }
};

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

// ---------------------------------------------------------------------------
// TMA ring: a persistent CTA walks its tiles (blockIdx.x, + gridDim.x, ...)
// and consumes a stream of items q = (tile round q / NV, field FIELD_ORDER[q % NV]).
// Item q is one 24x12x12-cell box (the 16x4x4 tile and its 4-cell halo) of one
// field, brought into ring slot q % NBUF by a single tensor-map load that
// completes on that slot's mbarrier. Thread 0 issues item q + NBUF - 1 when
// the CTA starts on item q, so loads run NBUF - 1 fields ahead and across tile
// boundaries. Rows of 24 doubles put the 16-wide x rows of a warp in distinct
// shared-memory banks for every stencil offset.
// ---------------------------------------------------------------------------
constexpr int V4_TX = 16, V4_TY = 4, V4_TZ = 4, V4_NT = V4_TX * V4_TY * V4_TZ;
static_assert(TMA_BOX[0] == V4_TX + 8 && TMA_BOX[1] == V4_TY + 8 && TMA_BOX[2] == V4_TZ + 8, "box = tile + halo");

template <int NBUF>
struct TmaRing {
    static constexpr int BX = TMA_BOX[0], BY = TMA_BOX[1], BZ = TMA_BOX[2];
    static constexpr int BOX = BX * BY * BZ;
    static constexpr unsigned BYTES = BOX * sizeof(double);  // complete_tx count of one item
    static_assert(BYTES % 128 == 0, "slots stay 128-byte aligned");
    static constexpr size_t SMEM = (size_t)NBUF * BYTES + NBUF * sizeof(unsigned long long) + 128;
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// One box of a 4-D tensor map (x, y, z, field) into shared memory.
__device__ __forceinline__ void tma_load_box(unsigned dst, const void* map, int x, int y, int z, int f,
                                             unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(dst),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(f), "r"(bar)
        : "memory");
}

// Wait limit of one ring slot: 2 s of wall time, then the kernel records the
// failure in StageArgs::errflag and stops waiting (results are then garbage
// and the host reports the error).
constexpr unsigned long long TMA_WAIT_NS = 2000000000ull;

// Per-tile precision launches: the CTA's selected tiles, in order, and their
// count at [TMA_SEL_CAP] (shared memory at a fixed address, so the per-point
// body keeps no register for them).
__shared__ int g_sel_list[TMA_SEL_CAP + 1];

template <int NBUF, bool SEL>
struct TmaSource {
    using R = TmaRing<NBUF>;
    const DevBlock* blocks;
    const Tile* tiles;
    const unsigned char* maps;  // CUtensorMap array, 128 bytes each
    int ntiles, in_sel;
    double* ring;      // NBUF slots of R::BOX doubles
    unsigned bar0;     // shared address of the slot mbarriers (8 bytes apart)
    const DevBlock* B; // block of the current tile (stencil coefficients)
    int lin;           // this thread's point within a slot
    int next;          // next item to consume
    bool failed;       // a wait of this thread gave up (at item fail_q); thread 0 then stops issuing
    unsigned int* err;
    int fail_q;
    int withhold;      // test switch: 1 + the item CTA 0 leaves unissued (0: none)

    // Tile of the CTA's r-th round: blockIdx.x + r gridDim.x, or with per-tile
    // precision (SEL) the r-th tile of that sequence whose flag the launch takes.
    __device__ __forceinline__ int round_tile(int r) const {
        if constexpr (SEL)
            return r < g_sel_list[TMA_SEL_CAP] ? g_sel_list[r] : ntiles;
        else
            return blockIdx.x + r * gridDim.x;
    }
    // thread 0 only
    __device__ __forceinline__ void issue(int q) const {
        const int ti = round_tile(q / NV);
        if (ti >= ntiles) return;
        if (withhold != 0 && q == withhold - 1 && blockIdx.x == 0) return;  // test switch: never issued
        const Tile t = tiles[ti];
        const int s = q % NBUF;
        const unsigned bar = bar0 + 8u * s;
        mbar_expect_tx(bar, R::BYTES);
        // box origin = tile origin - 4 cells = interior index (cells incl. ghosts start 4 lower)
        tma_load_box(smem_addr(ring + (size_t)s * R::BOX), maps + (size_t)(3 * t.block + in_sel) * 128, t.i0, t.j0,
                     t.k0, FIELD_ORDER[q % NV], bar);
    }
    __device__ __forceinline__ void wait(int q) {
        if (failed) return;
        const unsigned bar = bar0 + 8u * (q % NBUF), parity = (q / NBUF) & 1;
        unsigned long long t0 = 0;
        for (unsigned it = 1;; ++it) {
            if (mbar_try_wait(bar, parity)) return;
            if ((it & 255u) == 0) {
                const unsigned long long now = global_ns();
                if (t0 == 0) {
                    t0 = now;
                } else if (now - t0 > TMA_WAIT_NS) {
                    failed = true;
                    fail_q = q;
                    if (err) atomicExch(err, 1u);
                    return;
                }
            }
        }
    }
    // Every thread of the CTA calls der() for every item in order (the call
    // carries the CTA barrier that frees the slot the next load overwrites).
    template <bool HESS, bool EXACT, typename P>
    __device__ __forceinline__ FieldDer<P> der(int /*v*/, const double beta[3], P w) {
        __syncthreads();
        if (threadIdx.x == 0 && !failed) issue(next + NBUF - 1);
        wait(next);
        const SharedLoad L{ring + (size_t)(next % NBUF) * R::BOX + lin};
        ++next;
        const long long off[3] = {1, R::BX, R::BX * R::BY};
        return field_der_l<P, HESS, true, SharedLoad, EXACT>(*B, L, off, beta, w);
    }
};

// ---------------------------------------------------------------------------
// RHS at one interior point. Returns L(u) for the 22 fields in `out` (FP64).
// ---------------------------------------------------------------------------
// EXACT: FP64 stencils in the reference's operation order (P = double only).
template <typename P, bool EXACT, typename Src>
__device__ __forceinline__ void ccz4_point(const DevBlock& B, const double* __restrict__ u,
                                           long long c, const StageArgs& A, Src& S, double out[NV]) {
    const long long st = B.stride;
    const double* __restrict__ uc = u + c;
#define FP(v) (uc + (long long)(v) * st)
    // ---- pointwise state (FP64) -------------------------------------------
    const double chi_raw = __ldg(FP(CHI));
    const double chi = (isfinite(chi_raw) && chi_raw >= 1.0e-4) ? chi_raw : 1.0e-4;  // :279-280
    const double alpha_d = __ldg(FP(ALPHA));
    const double K_d = __ldg(FP(KTR));
    const double Th_d = __ldg(FP(THETA));
    double gtd[6], Atd[6], Ghd[3], beta[3];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        gtd[a] = __ldg(FP(GXX + a));
        Atd[a] = __ldg(FP(AXX + a));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Ghd[a] = __ldg(FP(GHX + a));
        beta[a] = __ldg(FP(BETAX + a));
    }
    // inverse conformal metric, FP64 (ccz4.cpp:318-330)
    double gtud[6];
    {
        const double det = gtd[0] * (gtd[3] * gtd[5] - gtd[4] * gtd[4]) -
            gtd[1] * (gtd[1] * gtd[5] - gtd[4] * gtd[2]) + gtd[2] * (gtd[1] * gtd[4] - gtd[3] * gtd[2]);
        const double inv = 1.0 / (det + 1.0e-30);
        gtud[0] = (gtd[3] * gtd[5] - gtd[4] * gtd[4]) * inv;
        gtud[1] = (gtd[2] * gtd[4] - gtd[1] * gtd[5]) * inv;
        gtud[2] = (gtd[1] * gtd[4] - gtd[2] * gtd[3]) * inv;
        gtud[3] = (gtd[0] * gtd[5] - gtd[2] * gtd[2]) * inv;
        gtud[4] = (gtd[1] * gtd[2] - gtd[0] * gtd[4]) * inv;
        gtud[5] = (gtd[0] * gtd[3] - gtd[1] * gtd[1]) * inv;
    }
    const P w = (P)(0.5 * (1.0 + tanh((chi - A.chi_c) / A.chi_w)));  // :565
    const P alpha = (P)alpha_d, K = (P)K_d, Theta = (P)Th_d;
    P gt[6], At[6], gtu[6], Gh[3];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        gt[a] = (P)gtd[a];
        At[a] = (P)Atd[a];
        gtu[a] = (P)gtud[a];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) Gh[a] = (P)Ghd[a];

    // ---- conformal metric: gradients, Hessian term of Ricci, advection ----
    P dg[6][3];     // d_k gt_ij
    P Rt[6];        // conformal Ricci (ccz4.cpp:465-516), accumulated term by term
    P agt[6], kgt[6];  // advection and KO of gt
    // Kept as a loop (one copy of the Hessian-field stencil code instead of
    // six): the per-point body is otherwise longer than the instruction caches
    // hold, and instruction fetch stalls the warps. The four arrays it fills
    // (36 values) live in L1-cached local memory for the loop's duration.
#pragma unroll 1
    for (int a = 0; a < 6; ++a) {
        FieldDer<P> fd = S.template der<true, EXACT>(GXX + a, beta, w);
#pragma unroll
        for (int d = 0; d < 3; ++d) dg[a][d] = fd.d[d];
        // term 1: -1/2 gtu^{lm} d_l d_m gt_ij
        Rt[a] = (P)-0.5 * (gtu[0] * fd.h[0] + gtu[3] * fd.h[3] + gtu[5] * fd.h[5] +
                           (P)2 * (gtu[1] * fd.h[1] + gtu[2] * fd.h[2] + gtu[4] * fd.h[4]));
        agt[a] = fd.adv;
        kgt[a] = fd.ko;
    }
    // first-kind Christoffels G1[k][ij] = 1/2 (d_i g_kj + d_j g_ki - d_k g_ij)
    P G1[3][6];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j)
                G1[k][sy(i, j)] = (P)0.5 * (dg[sy(k, j)][i] + dg[sy(k, i)][j] - dg[sy(i, j)][k]);
    // second-kind Christoffels chris[i][jk] = gtu^{il} G1[l][jk] (ccz4.cpp:408-444)
    P ch[3][6];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int jk = 0; jk < 6; ++jk)
            ch[i][jk] = gtu[sy(i, 0)] * G1[0][jk] + gtu[sy(i, 1)] * G1[1][jk] + gtu[sy(i, 2)] * G1[2][jk];
    // contracted Gamma^k = gtu^{lm} chris[k][lm]
    P Gc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        Gc[k] = gtu[0] * ch[k][0] + gtu[3] * ch[k][3] + gtu[5] * ch[k][5] +
            (P)2 * (gtu[1] * ch[k][1] + gtu[2] * ch[k][2] + gtu[4] * ch[k][4]);

    // ---- Gamma-hat: gradient (Ricci term 2), advection --------------------
    P dGh[3][3];
    P aGh[3], kGh[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        FieldDer<P> fd = S.template der<false, EXACT>(GHX + a, beta, w);
#pragma unroll
        for (int d = 0; d < 3; ++d) dGh[a][d] = fd.d[d];
        aGh[a] = fd.adv;
        kGh[a] = fd.ko;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            P t2 = (P)0;
#pragma unroll
            for (int k = 0; k < 3; ++k) t2 += gt[sy(k, i)] * dGh[k][j] + gt[sy(k, j)] * dGh[k][i];
            // term 2 + terms 3 and 5 (Gh^k - Gc^k) Gamma_{k,ij}
            Rt[sy(i, j)] += (P)0.5 * t2 + (Gh[0] - Gc[0]) * G1[0][sy(i, j)] +
                (Gh[1] - Gc[1]) * G1[1][sy(i, j)] + (Gh[2] - Gc[2]) * G1[2][sy(i, j)];
        }
    // term 4: gtu^{lm} (chris^k_{li} Gamma_{k,jm} + chris^k_{lj} Gamma_{k,im})
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        P Gu[3][3];  // Gu[j][l] = gtu^{lm} Gamma_{k,jm}
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int l = 0; l < 3; ++l)
                Gu[j][l] = gtu[sy(l, 0)] * G1[k][sy(j, 0)] + gtu[sy(l, 1)] * G1[k][sy(j, 1)] +
                    gtu[sy(l, 2)] * G1[k][sy(j, 2)];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j) {
                P t = (P)0;
#pragma unroll
                for (int l = 0; l < 3; ++l) t += ch[k][sy(l, i)] * Gu[j][l] + ch[k][sy(l, j)] * Gu[i][l];
                Rt[sy(i, j)] += t;
            }
    }

    // ---- chi: Ricci chi-part (ccz4.cpp:518-541) -----------------------------
    FieldDer<P> fchi = S.template der<true, EXACT>(CHI, beta, w);
    const P chiP = (P)chi;
    // 0.5/(chi+1e-30) and 0.25/(chi^2+1e-30) in FP64 (small chi near the puncture)
    const P c_half = (P)(0.5 / (chi + 1e-30));
    const P c_quart = (P)(0.25 / ((chi * chi) + 1e-30));
    P DDchi[6];
#pragma unroll
    for (int ij = 0; ij < 6; ++ij)
        DDchi[ij] = fchi.h[ij] - (ch[0][ij] * fchi.d[0] + ch[1][ij] * fchi.d[1] + ch[2][ij] * fchi.d[2]);
    const P lapchi = gtu[0] * DDchi[0] + gtu[3] * DDchi[3] + gtu[5] * DDchi[5] +
        (P)2 * (gtu[1] * DDchi[1] + gtu[2] * DDchi[2] + gtu[4] * DDchi[4]);
    P dchi2 = (P)0;
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int m = 0; m < 3; ++m) dchi2 += gtu[sy(l, m)] * fchi.d[l] * fchi.d[m];
    P Ric[6];  // R_ij = Rt_ij + Rchi_ij
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const int ij = sy(i, j);
            const P t1 = c_half * (DDchi[ij] + gt[ij] * lapchi);
            const P t2 = c_quart * (fchi.d[i] * fchi.d[j] - (P)3 * gt[ij] * dchi2);
            Ric[ij] = Rt[ij] + (t1 - t2);
        }
    P Rs = (P)0;  // chi gtu^{ij} R_ij (ccz4.cpp:654-660)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rs += gtu[sy(i, j)] * Ric[sy(i, j)];
    Rs *= chiP;

    // ---- lapse -------------------------------------------------------------
    FieldDer<P> fal = S.template der<true, EXACT>(ALPHA, beta, w);
    P DDa[6];
#pragma unroll
    for (int ij = 0; ij < 6; ++ij)
        DDa[ij] = fal.h[ij] - (ch[0][ij] * fal.d[0] + ch[1][ij] * fal.d[1] + ch[2][ij] * fal.d[2]);
    const P lapa = gtu[0] * DDa[0] + gtu[3] * DDa[3] + gtu[5] * DDa[5] +
        (P)2 * (gtu[1] * DDa[1] + gtu[2] * DDa[2] + gtu[4] * DDa[4]);
    P cga = (P)0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) cga += gtu[sy(a, b)] * fchi.d[a] * fal.d[b];
    const P phys_lap_alpha = chiP * lapa - (P)0.5 * cga;  // :648

    // ---- shift: gradient, Hessian terms T5/T6 ---------------------------------
    P db[3][3];  // d_j beta^i as db[i][j]
    P T5[3], ddiv[3];
    P abe[3], kbe[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) ddiv[d] = (P)0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        FieldDer<P> fb = S.template der<true, EXACT>(BETAX + a, beta, w);
#pragma unroll
        for (int d = 0; d < 3; ++d) db[a][d] = fb.d[d];
        T5[a] = gtu[0] * fb.h[0] + gtu[3] * fb.h[3] + gtu[5] * fb.h[5] +
            (P)2 * (gtu[1] * fb.h[1] + gtu[2] * fb.h[2] + gtu[4] * fb.h[4]);
        // d_j (d_k beta^k): add d_j d_a beta^a
#pragma unroll
        for (int d = 0; d < 3; ++d) ddiv[d] += fb.h[sy(a, d)];
        abe[a] = fb.adv;
        kbe[a] = fb.ko;
    }
    const P divb = db[0][0] + db[1][1] + db[2][2];  // :548

    // ---- A-tilde: mixed index, squares, advection ------------------------------
    P Am[3][3];  // Am[i][j] = gtu^{ik} At_kj
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Am[i][j] = gtu[sy(i, 0)] * At[sy(0, j)] + gtu[sy(i, 1)] * At[sy(1, j)] + gtu[sy(i, 2)] * At[sy(2, j)];
    P AtAt = (P)0;  // At_ij At^ij (ccz4.cpp:609-619)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) AtAt += Am[i][j] * Am[j][i];

    // matter sources (ccz4.cpp:651,664,682,764), zero in vacuum
    P rho = (P)0, Str = (P)0, Si[3] = {(P)0, (P)0, (P)0}, Sij[6] = {(P)0, (P)0, (P)0, (P)0, (P)0, (P)0};
    if (A.rho) {
        const long long cm = c + B.moff;
        rho = (P)__ldg(A.rho + cm);
        Str = (P)__ldg(A.S + cm);
#pragma unroll
        for (int a = 0; a < 3; ++a) Si[a] = (P)__ldg(A.Si + 3 * cm + a);
#pragma unroll
        for (int a = 0; a < 6; ++a) Sij[a] = (P)__ldg(A.Sij + 6 * cm + a);
    }
    const P PI = (P)PI_D;

    // ---- RHS assembly ----------------------------------------------------------
    // chi (ccz4.cpp:580)
    // each field: (RHS incl. advection) + KO, the order of ccz4.cpp:864,930
    out[CHI] = (double)(((P)(2.0 / 3.0) * chiP * (alpha * K - divb) + fchi.adv) + fchi.ko);
    // gt (ccz4.cpp:586-607)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const int ij = sy(i, j);
            P lie = agt[ij];
#pragma unroll
            for (int d = 0; d < 3; ++d) lie += gt[sy(i, d)] * db[d][j] + gt[sy(j, d)] * db[d][i];
            out[GXX + ij] = (double)(((P)-2 * alpha * At[ij] + lie - (P)(2.0 / 3.0) * gt[ij] * divb) + kgt[ij]);
        }
    // K (ccz4.cpp:650-652)
    {
        FieldDer<P> fK = S.template der<false, EXACT>(KTR, beta, w);
        const P k1 = (P)A.kappa1, k2 = (P)A.kappa2;
        out[KTR] = (double)((-phys_lap_alpha + alpha * (AtAt + K * K / (P)3) + (P)4 * PI * alpha * (rho + Str) +
                            k1 * ((P)1 - k2) * alpha * Theta + fK.adv) + fK.ko);
        // Gamma-hat (ccz4.cpp:747-815)
        const P c3a = (P)(3.0 * alpha_d / (chi + 1e-30));
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            P T1 = (P)0;
#pragma unroll
            for (int jk = 0; jk < 6; ++jk) T1 += (jk == 1 || jk == 2 || jk == 4 ? (P)2 : (P)1) * ch[i][jk] * At[jk];
            T1 *= (P)2 * alpha;
            const P T2 = -(P)(4.0 / 3.0) * alpha *
                (gtu[sy(i, 0)] * fK.d[0] + gtu[sy(i, 1)] * fK.d[1] + gtu[sy(i, 2)] * fK.d[2]);
            const P T3 = -(P)16 * PI * alpha * (gtu[sy(i, 0)] * Si[0] + gtu[sy(i, 1)] * Si[1] + gtu[sy(i, 2)] * Si[2]);
            const P T4 = c3a * (Am[i][0] * fchi.d[0] + Am[i][1] * fchi.d[1] + Am[i][2] * fchi.d[2]);
            const P T6 = (P)(1.0 / 3.0) *
                (gtu[sy(i, 0)] * ddiv[0] + gtu[sy(i, 1)] * ddiv[1] + gtu[sy(i, 2)] * ddiv[2]);
            P T7 = -(Gh[0] * db[i][0] + Gh[1] * db[i][1] + Gh[2] * db[i][2]);
            T7 += aGh[i] + (P)(2.0 / 3.0) * Gh[i] * divb;
            const P T8 = (P)-2 * (P)A.kappa1 * alpha * Gh[i];
            out[GHX + i] = (double)((T1 + T2 + T3 + T4 + T5[i] + T6 + T7 + T8) + kGh[i]);
        }
    }
    // Theta (ccz4.cpp:662-665)
    {
        FieldDer<P> fT = S.template der<false, EXACT>(THETA, beta, w);
        const P k1 = (P)A.kappa1, k2 = (P)A.kappa2;
        out[THETA] = (double)(((P)0.5 * alpha * (Rs - AtAt + (P)2 * K * K / (P)3 - (P)16 * PI * rho) -
                              alpha * k1 * ((P)2 + k2) * Theta + fT.adv) + fT.ko);
    }
    // A-tilde (ccz4.cpp:671-726): the advection is part of Lie_At and is
    // trace-removed with the rest; KO is added after the trace removal.
    {
        P raw[6], koA[6];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j) {
                const int ij = sy(i, j);
                FieldDer<P> fA = S.template der<false, EXACT>(AXX + ij, beta, w);
                koA[ij] = fA.ko;
                const P t1 = chiP * (-DDa[ij] + alpha * (Ric[ij] - (P)8 * PI * Sij[ij]));
                const P Asq = At[sy(i, 0)] * Am[0][j] + At[sy(i, 1)] * Am[1][j] + At[sy(i, 2)] * Am[2][j];
                const P t2 = alpha * (K * At[ij] - (P)2 * Asq);
                P lie = fA.adv;
#pragma unroll
                for (int d = 0; d < 3; ++d) lie += At[sy(i, d)] * db[d][j] + At[sy(j, d)] * db[d][i];
                lie -= (P)(2.0 / 3.0) * At[ij] * divb;
                raw[ij] = t1 + t2 + lie;
            }
        const P tr = gtu[0] * raw[0] + gtu[3] * raw[3] + gtu[5] * raw[5] +
            (P)2 * (gtu[1] * raw[1] + gtu[2] * raw[2] + gtu[4] * raw[4]);
#pragma unroll
        for (int a = 0; a < 6; ++a) out[AXX + a] = (double)(raw[a] - (P)(1.0 / 3.0) * gt[a] * tr + koA[a]);
    }
    // lapse (ccz4.cpp:820) and shift (ccz4.cpp:825-831)
    out[ALPHA] = (double)(((P)-2 * alpha * K + fal.adv) + fal.ko);
    {
        const P eta = (P)A.eta;
#pragma unroll
        for (int d = 0; d < 3; ++d) out[BETAX + d] = (double)(((P)0.75 * Gh[d] - eta * (P)beta[d] + abe[d]) + kbe[d]);
    }
#undef FP
}

// det(gt) = 1 and tr(At) = 0 at one point, main.cpp:612-671, evaluated
// without FMA contraction so it matches the host loop to the last bit (cbrt
// may differ by one ulp from the host libm).
__device__ __forceinline__ void algebraic_constraints(double r[NV]) {
#define M_(a, b) __dmul_rn(a, b)
#define A_(a, b) __dadd_rn(a, b)
#define S_(a, b) __dsub_rn(a, b)
    double gxx = r[GXX], gxy = r[GXY], gxz = r[GXZ], gyy = r[GYY], gyz = r[GYZ], gzz = r[GZZ];
    const double det = A_(S_(M_(gxx, S_(M_(gyy, gzz), M_(gyz, gyz))), M_(gxy, S_(M_(gxy, gzz), M_(gyz, gxz)))),
                          M_(gxz, S_(M_(gxy, gyz), M_(gyy, gxz))));
    if (isfinite(det) && det > 1.0e-10) {
        const double s = cbrt(1.0 / det);
        gxx = M_(gxx, s); gxy = M_(gxy, s); gxz = M_(gxz, s);
        gyy = M_(gyy, s); gyz = M_(gyz, s); gzz = M_(gzz, s);
    } else {
        gxx = 1.0; gxy = 0.0; gxz = 0.0; gyy = 1.0; gyz = 0.0; gzz = 1.0;
    }
    r[GXX] = gxx; r[GXY] = gxy; r[GXZ] = gxz; r[GYY] = gyy; r[GYZ] = gyz; r[GZZ] = gzz;
    const double ixx = S_(M_(gyy, gzz), M_(gyz, gyz));
    const double ixy = S_(M_(gxz, gyz), M_(gxy, gzz));
    const double ixz = S_(M_(gxy, gyz), M_(gxz, gyy));
    const double iyy = S_(M_(gxx, gzz), M_(gxz, gxz));
    const double iyz = S_(M_(gxz, gxy), M_(gxx, gyz));
    const double izz = S_(M_(gxx, gyy), M_(gxy, gxy));
    const double axx = r[AXX], axy = r[AXY], axz = r[AXZ], ayy = r[AYY], ayz = r[AYZ], azz = r[AZZ];
    const double trA = A_(A_(A_(M_(ixx, axx), M_(iyy, ayy)), M_(izz, azz)),
                          M_(2.0, A_(A_(M_(ixy, axy), M_(ixz, axz)), M_(iyz, ayz))));
    const double t3 = trA / 3.0;
    r[AXX] = S_(axx, M_(t3, gxx)); r[AXY] = S_(axy, M_(t3, gxy)); r[AXZ] = S_(axz, M_(t3, gxz));
    r[AYY] = S_(ayy, M_(t3, gyy)); r[AYZ] = S_(ayz, M_(t3, gyz)); r[AZZ] = S_(azz, M_(t3, gzz));
#undef M_
#undef A_
#undef S_
}

// RK combine without FMA contraction: a1*un + a2*ui + a3dt*L (main.cpp:327-328)
__device__ __forceinline__ double rk_combine(double a1, double un, double a2, double ui, double a3dt,
                                             double L) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a1, un), __dmul_rn(a2, ui)), __dmul_rn(a3dt, L));
}

}  // namespace

// The RHS at one point with the algebra of precision mode PM.
template <int PM, typename Src>
__device__ __forceinline__ void point_pm(const DevBlock& B, const double* __restrict__ u, long long c,
                                         const StageArgs& A, Src& S, double L[NV]) {
    if constexpr (PM == PM_FP64)
        ccz4_point<double, true>(B, u, c, A, S, L);
    else if constexpr (PM == PM_FP64F)
        ccz4_point<double, false>(B, u, c, A, S, L);
    else
        ccz4_point<float, false>(B, u, c, A, S, L);
}

// Shared epilogue: store L, or RK combine + floors (+ algebraic constraints).
template <int EPI>
__device__ __forceinline__ void stage_epilogue(const DevBlock& B, const StageArgs& A, long long c, const double L[NV]) {
    const long long st = B.stride;
    if (EPI == EPI_STORE) {
#pragma unroll
        for (int v = 0; v < NV; ++v) A.rhs[(long long)v * st + c] = L[v];
        return;
    }
    const double* __restrict__ uin = B.buf[A.in_sel];
    const double* __restrict__ un = B.buf[A.n_sel];
    double* __restrict__ out = B.buf[A.out_sel];
    double r[NV];
    if (A.in_sel == A.n_sel) {  // stage 1 reads u^n as both the stage input and u^n: load it once
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double unv = __ldg(un + (long long)v * st + c);
            r[v] = rk_combine(A.a1, unv, A.a2, unv, A.a3dt, L[v]);
        }
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v)
            r[v] = rk_combine(A.a1, __ldg(un + (long long)v * st + c), A.a2, __ldg(uin + (long long)v * st + c),
                              A.a3dt, L[v]);
    }
    // floors, main.cpp:592-606
    {
        double& chi = r[CHI];
        bool bad = !isfinite(chi);
        if (bad || chi < 1.0e-4) chi = 1.0e-4;
        if (chi > 1.5) chi = 1.5;
        double& al = r[ALPHA];
        bool bad2 = !isfinite(al);
        if (bad2 || al < 1.0e-6) al = 1.0e-6;
        if ((bad || bad2) && A.nonfinite) atomicAdd(A.nonfinite, 1ull);
    }
    if (A.final_stage) algebraic_constraints(r);
#pragma unroll
    for (int v = 0; v < NV; ++v) out[(long long)v * st + c] = r[v];
}

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
    double L[NV];
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
    double L[NV];
    point_pm<PM>(B, uin, c, A, S, L);
    if (!valid) return;  // no barrier follows the last field
    stage_epilogue<EPI>(B, A, c, L);
}

// Variant 4: persistent CTAs (grid <= SMs x resident CTAs), one 16x4x4 tile
// at a time, every field streamed through the TMA ring. Threads of partial
// tiles (past the block edge) compute on the zero-filled box and store nothing.
template <int PM, int EPI, int NBUF, bool SEL>
__global__ void __launch_bounds__(V4_NT, 1)
    ccz4_stage_tma_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int ntiles,
                          StageArgs A) {
    using R = TmaRing<NBUF>;
    extern __shared__ unsigned char smem_raw[];
    double* ring = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    const unsigned bar0 = smem_addr(ring + (size_t)NBUF * R::BOX);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NBUF; ++s) mbar_init(bar0 + 8u * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // SEL: the CTA's tiles blockIdx.x + m gridDim.x whose flag equals want_prec,
    // compacted in order into shared memory once (ballot scan over 256 candidates
    // at a time); the host keeps ntiles <= gridDim.x * TMA_SEL_CAP.
    __shared__ int warp_cnt[V4_NT / 32];
    if constexpr (SEL) {
        int nsel = 0;
        const int ncand = ntiles > (int)blockIdx.x ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
        const int lane = tid & 31, warp = tid >> 5;
        for (int m0 = 0; m0 < ncand; m0 += V4_NT) {
            const int m = m0 + tid;
            const int ti = blockIdx.x + m * gridDim.x;
            const bool take = m < ncand && A.tile_prec[ti] == A.want_prec;
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (lane == 0) warp_cnt[warp] = __popc(bal);
            __syncthreads();
            int off = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < V4_NT / 32; ++w) {
                off += w < warp ? warp_cnt[w] : 0;
                tot += warp_cnt[w];
            }
            const int pos = nsel + off + __popc(bal & ((1u << lane) - 1u));
            if (take && pos < TMA_SEL_CAP) g_sel_list[pos] = ti;
            nsel += tot;
            __syncthreads();
        }
        if (tid == 0) g_sel_list[TMA_SEL_CAP] = nsel < TMA_SEL_CAP ? nsel : TMA_SEL_CAP;  // (host keeps it below)
    }
    __syncthreads();
    const int lx = tid % V4_TX, ly = (tid / V4_TX) % V4_TY, lz = tid / (V4_TX * V4_TY);
    TmaSource<NBUF, SEL> S{blocks, tiles, static_cast<const unsigned char*>(A.tmaps), ntiles, A.in_sel, ring, bar0,
                         nullptr, (lx + 4) + R::BX * ((ly + 4) + R::BY * (lz + 4)), 0, false,
                         A.errflag, 0, A.test_withhold};
    if (tid == 0)
        for (int q = 0; q < NBUF - 1; ++q) S.issue(q);
    for (int r = 0;; ++r) {
        const int ti = S.round_tile(r);
        if (ti >= ntiles) break;
        const Tile t = tiles[ti];
        const DevBlock& B = blocks[t.block];
        S.B = &B;
        const int i = t.i0 + lx, j = t.j0 + ly, k = t.k0 + lz;
        const bool valid = i < B.n[0] && j < B.n[1] && k < B.n[2];
        // pointwise loads of threads outside the block use a valid cell; their results are dropped
        const int ic = min(i, B.n[0] - 1), jc = min(j, B.n[1] - 1), kc = min(k, B.n[2] - 1);
        const long long c = cell_index(B, ic + NG, jc + NG, kc + NG);
        const double* __restrict__ uin = B.buf[A.in_sel];
        double L[NV];
        point_pm<PM>(B, uin, c, A, S, L);
        if (valid) stage_epilogue<EPI>(B, A, c, L);
    }
    // Every issued item was consumed (issue() skips items past this CTA's last
    // tile), so no copy into the ring is in flight when the CTA exits. If
    // thread 0 gave up waiting at item f (which already had its full wait), it
    // had issued items up to f + NBUF - 1 and nothing after: each of
    // f + 1 .. f + NBUF - 1 that was issued gets its own bounded wait, whatever
    // the others do, so no copy into this CTA's shared memory outlives it.
    if (S.failed && tid == 0) {
        const int f = S.fail_q;
        for (int q = f + 1; q < f + NBUF; ++q) {
            if (S.round_tile(q / NV) >= ntiles) continue;
            S.failed = false;
            S.wait(q);
        }
    }
}

// Per-tile precision flags: flag[ti] = 1 (FP64 algebra) when a point of tile ti
// has chi below chi_fp64 in buffer slot `sel` (or a non-finite chi), else 0.
__global__ void __launch_bounds__(128)
    classify_tiles_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int first, int sel,
                          int tx, int ty, int tz, double chi_fp64, unsigned char* __restrict__ flag) {
    const int ti = first + blockIdx.x;
    const Tile t = tiles[ti];
    const DevBlock& B = blocks[t.block];
    const int w = t.w > 0 ? t.w : tx, h = t.w > 0 ? 128 / t.w : ty, d = t.w > 0 ? 1 : tz;
    const double* chi = B.buf[sel] + (long long)CHI * B.stride;
    bool low = false;
    for (int p = threadIdx.x; p < w * h * d; p += blockDim.x) {
        const int i = t.i0 + p % w, j = t.j0 + (p / w) % h, k = t.k0 + p / (w * h);
        if (i < B.n[0] && j < B.n[1] && k < B.n[2])
            low |= !(__ldg(chi + cell_index(B, i + NG, j + NG, k + NG)) >= chi_fp64);
    }
    low = __syncthreads_or(low);
    if (threadIdx.x == 0) flag[ti] = low ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
constexpr int V0_TX = 32, V0_TY = 4, V0_TZ = 1;
constexpr int V1_TX = 16, V1_TY = 4, V1_TZ = 2, V1_NBUF = 3;
constexpr int V4_NBUF = 3;

int stage_tile_dims(int variant, int* tx, int* ty, int* tz) {
    if (variant == VARIANT_TMA) {
        *tx = V4_TX;
        *ty = V4_TY;
        *tz = V4_TZ;
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

// Persistent grid of the TMA variant on each device: SMs x resident CTAs.
constexpr int MAX_DEVICES = 64;
static int g_tma_grid[MAX_DEVICES][3][2];  // [device][precision mode][epi]

template <int PM, int EPI, bool SEL = false>
static cudaError_t configure_tma(int dev, int nsm) {
    auto k = ccz4_stage_tma_kernel<PM, EPI, V4_NBUF, SEL>;
    constexpr size_t bytes = TmaRing<V4_NBUF>::SMEM;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, V4_NT, bytes))) return e;
    if (!SEL) g_tma_grid[dev][PM][EPI] = nsm * (per_sm > 0 ? per_sm : 1);
    return cudaSuccess;
}

int tma_grid() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return 0;
    return g_tma_grid[dev][PM_MIXED][EPI_RK];
}

template <int PM, int EPI>
static cudaError_t launch_tma(const DevBlock* blocks, const Tile* tiles, int ntiles, const StageArgs& args,
                              cudaStream_t stream) {
    if (!args.tmaps) return cudaErrorInvalidValue;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int cap = (dev >= 0 && dev < MAX_DEVICES) ? g_tma_grid[dev][PM][EPI] : 0;
    if (cap <= 0) return cudaErrorInvalidConfiguration;  // configure_stage_kernels() not run on this device
    const int grid = ntiles < cap ? ntiles : cap;
    if (args.tile_prec) {  // per-tile precision passes (RK epilogue)
        if (EPI != EPI_RK) return cudaErrorInvalidValue;
        ccz4_stage_tma_kernel<PM, EPI_RK, V4_NBUF, true>
            <<<grid, V4_NT, TmaRing<V4_NBUF>::SMEM, stream>>>(blocks, tiles, ntiles, args);
    } else {
        ccz4_stage_tma_kernel<PM, EPI, V4_NBUF, false>
            <<<grid, V4_NT, TmaRing<V4_NBUF>::SMEM, stream>>>(blocks, tiles, ntiles, args);
    }
    return cudaGetLastError();
}

// Opt the shared-memory variants into more than 48 KB of dynamic shared memory
// on the current device and size the persistent grid (called once per context
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
    if ((e = configure_tma<PM_FP64, EPI_STORE>(dev, nsm))) return e;
    if ((e = configure_tma<PM_FP64, EPI_RK>(dev, nsm))) return e;
    if ((e = configure_tma<PM_MIXED, EPI_STORE>(dev, nsm))) return e;
    if ((e = configure_tma<PM_MIXED, EPI_RK>(dev, nsm))) return e;
    if ((e = configure_tma<PM_FP64F, EPI_RK>(dev, nsm))) return e;
    if ((e = configure_tma<PM_FP64, EPI_RK, true>(dev, nsm))) return e;
    if ((e = configure_tma<PM_FP64F, EPI_RK, true>(dev, nsm))) return e;
    return configure_tma<PM_MIXED, EPI_RK, true>(dev, nsm);
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
struct RunTma {
    static cudaError_t run(const DevBlock* b, const Tile* t, int n, const StageArgs& a, cudaStream_t s) {
        return launch_tma<PM, EPI>(b, t, n, a, s);
    }
};
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

cudaError_t launch_classify(int variant, const DevBlock* blocks, const Tile* tiles, int first, int ntiles, int sel,
                            double chi_fp64, unsigned char* flag, cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    int tx, ty, tz;
    stage_tile_dims(variant, &tx, &ty, &tz);
    classify_tiles_kernel<<<ntiles, 128, 0, stream>>>(blocks, tiles, first, sel, tx, ty, tz, chi_fp64, flag);
    return cudaGetLastError();
}

cudaError_t launch_stage(int variant, int precision, int epi, const DevBlock* blocks, const Tile* tiles, int ntiles,
                         const StageArgs& args, cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    switch (variant) {
        case VARIANT_TMA: return dispatch<RunTma>(precision, epi, blocks, tiles, ntiles, args, stream);
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
