// ccz4_stage_tma.cuh -- the TMA-ring stage kernel, templated on its tuning
// configuration. Each ccz4_tma_cfg<k>.cu instantiates one entry of TMA_CFGS
// (ccz4_kernels.h), so the configurations compile in parallel and the
// autotuner can pick one per block-size class at run time.
//
// A persistent CTA walks its tiles (blockIdx.x, + gridDim.x, ...) and consumes
// a stream of items q = (tile round q / NV, field FIELD_ORDER[q % NV]). Item q
// is one (16 + 8) x (4 + 8) x (TZ + 8)-cell box (the 16 x 4 x TZ tile and its
// 4-cell halo) of one field, brought into ring slot q % NBUF by a single
// cp.async.bulk.tensor load that completes on that slot's mbarrier. Every BAR
// items (BAR = 1 or 2) the CTA meets at a barrier, after which the slots of
// the last BAR items are free and thread 0 issues items q + NBUF - BAR ..
// q + NBUF - 1 into them: loads run NBUF - BAR to NBUF - 1 fields ahead, across
// tile boundaries. Rows of 24 doubles put the 16-wide x rows of a warp in
// distinct shared-memory banks for every stencil offset.
//
// Options of a configuration:
//   TIN  every field's centre value is copied from the ring into a per-thread
//        column of shared memory as it streams through, and the RK epilogue
//        reads the stage input there instead of from global memory;
//   PF   the epilogue's u^n cells and the next tile's pointwise cells are
//        prefetched into L2 at the start of each tile (always with TIN);
//   HS   the 36 values of the Hessian-field loop live in a per-thread column of
//        shared memory instead of local memory;
//   MINB resident CTAs per SM that the register allocation is sized for
//        (__launch_bounds__): 3 CTAs of 128 threads cap a thread at 168
//        registers, and the ring (with or without TIN) still fits three times in
//        an SM's shared memory;
//   BAR  ring items per CTA barrier: 2 halves the barriers of a tile (22 fields)
//        at the price of a shallower look-ahead on every other item.
#pragma once

#include <cstdint>
#include <type_traits>

#include "ccz4_point.cuh"

namespace granite_b200 {

namespace {

template <int TZ_, int NBUF_, bool TIN_, bool HS_, int MINB_, int BAR_ = 1, int REM_ = 0, bool PF_ = false>
struct TmaCfgT {
    static constexpr int TZ = TZ_, NBUF = NBUF_, BAR = BAR_;
    // a tile round's first item starts a barrier group (the round's shared push
    // boxes rely on it), and at least one item is loaded ahead
    static_assert((BAR == 1 || BAR == 2) && NV % BAR == 0 && NBUF > BAR, "barrier grouping");
    static constexpr bool TIN = TIN_, HS = HS_;
    // x-remainder tiles: REM, one box of the 2 TZ shape per field; REM2, two
    // boxes of this configuration's own shape per field (one per half of the
    // tile along z), two ring items that one barrier group frees together
    static constexpr bool REM = REM_ == 1, REM2 = REM_ == 2;
    static constexpr bool PF = TIN || PF_;  // the L2 prefetches at the start of each tile
    static constexpr int TX = 16, TY = 4, NT = TX * TY * TZ;
    static_assert(!REM2 || (BAR == 2 && TMA_REM_X * TY * 2 * TZ == NT), "two-box remainder tiles");
    static constexpr int MINB = MINB_;  // resident CTAs per SM asked of the register allocator
    static constexpr int BX = TX + 8, BY = TY + 8, BZ = TZ + 8;
    static constexpr int BOX = BX * BY * BZ;
    static constexpr unsigned BYTES = BOX * sizeof(double);  // complete_tx count of one item
    // x-remainder tiles: TMA_REM_X x TY x 2 TZ points, the same rows (BX, BY) and
    // 2 TZ + 8 planes per box, so the stencil offsets stay those of the full tiles
    static_assert(!REM || (tma_shape_for_tz(2 * TZ) >= 0 && TMA_REM_X * TY * 2 * TZ == NT),
                  "remainder tiles: one point per thread, loaded with the 2 TZ box shape");
    static constexpr int BOX_REM = BX * BY * (2 * TZ + 8);
    static constexpr unsigned BYTES_REM = BOX_REM * sizeof(double);
    static constexpr int SLOT = REM ? BOX_REM : BOX;  // doubles per ring slot
    static_assert(BYTES % 128 == 0 && (SLOT * sizeof(double)) % 128 == 0, "slots stay 128-byte aligned");
    static_assert(BX == TMA_BOX_X && BY == TMA_BOX_Y, "box = tile + halo");
    // dynamic shared memory: ring | mbarriers | stage-input column | Hessian slots
    static constexpr size_t OFF_BAR = (size_t)NBUF * SLOT * sizeof(double);
    static constexpr size_t OFF_TIN = (OFF_BAR + NBUF * sizeof(unsigned long long) + 127) / 128 * 128;
    static constexpr size_t OFF_HS = OFF_TIN + (TIN ? (size_t)NV * NT * sizeof(double) : 0);
    template <typename P>
    static constexpr size_t smem() {
        return OFF_HS + (HS ? (size_t)36 * NT * sizeof(P) : 0) + 128;  // + alignment of the base
    }
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
// The same test with a suspend-time hint: a thread whose phase is not complete
// yet is suspended (issuing nothing) until it completes or about hint_ns pass,
// instead of spinning.
__device__ __forceinline__ bool mbar_try_wait_sleep(unsigned bar, unsigned parity, unsigned hint_ns) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
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
// Bring the line holding p into L2 with the evict-last priority (a hint: no
// register, no completion to wait for).
__device__ __forceinline__ void prefetch_l2(const double* p) {
    asm volatile("prefetch.global.L2::evict_last [%0];" ::"l"(p));
}

// Wait limit of one ring slot: 2 s of wall time, then the kernel records the
// failure in StageArgs::errflag and stops waiting (results are then garbage
// and the host reports the error).
constexpr unsigned long long TMA_WAIT_NS = 2000000000ull;
// Suspend-time hint of one wait attempt (the limit is checked between attempts).
constexpr unsigned TMA_WAIT_HINT_NS = 100000u;

// Per-tile precision launches: the CTA's selected tiles, in order, and their
// count at [TMA_SEL_CAP] (shared memory at a fixed address, so the per-point
// body keeps no register for them).
__shared__ int g_sel_list[TMA_SEL_CAP + 1];

template <class C, bool SEL>
struct TmaSource {
    static constexpr bool HS = C::HS, UNROLL = false;
    static constexpr int NT = C::NT;
    const DevBlock* blocks;
    const Tile* tiles;
    const unsigned char* maps;  // CUtensorMap array of this box shape, 128 bytes each
    const unsigned char* maps_rem;  // REM: the same for the remainder tiles' box shape
    int ntiles, in_sel;
    double* ring;      // NBUF slots of C::SLOT doubles
    unsigned bar0;     // shared address of the slot mbarriers (8 bytes apart)
    double* tin;       // TIN: this thread's stage-input column (field v at tin[v * NT])
    void* hs;          // HS: this thread's Hessian-loop column (slot q at hs[q * NT])
    const DevBlock* B; // block of the current tile (stencil coefficients)
    int lin;           // this thread's point within a slot
    int next;          // next item to consume
    bool failed;       // a wait of this thread gave up (at item fail_q); thread 0 then stops issuing
    unsigned int* err;
    int fail_q;
    int withhold;      // test switch: 1 + the item CTA 0 leaves unissued (0: none)
    // REM2: the item stream has 2 NV items in a remainder tile's round (field
    // FIELD_ORDER[p / 2], half p % 2), NV in the others; thread 0 keeps its issue
    // position as a cursor (round, position, items issued)
    int ic_round = 0, ic_pos = 0, issued = 0;
    bool rem_round = false;  // REM2: the current round is a remainder tile
    int half = 0;            // REM2: this thread's half of a remainder tile

    template <typename P>
    __device__ __forceinline__ P* hess_slots() const {
        return static_cast<P*>(hs);
    }
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
        const bool rem = C::REM && t.w < 0;
        const int s = q % C::NBUF;
        const unsigned bar = bar0 + 8u * s;
        mbar_expect_tx(bar, rem ? C::BYTES_REM : C::BYTES);
        // box origin = tile origin - 4 cells = interior index (cells incl. ghosts start 4 lower)
        tma_load_box(smem_addr(ring + (size_t)s * C::SLOT), (rem ? maps_rem : maps) + (size_t)(3 * t.block + in_sel) * 128,
                     t.i0, t.j0, t.k0, FIELD_ORDER[q % NV], bar);
    }
    // thread 0 only (REM2): issue the next item of the stream
    __device__ __forceinline__ void issue_next() {
        const int ti = round_tile(ic_round);
        if (ti >= ntiles) return;  // nothing after the CTA's last tile
        const Tile t = tiles[ti];
        const bool rem = t.w < 0;
        const int q = issued++;
        const int fpos = rem ? ic_pos >> 1 : ic_pos, hf = rem ? ic_pos & 1 : 0;
        if (++ic_pos == (rem ? 2 * NV : NV)) {
            ++ic_round;
            ic_pos = 0;
        }
        if (withhold != 0 && q == withhold - 1 && blockIdx.x == 0) return;  // test switch: never issued
        const int s = q % C::NBUF;
        const unsigned bar = bar0 + 8u * s;
        mbar_expect_tx(bar, C::BYTES);
        tma_load_box(smem_addr(ring + (size_t)s * C::SLOT), maps + (size_t)(3 * t.block + in_sel) * 128, t.i0, t.j0,
                     t.k0 + hf * C::TZ, FIELD_ORDER[fpos], bar);
    }
    __device__ __forceinline__ void wait(int q) {
        if (failed) return;
        const unsigned bar = bar0 + 8u * (q % C::NBUF), parity = (q / C::NBUF) & 1;
        if (mbar_try_wait(bar, parity)) return;
        const unsigned long long t0 = global_ns();
        for (;;) {
            if (mbar_try_wait_sleep(bar, parity, TMA_WAIT_HINT_NS)) return;
            if (global_ns() - t0 > TMA_WAIT_NS) {
                failed = true;
                fail_q = q;
                if (err) atomicExch(err, 1u);
                return;
            }
        }
    }
    // Every thread of the CTA calls der() for every item in order (every BAR-th
    // call carries the CTA barrier that frees the slots of the last BAR items,
    // which the next BAR loads overwrite).
    template <bool HESS, bool EXACT, typename P>
    __device__ __forceinline__ FieldDer<P> der(int v, const double beta[3], P w) {
        int q = next;
        if constexpr (C::REM2) {
            // a remainder tile's field is two items (one per half): its der()
            // always starts a barrier group and consumes both
            if (next % 2 == 0) {
                __syncthreads();
                if (threadIdx.x == 0 && !failed) {
                    issue_next();
                    issue_next();
                }
            }
            q = next + (rem_round ? half : 0);
            next += rem_round ? 2 : 1;
        } else {
            if (next % C::BAR == 0) {
                __syncthreads();
                if (threadIdx.x == 0 && !failed)
#pragma unroll
                    for (int j = C::NBUF - C::BAR; j < C::NBUF; ++j) issue(next + j);
            }
            ++next;
        }
        wait(q);
        const double* box = ring + (size_t)(q % C::NBUF) * C::SLOT + lin;
        if constexpr (C::TIN) tin[v * NT] = box[0];
        const SharedLoad L{box};
        const long long off[3] = {1, C::BX, C::BX * C::BY};
        return field_der_l<P, HESS, true, SharedLoad, EXACT>(*B, L, off, beta, w);
    }
};

}  // namespace

// Persistent CTAs (grid <= SMs x resident CTAs), one 16 x 4 x TZ tile at a
// time, every field streamed through the TMA ring. Threads of partial tiles
// (past the block edge) compute on the zero-filled box and store nothing.
template <int PM, int EPI, class C, bool SEL>
__global__ void __launch_bounds__(C::NT, C::MINB)
    ccz4_stage_tma_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int ntiles,
                          StageArgs A) {
    using P = typename std::conditional<PM == PM_MIXED, float, double>::type;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) &
                                                           ~uintptr_t(127));
    double* ring = reinterpret_cast<double*>(base);
    const unsigned bar0 = smem_addr(base + C::OFF_BAR);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < C::NBUF; ++s) mbar_init(bar0 + 8u * s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // SEL: the CTA's tiles blockIdx.x + m gridDim.x whose flag equals want_prec,
    // compacted in order into shared memory once (ballot scan over NT candidates
    // at a time); the host keeps ntiles <= gridDim.x * TMA_SEL_CAP.
    __shared__ int warp_cnt[C::NT / 32];
    if constexpr (SEL) {
        int nsel = 0;
        const int ncand = ntiles > (int)blockIdx.x ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
        const int lane = tid & 31, warp = tid >> 5;
        for (int m0 = 0; m0 < ncand; m0 += C::NT) {
            const int m = m0 + tid;
            const int ti = blockIdx.x + m * gridDim.x;
            const bool take = m < ncand && A.tile_prec[ti] == A.want_prec;
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (lane == 0) warp_cnt[warp] = __popc(bal);
            __syncthreads();
            int off = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < C::NT / 32; ++w) {
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
    // push boxes of the current tile, double-buffered by tile round: staged when
    // the round starts, read in its epilogue (the round's first field barrier
    // lies between), overwritten two rounds later
    __shared__ PushBox s_push[2][PUSH_STAGE_MAX];
    // this thread's point within a tile: 16 x 4 x TZ, or TMA_REM_X x 4 x 2 TZ
    // for an x-remainder tile (the box rows are the same, so is the stencil code)
    auto local = [&](const Tile& t, int& px, int& py, int& pz) {
        if ((C::REM || C::REM2) && t.w < 0) {
            px = tid % TMA_REM_X;
            py = (tid / TMA_REM_X) % C::TY;
            pz = tid / (TMA_REM_X * C::TY);
        } else {
            px = tid % C::TX;
            py = (tid / C::TX) % C::TY;
            pz = tid / (C::TX * C::TY);
        }
    };
    double* tin = C::TIN ? reinterpret_cast<double*>(base + C::OFF_TIN) + tid : nullptr;
    void* hs = C::HS ? static_cast<void*>(reinterpret_cast<P*>(base + C::OFF_HS) + tid) : nullptr;
    TmaSource<C, SEL> S{blocks, tiles, static_cast<const unsigned char*>(A.tmaps),
                        static_cast<const unsigned char*>(A.tmaps_rem), ntiles, A.in_sel, ring, bar0,
                        tin, hs, nullptr, 0, 0, false, A.errflag, 0, A.test_withhold};
    if (tid == 0) {
        if constexpr (C::REM2)
            for (int q = 0; q < C::NBUF - C::BAR; ++q) S.issue_next();
        else
            for (int q = 0; q < C::NBUF - C::BAR; ++q) S.issue(q);
    }
    for (int r = 0;; ++r) {
        const int ti = S.round_tile(r);
        if (ti >= ntiles) break;
        const Tile t = tiles[ti];
        const DevBlock& B = blocks[t.block];
        S.B = &B;
        int lx, ly, lz;
        local(t, lx, ly, lz);
        if constexpr (C::REM2) {
            // a remainder tile's two halves along z each have their own box
            S.rem_round = t.w < 0;
            S.half = S.rem_round ? lz / C::TZ : 0;
            S.lin = (lx + 4) + C::BX * ((ly + 4) + C::BY * (lz - S.half * C::TZ + 4));
        } else {
            S.lin = (lx + 4) + C::BX * ((ly + 4) + C::BY * (lz + 4));
        }
        const int i = t.i0 + lx, j = t.j0 + ly, k = t.k0 + lz;
        const bool valid = i < B.n[0] && j < B.n[1] && k < B.n[2];
        // pointwise loads of threads outside the block use a valid cell; their results are dropped
        const int ic = min(i, B.n[0] - 1), jc = min(j, B.n[1] - 1), kc = min(k, B.n[2] - 1);
        const long long c = cell_index(B, ic + NG, jc + NG, kc + NG);
        const double* __restrict__ uin = B.buf[A.in_sel];
        const PushBox* pushes = nullptr;
        int npush = 0;
        if (A.push) {
            const int2 pr = A.tile_push[ti];
            npush = pr.y;
            if (npush <= PUSH_STAGE_MAX) {
                if (tid < npush) s_push[r & 1][tid] = A.push[pr.x + tid];
                pushes = s_push[r & 1];
            } else {
                pushes = A.push + pr.x;
            }
        }
        if constexpr (C::PF) {
            // L2 prefetches: this tile's u^n (read by the epilogue; stage 1 takes
            // it from the ring) and the next tile's pointwise cells
            if (EPI == EPI_RK && A.n_sel != A.in_sel) {
                const double* un = B.buf[A.n_sel] + c;
#pragma unroll
                for (int v = 0; v < NV; ++v) prefetch_l2(un + (long long)v * B.stride);
            }
            const int tn = S.round_tile(r + 1);
            if (tn < ntiles) {
                const Tile t2 = tiles[tn];
                const DevBlock& B2 = blocks[t2.block];
                int x2, y2, z2;
                local(t2, x2, y2, z2);
                const long long c2 = cell_index(B2, min(t2.i0 + x2, B2.n[0] - 1) + NG, min(t2.j0 + y2, B2.n[1] - 1) + NG,
                                                min(t2.k0 + z2, B2.n[2] - 1) + NG);
                const double* u2 = B2.buf[A.in_sel] + c2;
#pragma unroll
                for (int v = 0; v < NV; ++v) prefetch_l2(u2 + (long long)v * B2.stride);
            }
        }
        AlgebraT<PM> L[NV];
        point_pm<PM>(B, uin, c, A, S, L);
        if (valid) stage_epilogue<EPI>(B, A, c, L, tin, C::NT, pushes, npush, i, j, k);
    }
    // Every issued item was consumed (issue() skips items past this CTA's last
    // tile), so no copy into the ring is in flight when the CTA exits. If
    // thread 0 gave up waiting at item f (which already had its full wait), it
    // had issued items up to f0 + NBUF - 1 (f0 = f rounded down to its barrier
    // group) and nothing after: each of f + 1 .. f0 + NBUF - 1 that was issued
    // gets its own bounded wait, whatever the others do, so no copy into this
    // CTA's shared memory outlives it.
    if (S.failed && tid == 0) {
        const int f = S.fail_q;
        if constexpr (C::REM2) {
            // the cursor counted every item issued (one the test switch withheld
            // included: its wait runs out as that of item f did)
            for (int q = f + 1; q < S.issued; ++q) {
                S.failed = false;
                S.wait(q);
            }
        } else {
            for (int q = f + 1; q < f - f % C::BAR + C::NBUF; ++q) {
                if (S.round_tile(q / NV) >= ntiles) continue;
                S.failed = false;
                S.wait(q);
            }
        }
    }
}

// Launchers of one configuration: grids[pm][epi][sel] is the persistent grid
// (SMs x resident CTAs) measured by tma_configure; 0 = not instantiated.
template <class C>
struct TmaConfigOps {
    template <int PM, int EPI, bool SEL>
    static cudaError_t configure_one(int nsm, int grids[3][2][2]) {
        using P = typename std::conditional<PM == PM_MIXED, float, double>::type;
        auto k = ccz4_stage_tma_kernel<PM, EPI, C, SEL>;
        constexpr size_t bytes = C::template smem<P>();
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, C::NT, bytes))) return e;
        grids[PM][EPI][SEL ? 1 : 0] = nsm * (per_sm > 0 ? per_sm : 1);
        return cudaSuccess;
    }
    template <int PM, int EPI, bool SEL>
    static cudaError_t launch_one(const DevBlock* blocks, const Tile* tiles, int ntiles, const StageArgs& args,
                                  cudaStream_t stream, int grid) {
        using P = typename std::conditional<PM == PM_MIXED, float, double>::type;
        ccz4_stage_tma_kernel<PM, EPI, C, SEL>
            <<<grid, C::NT, C::template smem<P>(), stream>>>(blocks, tiles, ntiles, args);
        return cudaGetLastError();
    }
    // The RK-epilogue kernels every configuration has (FP64; MIXED with and
    // without per-tile selection; the FP64 pass of the per-tile precision),
    // plus the store epilogue where STORE is set.
    template <bool STORE>
    static cudaError_t configure(int nsm, int grids[3][2][2]) {
        cudaError_t e;
        if ((e = configure_one<PM_FP64, EPI_RK, false>(nsm, grids))) return e;
        if ((e = configure_one<PM_MIXED, EPI_RK, false>(nsm, grids))) return e;
        if ((e = configure_one<PM_MIXED, EPI_RK, true>(nsm, grids))) return e;
        if ((e = configure_one<PM_FP64F, EPI_RK, true>(nsm, grids))) return e;
        if constexpr (STORE) {
            if ((e = configure_one<PM_FP64, EPI_STORE, false>(nsm, grids))) return e;
            if ((e = configure_one<PM_MIXED, EPI_STORE, false>(nsm, grids))) return e;
        }
        return cudaSuccess;
    }
    template <bool STORE>
    static cudaError_t launch(int pm, int epi, bool sel, const DevBlock* blocks, const Tile* tiles, int ntiles,
                              const StageArgs& args, cudaStream_t stream, int grid) {
        if (epi == EPI_RK) {
            if (pm == PM_FP64 && !sel) return launch_one<PM_FP64, EPI_RK, false>(blocks, tiles, ntiles, args, stream, grid);
            if (pm == PM_MIXED && !sel) return launch_one<PM_MIXED, EPI_RK, false>(blocks, tiles, ntiles, args, stream, grid);
            if (pm == PM_MIXED && sel) return launch_one<PM_MIXED, EPI_RK, true>(blocks, tiles, ntiles, args, stream, grid);
            if (pm == PM_FP64F && sel) return launch_one<PM_FP64F, EPI_RK, true>(blocks, tiles, ntiles, args, stream, grid);
        } else if constexpr (STORE) {
            if (pm == PM_FP64 && !sel) return launch_one<PM_FP64, EPI_STORE, false>(blocks, tiles, ntiles, args, stream, grid);
            if (pm == PM_MIXED && !sel) return launch_one<PM_MIXED, EPI_STORE, false>(blocks, tiles, ntiles, args, stream, grid);
        }
        return cudaErrorInvalidValue;
    }
};

}  // namespace granite_b200

// One translation unit per configuration k of TMA_CFGS defines its entry points.
#define GRANITE_TMA_CFG_UNIT(K, STORE)                                                                               \
    namespace granite_b200 {                                                                                         \
    using TmaCfg##K =                                                                                                \
        TmaCfgT<TMA_CFGS[K].tz, TMA_CFGS[K].nbuf, TMA_CFGS[K].tin != 0, TMA_CFGS[K].hs != 0, TMA_CFGS[K].minb,      \
                TMA_CFGS[K].bar, TMA_CFGS[K].rem, TMA_CFGS[K].pf != 0>;                                              \
    cudaError_t configure_tma_cfg##K(int nsm, int grids[3][2][2]) {                                                  \
        return TmaConfigOps<TmaCfg##K>::configure<STORE>(nsm, grids);                                                \
    }                                                                                                                \
    cudaError_t launch_tma_cfg##K(int pm, int epi, bool sel, const DevBlock* blocks, const Tile* tiles, int ntiles,  \
                                  const StageArgs& args, cudaStream_t stream, int grid) {                            \
        return TmaConfigOps<TmaCfg##K>::launch<STORE>(pm, epi, sel, blocks, tiles, ntiles, args, stream, grid);      \
    }                                                                                                                \
    }
