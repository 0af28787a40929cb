// ccz4_stage_ws.cuh -- warp-specialized TMA stage kernel of the mixed form.
//
// The stage kernel of ccz4_stage_tma.cuh runs the stencils and the algebra of
// a point in one thread, which needs ~250 registers and leaves 8 warps per SM.
// Here the two halves of that work run in different warps of the CTA, with a
// ring of derivative slots in shared memory between them:
//
//   warps 4-7 (producers, 88 registers): per field, wait for its TMA box in the
//     ring, evaluate the field's stencils at their point (FP64 pair
//     differences rounded to FP32 after the cancellation, exactly as the fused
//     kernel does: d_i, the blended advection, KO, and the Hessian where the
//     algebra needs it) and write the 11 values into the next derivative slot;
//   warps 0-3 (consumers, 168 registers): the CCZ4 algebra of ccz4_point on
//     those values, the RK combine, floors and algebraic constraints.
//
// The launch gives every thread 128 registers (256 threads, two CTAs per SM,
// 16 warps per SM); setmaxnreg moves 40 registers per thread from the
// producer warpgroup to the consumer warpgroup (128 x 88 + 128 x 168 =
// 256 x 128). The host enables the kernel only when the launch register count
// covers that split (ws_registers_ok).
//
// Tiles are 16 x 4 x 2 points (the tile shape of the tz = 2 configurations, so
// the FP64 pass of the per-tile precision shares its tile list). Every wait is
// bounded (TMA_WAIT_NS): a thread whose wait gives up records it in
// StageArgs::errflag and skips its later waits, so the kernel always ends.
#pragma once

#include "ccz4_stage_tma.cuh"

namespace granite_b200 {

namespace {

template <int NBUF_, int DBUF_>
struct WsCfgT {
    static constexpr int TX = 16, TY = 4, TZ = 2, NP = TX * TY * TZ, NTHR = 2 * NP, MINB = 2;
    static constexpr int NBUF = NBUF_, DBUF = DBUF_;
    static constexpr int BX = TX + 8, BY = TY + 8, BZ = TZ + 8, BOX = BX * BY * BZ;
    static constexpr unsigned BYTES = BOX * sizeof(double);
    static_assert(BYTES % 128 == 0, "slots stay 128-byte aligned");
    static constexpr int DVALS = 11;  // d[3], adv, ko, h[6]
    static constexpr size_t DSLOT = (size_t)DVALS * NP * sizeof(float);
    // dynamic shared memory: TMA ring | TMA mbarriers | derivative slots | full | empty
    static constexpr size_t OFF_TBAR = (size_t)NBUF * BYTES;
    static constexpr size_t OFF_DER = (OFF_TBAR + NBUF * sizeof(unsigned long long) + 127) / 128 * 128;
    static constexpr size_t OFF_FULL = OFF_DER + DBUF * DSLOT;
    static constexpr size_t OFF_EMPTY = OFF_FULL + DBUF * sizeof(unsigned long long);
    static constexpr size_t SMEM = OFF_EMPTY + DBUF * sizeof(unsigned long long) + 128;
    static constexpr int PROD_REGS = 88, CONS_REGS = 168;
    static_assert(NP * PROD_REGS + NP * CONS_REGS == NTHR * 128, "the split moves registers, it adds none");
};

__device__ __forceinline__ void mbar_arrive(unsigned bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
// Bounded wait for the completion of the phase of parity `parity`; on a
// timeout the failure is recorded and the thread's later waits are skipped.
// (A waiting warp is suspended rather than spinning, so it takes no issue
// slots from the warps it waits for.)
__device__ __forceinline__ void ws_wait(unsigned bar, unsigned parity, bool& failed, unsigned int* err) {
    if (failed) return;
    if (mbar_try_wait(bar, parity)) return;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try_wait_sleep(bar, parity, TMA_WAIT_HINT_NS)) return;
        if (global_ns() - t0 > TMA_WAIT_NS) {
            failed = true;
            if (err) atomicExch(err, 1u);
            return;
        }
    }
}
// One arrival per warp, after every lane's shared-memory accesses (the warp
// barrier orders them before lane 0's release).
__device__ __forceinline__ void warp_arrive(unsigned bar) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(bar);
}
__device__ __forceinline__ void producer_barrier() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }

// Fields whose Hessian the algebra uses (ccz4_point asks der<true> for them):
// FIELD_ORDER positions 0-5 (gt_ij), 9 (chi), 10 (alpha), 11-13 (beta^i).
__device__ __forceinline__ bool hessian_position(int f) { return f <= 5 || (f >= 9 && f <= 13); }

// The consumers' stencil source: derivative slots filled by the producers.
template <class C>
struct DerivSource {
    static constexpr bool HS = false, UNROLL = true;
    const float* dring;  // DBUF slots of DVALS x NP floats
    unsigned full0, empty0;
    int pt;               // this thread's point in the tile
    int q;                // next item (tile round q / NV, field q % NV)
    bool failed;
    unsigned int* err;
    template <bool HESS, bool EXACT, typename P>
    __device__ __forceinline__ FieldDer<P> der(int /*v*/, const double /*beta*/[3], P /*w*/) {
        static_assert(sizeof(P) == sizeof(float), "the producers write FP32 derivatives");
        const int d = q % C::DBUF;
        ws_wait(full0 + 8u * d, (unsigned)(q / C::DBUF) & 1u, failed, err);
        const float* s = dring + (size_t)d * C::DVALS * C::NP + pt;
        FieldDer<P> r;
        r.d[0] = s[0];
        r.d[1] = s[C::NP];
        r.d[2] = s[2 * C::NP];
        r.adv = s[3 * C::NP];
        r.ko = s[4 * C::NP];
#pragma unroll
        for (int a = 0; a < 6; ++a) r.h[a] = HESS ? s[(5 + a) * C::NP] : (P)0;
        warp_arrive(empty0 + 8u * d);
        ++q;
        return r;
    }
};

}  // namespace

template <int EPI, class C, bool SEL>
__global__ void __launch_bounds__(C::NTHR, C::MINB)
    ccz4_stage_ws_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int ntiles,
                         StageArgs A) {
    using P = float;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) &
                                                           ~uintptr_t(127));
    double* ring = reinterpret_cast<double*>(base);
    const unsigned tbar0 = smem_addr(base + C::OFF_TBAR);
    const unsigned full0 = smem_addr(base + C::OFF_FULL), empty0 = smem_addr(base + C::OFF_EMPTY);
    float* dring = reinterpret_cast<float*>(base + C::OFF_DER);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < C::NBUF; ++s) mbar_init(tbar0 + 8u * s, 1);
        for (int s = 0; s < C::DBUF; ++s) {
            mbar_init(full0 + 8u * s, C::NP / 32);   // every producer warp arrives
            mbar_init(empty0 + 8u * s, C::NP / 32);  // every consumer warp arrives
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // SEL: the CTA's tiles blockIdx.x + m gridDim.x whose flag equals want_prec,
    // compacted in order into shared memory once (all threads, before the split)
    __shared__ int warp_cnt[C::NTHR / 32];
    if constexpr (SEL) {
        int nsel = 0;
        const int ncand = ntiles > (int)blockIdx.x ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
        const int lane = tid & 31, warp = tid >> 5;
        for (int m0 = 0; m0 < ncand; m0 += C::NTHR) {
            const int m = m0 + tid;
            const int ti = blockIdx.x + m * gridDim.x;
            const bool take = m < ncand && A.tile_prec[ti] == A.want_prec;
            const unsigned bal = __ballot_sync(0xffffffffu, take);
            if (lane == 0) warp_cnt[warp] = __popc(bal);
            __syncthreads();
            int off = 0, tot = 0;
#pragma unroll
            for (int w = 0; w < C::NTHR / 32; ++w) {
                off += w < warp ? warp_cnt[w] : 0;
                tot += warp_cnt[w];
            }
            const int pos = nsel + off + __popc(bal & ((1u << lane) - 1u));
            if (take && pos < TMA_SEL_CAP) g_sel_list[pos] = ti;
            nsel += tot;
            __syncthreads();
        }
        if (tid == 0) g_sel_list[TMA_SEL_CAP] = nsel < TMA_SEL_CAP ? nsel : TMA_SEL_CAP;
    }
    __syncthreads();
    auto round_tile = [&](int r) -> int {
        if constexpr (SEL)
            return r < g_sel_list[TMA_SEL_CAP] ? g_sel_list[r] : ntiles;
        else
            return blockIdx.x + r * gridDim.x;
    };
    const int pt = tid & (C::NP - 1);  // point of the tile (producer and consumer alike)
    const int lx = pt % C::TX, ly = (pt / C::TX) % C::TY, lz = pt / (C::TX * C::TY);

    if (tid >= C::NP) {
        // ------------------------------ producers ------------------------------
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(C::PROD_REGS));
        const unsigned char* maps = static_cast<const unsigned char*>(A.tmaps);
        bool failed = false;  // a wait of this thread gave up
        int waited_ok = -1;   // the last TMA item this thread waited for successfully
        int issued_hi = -1;   // (thread 0 of the producers) the last TMA item it issued
        auto issue = [&](int q) {
            const int ti = round_tile(q / NV);
            if (ti >= ntiles) return;
            issued_hi = q;
            if (A.test_withhold != 0 && q == A.test_withhold - 1 && blockIdx.x == 0) return;  // test switch
            const Tile t = tiles[ti];
            const int s = q % C::NBUF;
            const unsigned bar = tbar0 + 8u * s;
            mbar_expect_tx(bar, C::BYTES);
            tma_load_box(smem_addr(ring + (size_t)s * C::BOX), maps + (size_t)(3 * t.block + A.in_sel) * 128, t.i0,
                         t.j0, t.k0, FIELD_ORDER[q % NV], bar);
        };
        if (pt == 0)
            for (int q = 0; q < C::NBUF - 1; ++q) issue(q);
        const int lin = (lx + 4) + C::BX * ((ly + 4) + C::BY * (lz + 4));
        const long long off[3] = {1, C::BX, C::BX * C::BY};
        int q = 0;
        for (int r = 0;; ++r) {
            const int ti = round_tile(r);
            if (ti >= ntiles) break;
            const Tile t = tiles[ti];
            const DevBlock& B = blocks[t.block];
            const int ic = min(t.i0 + lx, B.n[0] - 1), jc = min(t.j0 + ly, B.n[1] - 1), kc = min(t.k0 + lz, B.n[2] - 1);
            const long long c = cell_index(B, ic + NG, jc + NG, kc + NG);
            const double* __restrict__ uin = B.buf[A.in_sel] + c;
            // the pointwise values the stencils need: the shift (upwind side) and
            // the blend weight from chi (ccz4.cpp:279-280, 565)
            double beta[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) beta[a] = __ldg(uin + (long long)(BETAX + a) * B.stride);
            const double chi_raw = __ldg(uin + (long long)CHI * B.stride);
            const double chi = (isfinite(chi_raw) && chi_raw >= 1.0e-4) ? chi_raw : 1.0e-4;
            const P w = (P)(0.5 * (1.0 + tanh((chi - A.chi_c) / A.chi_w)));
            for (int f = 0; f < NV; ++f, ++q) {
                producer_barrier();  // every producer is done with the slot the next load overwrites
                if (pt == 0 && !failed) issue(q + C::NBUF - 1);
                ws_wait(tbar0 + 8u * (q % C::NBUF), (unsigned)(q / C::NBUF) & 1u, failed, A.errflag);
                if (!failed) waited_ok = q;
                const SharedLoad L{ring + (size_t)(q % C::NBUF) * C::BOX + lin};
                FieldDer<P> fd;
                const bool hess = hessian_position(f);
                if (hess)
                    fd = field_der_l<P, true, true, SharedLoad, false>(B, L, off, beta, w);
                else
                    fd = field_der_l<P, false, true, SharedLoad, false>(B, L, off, beta, w);
                const int d = q % C::DBUF;
                ws_wait(empty0 + 8u * d, ((unsigned)(q / C::DBUF) & 1u) ^ 1u, failed, A.errflag);
                float* s = dring + (size_t)d * C::DVALS * C::NP + pt;
                s[0] = fd.d[0];
                s[C::NP] = fd.d[1];
                s[2 * C::NP] = fd.d[2];
                s[3 * C::NP] = fd.adv;
                s[4 * C::NP] = fd.ko;
                if (hess) {
#pragma unroll
                    for (int a = 0; a < 6; ++a) s[(5 + a) * C::NP] = fd.h[a];
                }
                warp_arrive(full0 + 8u * d);
            }
        }
        // no bulk copy into shared memory may outlive the CTA: when a wait of the
        // issuing thread gave up (on a TMA item or a derivative slot), every item
        // it issued after the last one it waited for gets its own bounded wait
        // (at most NBUF - 1 items, one per ring slot)
        if (pt == 0 && failed) {
            for (int qq = waited_ok + 1; qq <= issued_hi; ++qq) {
                if (A.test_withhold != 0 && qq == A.test_withhold - 1 && blockIdx.x == 0) continue;  // never issued
                bool f2 = false;
                ws_wait(tbar0 + 8u * (qq % C::NBUF), (unsigned)(qq / C::NBUF) & 1u, f2, A.errflag);
            }
        }
        return;
    }
    // ------------------------------ consumers ------------------------------
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(C::CONS_REGS));
    DerivSource<C> S{dring, full0, empty0, pt, 0, false, A.errflag};
    for (int r = 0;; ++r) {
        const int ti = round_tile(r);
        if (ti >= ntiles) break;
        const Tile t = tiles[ti];
        const DevBlock& B = blocks[t.block];
        const int i = t.i0 + lx, j = t.j0 + ly, k = t.k0 + lz;
        const bool valid = i < B.n[0] && j < B.n[1] && k < B.n[2];
        const int ic = min(i, B.n[0] - 1), jc = min(j, B.n[1] - 1), kc = min(k, B.n[2] - 1);
        const long long c = cell_index(B, ic + NG, jc + NG, kc + NG);
        const double* __restrict__ uin = B.buf[A.in_sel];
        // L2 prefetches: this tile's u^n (the epilogue's) and the next tile's pointwise cells
        if (EPI == EPI_RK && A.n_sel != A.in_sel) {
            const double* un = B.buf[A.n_sel] + c;
#pragma unroll
            for (int v = 0; v < NV; ++v) prefetch_l2(un + (long long)v * B.stride);
        }
        const int tn = round_tile(r + 1);
        if (tn < ntiles) {
            const Tile t2 = tiles[tn];
            const DevBlock& B2 = blocks[t2.block];
            const long long c2 = cell_index(B2, min(t2.i0 + lx, B2.n[0] - 1) + NG, min(t2.j0 + ly, B2.n[1] - 1) + NG,
                                            min(t2.k0 + lz, B2.n[2] - 1) + NG);
            const double* u2 = B2.buf[A.in_sel] + c2;
#pragma unroll
            for (int v = 0; v < NV; ++v) prefetch_l2(u2 + (long long)v * B2.stride);
        }
        P L[NV];
        ccz4_point<P, false>(B, uin, c, A, S, L);
        // (the consumers have no tile barrier to stage the push boxes behind: global reads)
        const int2 pr = A.push ? A.tile_push[ti] : make_int2(0, 0);
        if (valid) stage_epilogue<EPI>(B, A, c, L, nullptr, 0, A.push ? A.push + pr.x : nullptr, pr.y, i, j, k);
    }
}

// Launch-time check of the register split: the launch must give every thread
// at least 128 registers, or the consumers' setmaxnreg.inc would wait for
// registers that never free up.
template <class C, bool SEL>
bool ws_registers_ok() {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, ccz4_stage_ws_kernel<EPI_RK, C, SEL>) != cudaSuccess) return false;
    return (long long)fa.numRegs * C::NTHR >= (long long)C::NP * (C::PROD_REGS + C::CONS_REGS);
}

// The configuration's operations: the mixed RK kernels are warp-specialized;
// the FP64 kernel and the FP64 pass of the per-tile precision are the fused
// kernel with the same 16 x 4 x 2 tiles (T, a TmaCfgT of tz = 2).
template <class C, class T>
struct WsConfigOps {
    template <bool SEL>
    static cudaError_t configure_ws(int nsm, int grids[3][2][2]) {
        auto k = ccz4_stage_ws_kernel<EPI_RK, C, SEL>;
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, C::NTHR, C::SMEM))) return e;
        // left unavailable (grid 0) when the register split is not covered
        grids[PM_MIXED][EPI_RK][SEL ? 1 : 0] = ws_registers_ok<C, SEL>() ? nsm * (per_sm > 0 ? per_sm : 1) : 0;
        return cudaSuccess;
    }
    static cudaError_t configure(int nsm, int grids[3][2][2]) {
        cudaError_t e;
        if ((e = TmaConfigOps<T>::template configure_one<PM_FP64, EPI_RK, false>(nsm, grids))) return e;
        if ((e = TmaConfigOps<T>::template configure_one<PM_FP64F, EPI_RK, true>(nsm, grids))) return e;
        if ((e = configure_ws<false>(nsm, grids))) return e;
        return configure_ws<true>(nsm, grids);
    }
    static cudaError_t launch(int pm, int epi, bool sel, const DevBlock* blocks, const Tile* tiles, int ntiles,
                              const StageArgs& args, cudaStream_t stream, int grid) {
        if (epi != EPI_RK) return cudaErrorInvalidValue;
        if (pm == PM_FP64 && !sel)
            return TmaConfigOps<T>::template launch_one<PM_FP64, EPI_RK, false>(blocks, tiles, ntiles, args, stream, grid);
        if (pm == PM_FP64F && sel)
            return TmaConfigOps<T>::template launch_one<PM_FP64F, EPI_RK, true>(blocks, tiles, ntiles, args, stream, grid);
        if (pm == PM_MIXED) {
            if (sel)
                ccz4_stage_ws_kernel<EPI_RK, C, true><<<grid, C::NTHR, C::SMEM, stream>>>(blocks, tiles, ntiles, args);
            else
                ccz4_stage_ws_kernel<EPI_RK, C, false><<<grid, C::NTHR, C::SMEM, stream>>>(blocks, tiles, ntiles, args);
            return cudaGetLastError();
        }
        return cudaErrorInvalidValue;
    }
};

}  // namespace granite_b200
