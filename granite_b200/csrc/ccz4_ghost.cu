// ccz4_ghost.cu -- ghost-cell fills and inter-block transfers.
//
// All arithmetic here uses explicitly rounded intrinsics (no FMA contraction)
// so the fills reproduce the reference host loops bit for bit:
//   zero-gradient level fill   amr.cpp:447-480 (all faces, or the faces the
//                              reference leaves uncovered by a parent block)
//   1/r outer falloff          main.cpp:351-463 (x faces, then y, then z)
//   trilinear prolongation     amr.cpp:484-564
//   2x2x2 restriction          amr.cpp:566-626
// The work is described by host-built lists (ghost-cell chunks, transfer
// boxes cut into chunks), so one launch serves every block of a level
// whatever its size.
#include "ccz4_common.cuh"
#include "ccz4_kernels.h"

namespace granite_b200 {

namespace {

__device__ __forceinline__ int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }

__device__ __forceinline__ double sq3(double a, double b, double c) {
    // sqrt(a*a + b*b + c*c) + 1e-30, left-to-right, no contraction
    return __dadd_rn(__dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c))), 1e-30);
}

// finf + (f_int - finf) * r_int / r_gh
__device__ __forceinline__ double falloff(double finf, double fint, double ri, double rg) {
    return __dadd_rn(finf, __ddiv_rn(__dmul_rn(__dsub_rn(fint, finf), ri), rg));
}

__device__ __forceinline__ bool inside(int a, int n) { return a >= NG && a < NG + n; }

// Value the reference's three 1/r passes leave in a ghost cell, with the
// radii shared by all 22 fields: the passes a ghost
// cell goes through (x, then y, then z, each only if that coordinate is a
// ghost) read a chain of cells whose end is an interior cell; every pass is
// finf + (f - finf) * r_in / r_out with its own pair of radii.
struct FalloffChain {
    int npass;
    long long src;     // interior cell at the end of the chain
    double ri[3], rg[3];
};

__device__ FalloffChain falloff_chain(const DevBlock& B, int i, int j, int k) {
    FalloffChain ch;
    ch.npass = 0;
    const bool gx = !inside(i, B.n[0]), gy = !inside(j, B.n[1]), gz = !inside(k, B.n[2]);
    const int ic = clampi(i, NG, NG + B.n[0] - 1), jc = clampi(j, NG, NG + B.n[1] - 1),
              kc = clampi(k, NG, NG + B.n[2] - 1);
    ch.src = cell_index(B, ic, jc, kc);
    // coordinates seen by each pass (main.cpp:395-463)
    const double xi = coord(B, 0, ic), xg = coord(B, 0, i);
    const double yi = coord(B, 1, jc), yg = coord(B, 1, j);
    const double zi = coord(B, 2, kc), zg = coord(B, 2, k);
    const double yx = gy ? yi : yg, zx = gz ? zi : zg;  // the x pass runs at (i, jc or j, kc or k)
    if (gx) {
        ch.ri[ch.npass] = sq3(xi, yx, zx);
        ch.rg[ch.npass] = sq3(xg, yx, zx);
        ++ch.npass;
    }
    if (gy) {  // the y pass runs at (i, j, kc or k)
        ch.ri[ch.npass] = sq3(xg, yi, zx);
        ch.rg[ch.npass] = sq3(xg, yg, zx);
        ++ch.npass;
    }
    if (gz) {
        ch.ri[ch.npass] = sq3(xg, yg, zi);
        ch.rg[ch.npass] = sq3(xg, yg, zg);
        ++ch.npass;
    }
    return ch;
}

// r-th ghost cell of a block: z slabs first, then y slabs, then x slabs.
__device__ __forceinline__ bool ghost_coords(const DevBlock& B, long long r, int& i, int& j, int& k) {
    const int T0 = B.tx, T1 = B.ty;
    const int n0 = B.n[0], n1 = B.n[1], n2 = B.n[2];
    const long long A = (long long)T0 * T1 * (2 * NG);
    if (r < A) {
        const int kk = (int)(r / ((long long)T0 * T1));
        const long long rem = r % ((long long)T0 * T1);
        k = kk < NG ? kk : kk + n2;
        j = (int)(rem / T0);
        i = (int)(rem % T0);
        return true;
    }
    r -= A;
    const long long Bc = (long long)T0 * (2 * NG) * n2;
    if (r < Bc) {
        k = NG + (int)(r / ((long long)T0 * 2 * NG));
        const long long rem = r % ((long long)T0 * 2 * NG);
        const int jj = (int)(rem / T0);
        j = jj < NG ? jj : jj + n1;
        i = (int)(rem % T0);
        return true;
    }
    r -= Bc;
    const long long Cc = (long long)(2 * NG) * n1 * n2;
    if (r < Cc) {
        k = NG + (int)(r / ((long long)2 * NG * n1));
        const long long rem = r % ((long long)2 * NG * n1);
        j = NG + (int)(rem / (2 * NG));
        const int ii = (int)(rem % (2 * NG));
        i = ii < NG ? ii : ii + n0;
        return true;
    }
    return false;
}

// Zero-gradient with a face mask: the reference's x, y, z passes over the
// flagged faces only. Copies are exact, so the result is the cell reached by
// clamping each coordinate that lies beyond a flagged face (amr.cpp:447-480).
__device__ __forceinline__ int masked_clamp(int a, int n, unsigned mask, int axis) {
    if (a < NG) return (mask >> (2 * axis)) & 1u ? NG : a;
    if (a >= NG + n) return (mask >> (2 * axis + 1)) & 1u ? NG + n - 1 : a;
    return a;
}

// items[x].cell holds the first ghost rank of a chunk of blockDim.x ranks.
__global__ void ghost_fill_kernel(int mode, const DevBlock* __restrict__ blocks, const GhostItem* __restrict__ items,
                                  int sel, const unsigned char* __restrict__ facemask) {
    const GhostItem it = items[blockIdx.x];
    const DevBlock& B = blocks[it.block];
    int i, j, k;
    if (!ghost_coords(B, (long long)it.cell + threadIdx.x, i, j, k)) return;
    double* base = B.buf[sel];
    const long long c = cell_index(B, i, j, k);
    if (mode == GHOST_SOMMERFELD) {
        const FalloffChain ch = falloff_chain(B, i, j, k);
        for (int v = 0; v < NV; ++v) {
            const double fi = f_inf(v);
            double val = base[(long long)v * B.stride + ch.src];
#pragma unroll
            for (int p = 0; p < 3; ++p)  // unrolled with a guard: the radii stay in registers
                if (p < ch.npass) val = falloff(fi, val, ch.ri[p], ch.rg[p]);
            base[(long long)v * B.stride + c] = val;
        }
        return;
    }
    int si, sj, sk;
    if (mode == GHOST_ZERO_GRADIENT) {
        si = clampi(i, NG, NG + B.n[0] - 1);
        sj = clampi(j, NG, NG + B.n[1] - 1);
        sk = clampi(k, NG, NG + B.n[2] - 1);
    } else if (mode == GHOST_ZERO_GRADIENT_MASKED) {
        const unsigned m = facemask[it.block];
        si = masked_clamp(i, B.n[0], m, 0);
        sj = masked_clamp(j, B.n[1], m, 1);
        sk = masked_clamp(k, B.n[2], m, 2);
        if (si == i && sj == j && sk == k) return;
    } else {  // periodic
        si = i < NG ? i + B.n[0] : (i >= NG + B.n[0] ? i - B.n[0] : i);
        sj = j < NG ? j + B.n[1] : (j >= NG + B.n[1] ? j - B.n[1] : j);
        sk = k < NG ? k + B.n[2] : (k >= NG + B.n[2] ? k - B.n[2] : k);
    }
    const long long s = cell_index(B, si, sj, sk);
    for (int v = 0; v < NV; ++v) base[(long long)v * B.stride + c] = base[(long long)v * B.stride + s];
}

// Trilinear prolongation of coarse block C into fine cell (i,j,k) of F,
// amr.cpp:496-561: nearest coarse centre by rounding, one-sided neighbour by
// the sign of the fractional offset, indices clamped to the coarse block.
__device__ void prolong_cell(const DevBlock& F, const DevBlock& C, int i, int j, int k, double* __restrict__ fb,
                             const double* __restrict__ cb) {
    const int fi[3] = {i, j, k};
    const int ct[3] = {C.tx, C.ty, C.tz};
    int c0[3], c1[3];
    double ax[3];
    for (int d = 0; d < 3; ++d) {
        const double f = __dadd_rn(__ddiv_rn(__dsub_rn(coord(F, d, fi[d]), coord(C, d, NG)), C.dx[d]), (double)NG);
        int a = (int)round(f);
        a = a > ct[d] - 1 ? ct[d] - 1 : a;
        a = a < 0 ? 0 : a;
        const double fr = __dsub_rn(f, (double)a);
        int b = a + (fr >= 0.0 ? 1 : -1);
        b = b > ct[d] - 1 ? ct[d] - 1 : b;
        b = b < 0 ? 0 : b;
        c0[d] = a;
        c1[d] = b;
        ax[d] = fabs(fr);
    }
    const double bx = __dsub_rn(1.0, ax[0]), by = __dsub_rn(1.0, ax[1]), bz = __dsub_rn(1.0, ax[2]);
    const double w000 = __dmul_rn(__dmul_rn(bx, by), bz);
    const double w100 = __dmul_rn(__dmul_rn(ax[0], by), bz);
    const double w010 = __dmul_rn(__dmul_rn(bx, ax[1]), bz);
    const double w001 = __dmul_rn(__dmul_rn(bx, by), ax[2]);
    const double w110 = __dmul_rn(__dmul_rn(ax[0], ax[1]), bz);
    const double w101 = __dmul_rn(__dmul_rn(ax[0], by), ax[2]);
    const double w011 = __dmul_rn(__dmul_rn(bx, ax[1]), ax[2]);
    const double w111 = __dmul_rn(__dmul_rn(ax[0], ax[1]), ax[2]);
    const int o000 = (int)cell_index(C, c0[0], c0[1], c0[2]), o100 = (int)cell_index(C, c1[0], c0[1], c0[2]);
    const int o010 = (int)cell_index(C, c0[0], c1[1], c0[2]), o001 = (int)cell_index(C, c0[0], c0[1], c1[2]);
    const int o110 = (int)cell_index(C, c1[0], c1[1], c0[2]), o101 = (int)cell_index(C, c1[0], c0[1], c1[2]);
    const int o011 = (int)cell_index(C, c0[0], c1[1], c1[2]), o111 = (int)cell_index(C, c1[0], c1[1], c1[2]);
    const long long fc = cell_index(F, i, j, k);
#pragma unroll 2
    for (int v = 0; v < NV; ++v) {
        const double* q = cb + (long long)v * C.stride;
        double val = __dmul_rn(w000, __ldg(q + o000));
        val = __dadd_rn(val, __dmul_rn(w100, __ldg(q + o100)));
        val = __dadd_rn(val, __dmul_rn(w010, __ldg(q + o010)));
        val = __dadd_rn(val, __dmul_rn(w001, __ldg(q + o001)));
        val = __dadd_rn(val, __dmul_rn(w110, __ldg(q + o110)));
        val = __dadd_rn(val, __dmul_rn(w101, __ldg(q + o101)));
        val = __dadd_rn(val, __dmul_rn(w011, __ldg(q + o011)));
        val = __dadd_rn(val, __dmul_rn(w111, __ldg(q + o111)));
        fb[(long long)v * F.stride + fc] = val;
    }
}

__global__ void xfer_kernel(int kind, const DevBlock* __restrict__ blocks, const XferBox* __restrict__ boxes,
                            const BoxChunk* __restrict__ chunks, int dst_sel, int src_sel) {
    const BoxChunk ch = chunks[blockIdx.x];
    const XferBox bx = boxes[ch.box];
    const int r = ch.start + threadIdx.x;
    if (r >= bx.n[0] * bx.n[1] * bx.n[2]) return;
    const int a = r % bx.n[0], b = (r / bx.n[0]) % bx.n[1], c = r / (bx.n[0] * bx.n[1]);
    const DevBlock& D = blocks[bx.dst];
    const DevBlock& S = blocks[bx.src];
    const int i = bx.d0[0] + a, j = bx.d0[1] + b, k = bx.d0[2] + c;
    double* db = D.buf[dst_sel];
    const double* sb = S.buf[src_sel];
    if (kind == XFER_PROLONG) {
        prolong_cell(D, S, i, j, k, db, sb);
        return;
    }
    const long long dc = cell_index(D, i, j, k);
    if (kind == XFER_COPY) {
        const long long sc = cell_index(S, bx.s0[0] + a, bx.s0[1] + b, bx.s0[2] + c);
        for (int v = 0; v < NV; ++v) db[(long long)v * D.stride + dc] = __ldg(sb + (long long)v * S.stride + sc);
        return;
    }
    // restriction: mean of the 2x2x2 fine cells, summed rk, rj, ri (amr.cpp:601-609)
    const long long f0 = cell_index(S, bx.s0[0] + 2 * a, bx.s0[1] + 2 * b, bx.s0[2] + 2 * c);
    const long long sx = 1, sy = S.tx, sz = (long long)S.tx * S.ty;
    for (int v = 0; v < NV; ++v) {
        const double* q = sb + (long long)v * S.stride + f0;
        double s = 0.0;
        for (int rk = 0; rk < 2; ++rk)
            for (int rj = 0; rj < 2; ++rj)
                for (int ri = 0; ri < 2; ++ri) s = __dadd_rn(s, __ldg(q + ri * sx + rj * sy + rk * sz));
        db[(long long)v * D.stride + dc] = __ddiv_rn(s, 8.0);
    }
}

// One thread per listed ghost cell; each cell is written exactly once. The
// cells a launch reads (interior cells of this level, coarse slot 0) are never
// written by it, so every value of a cell is loaded before any is stored.
// 4 CTAs of 256 threads per SM (64 registers): the fields of a cell are moved in
// two halves and the prolongation keeps 32-bit offsets, so the paths fit without
// the 127 registers (16 warps per SM) of a one-pass version; about 5 % faster on
// the hierarchy's fills.
__global__ void __launch_bounds__(256, 4) ghost_sources_kernel(const DevBlock* __restrict__ blocks, const GhostSrc* __restrict__ items,
                                     long long n, int sel, int local_mode) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const GhostSrc it = items[t];
    const DevBlock& D = blocks[it.dst_block];
    double* db = D.buf[sel];
    const long long dst = it.dst_cell, dstr = D.stride;
    const int i = it.dst_cell % D.tx, j = (it.dst_cell / D.tx) % D.ty, k = it.dst_cell / (D.tx * D.ty);
    if (it.src_block >= 0 && it.src_cell < 0) {  // coarse level
        const DevBlock& C = blocks[it.src_block];
        prolong_cell(D, C, i, j, k, db, C.buf[0]);
        return;
    }
    const double* src;
    long long sstr;
    if (it.src_block >= 0) {  // same-level neighbour
        const DevBlock& S = blocks[it.src_block];
        src = S.buf[sel] + it.src_cell;
        sstr = S.stride;
    } else if (local_mode == GHOST_SOMMERFELD) {
        const FalloffChain ch = falloff_chain(D, i, j, k);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double v_[NV / 2];
#pragma unroll
            for (int v = 0; v < NV / 2; ++v) v_[v] = __ldg(db + (h * (NV / 2) + v) * dstr + ch.src);
#pragma unroll
            for (int v = 0; v < NV / 2; ++v) {
                const double fi = f_inf(h * (NV / 2) + v);
                double val = v_[v];
    #pragma unroll
            for (int p = 0; p < 3; ++p)  // unrolled with a guard: the radii stay in registers
                if (p < ch.npass) val = falloff(fi, val, ch.ri[p], ch.rg[p]);
                db[(h * (NV / 2) + v) * dstr + dst] = val;
            }
        }
        return;
    } else {  // zero gradient
        src = db + cell_index(D, clampi(i, NG, NG + D.n[0] - 1), clampi(j, NG, NG + D.n[1] - 1),
                              clampi(k, NG, NG + D.n[2] - 1));
        sstr = dstr;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        double v_[NV / 2];
#pragma unroll
        for (int v = 0; v < NV / 2; ++v) v_[v] = __ldg(src + (h * (NV / 2) + v) * sstr);
#pragma unroll
        for (int v = 0; v < NV / 2; ++v) db[(h * (NV / 2) + v) * dstr + dst] = v_[v];
    }
}

}  // namespace

cudaError_t launch_ghost_sources(const DevBlock* blocks, const GhostSrc* items, long long nitems, int sel,
                                 int local_mode, cudaStream_t stream) {
    if (nitems <= 0) return cudaSuccess;
    ghost_sources_kernel<<<(unsigned)((nitems + 255) / 256), 256, 0, stream>>>(blocks, items, nitems, sel,
                                                                            local_mode);
    return cudaGetLastError();
}

constexpr int GHOST_CHUNK = 256;

cudaError_t launch_ghost_fill(int mode, const DevBlock* blocks, const GhostItem* items, int nitems, int sel,
                              const unsigned char* facemask, cudaStream_t stream) {
    if (nitems <= 0) return cudaSuccess;
    ghost_fill_kernel<<<nitems, GHOST_CHUNK, 0, stream>>>(mode, blocks, items, sel, facemask);
    return cudaGetLastError();
}

cudaError_t launch_xfer(int kind, const DevBlock* blocks, const XferBox* boxes, const BoxChunk* chunks, int nchunks,
                        int dst_sel, int src_sel, cudaStream_t stream) {
    if (nchunks <= 0) return cudaSuccess;
    xfer_kernel<<<nchunks, XFER_CHUNK, 0, stream>>>(kind, blocks, boxes, chunks, dst_sel, src_sel);
    return cudaGetLastError();
}

}  // namespace granite_b200
