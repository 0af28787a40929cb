// ccz4_constraints.cu -- Hamiltonian / momentum constraint monitor (FP64).
//
// CCZ4Evolution::computeConstraints (ccz4.cpp:941-1159): H = R + 2/3 K^2 -
// A_ij A^ij (vacuum), M_i = gtu^{jk} D_j A_ki - 3/(2 chi) A_ij gtu^{jk} d_k chi
// - 2/3 d_i K. chi is not clamped here (ccz4.cpp:963). The norms of
// main.cpp:1216-1254 are sqrt(sum H^2 / N) over interior points; each CTA
// writes its partial sums, and a single-CTA kernel adds the partials in a
// fixed order, so the result does not depend on scheduling.
#include <mutex>

#include "../../include/granite_ccz4.h"
#include "ccz4_common.cuh"
#include "ccz4_kernels.h"
#include "ccz4_stencil.cuh"

namespace granite_b200 {

namespace {

__device__ void constraint_point(const DevBlock& B, const double* __restrict__ u, long long c, double& H,
                                 double M[3]) {
    using P = double;
    const long long st = B.stride;
    const double* __restrict__ uc = u + c;
#define FP(v) (uc + (long long)(v) * st)
    const double chi = __ldg(FP(CHI));
    const double K = __ldg(FP(KTR));
    double gt[6], At[6], Gh[3], gtu[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        gt[a] = __ldg(FP(GXX + a));
        At[a] = __ldg(FP(AXX + a));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) Gh[a] = __ldg(FP(GHX + a));
    {
        const double det = gt[0] * (gt[3] * gt[5] - gt[4] * gt[4]) - gt[1] * (gt[1] * gt[5] - gt[4] * gt[2]) +
            gt[2] * (gt[1] * gt[4] - gt[3] * gt[2]);
        const double inv = 1.0 / (det + 1.0e-30);
        gtu[0] = (gt[3] * gt[5] - gt[4] * gt[4]) * inv;
        gtu[1] = (gt[2] * gt[4] - gt[1] * gt[5]) * inv;
        gtu[2] = (gt[1] * gt[4] - gt[2] * gt[3]) * inv;
        gtu[3] = (gt[0] * gt[5] - gt[2] * gt[2]) * inv;
        gtu[4] = (gt[1] * gt[2] - gt[0] * gt[4]) * inv;
        gtu[5] = (gt[0] * gt[3] - gt[1] * gt[1]) * inv;
    }
    const double beta0[3] = {0.0, 0.0, 0.0};
    double dg[6][3], Rt[6];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        FieldDer<P> fd = field_der_noko<P, true>(B, FP(GXX + a), beta0, 0.0);
#pragma unroll
        for (int d = 0; d < 3; ++d) dg[a][d] = fd.d[d];
        Rt[a] = -0.5 * (gtu[0] * fd.h[0] + gtu[3] * fd.h[3] + gtu[5] * fd.h[5] +
                        2.0 * (gtu[1] * fd.h[1] + gtu[2] * fd.h[2] + gtu[4] * fd.h[4]));
    }
    double G1[3][6], ch[3][6], Gc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j)
                G1[k][sy(i, j)] = 0.5 * (dg[sy(k, j)][i] + dg[sy(k, i)][j] - dg[sy(i, j)][k]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int jk = 0; jk < 6; ++jk)
            ch[i][jk] = gtu[sy(i, 0)] * G1[0][jk] + gtu[sy(i, 1)] * G1[1][jk] + gtu[sy(i, 2)] * G1[2][jk];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        Gc[k] = gtu[0] * ch[k][0] + gtu[3] * ch[k][3] + gtu[5] * ch[k][5] +
            2.0 * (gtu[1] * ch[k][1] + gtu[2] * ch[k][2] + gtu[4] * ch[k][4]);
    double dGh[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        FieldDer<P> fd = field_der_noko<P, false>(B, FP(GHX + a), beta0, 0.0);
#pragma unroll
        for (int d = 0; d < 3; ++d) dGh[a][d] = fd.d[d];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            double t2 = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) t2 += gt[sy(k, i)] * dGh[k][j] + gt[sy(k, j)] * dGh[k][i];
            Rt[sy(i, j)] += 0.5 * t2 + (Gh[0] - Gc[0]) * G1[0][sy(i, j)] + (Gh[1] - Gc[1]) * G1[1][sy(i, j)] +
                (Gh[2] - Gc[2]) * G1[2][sy(i, j)];
        }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double Gu[3][3];
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
                double t = 0.0;
#pragma unroll
                for (int l = 0; l < 3; ++l) t += ch[k][sy(l, i)] * Gu[j][l] + ch[k][sy(l, j)] * Gu[i][l];
                Rt[sy(i, j)] += t;
            }
    }
    FieldDer<P> fchi = field_der_noko<P, true>(B, FP(CHI), beta0, 0.0);
    const double c_half = 0.5 / (chi + 1e-30), c_quart = 0.25 / ((chi * chi) + 1e-30);
    double DDchi[6];
#pragma unroll
    for (int ij = 0; ij < 6; ++ij)
        DDchi[ij] = fchi.h[ij] - (ch[0][ij] * fchi.d[0] + ch[1][ij] * fchi.d[1] + ch[2][ij] * fchi.d[2]);
    const double lapchi = gtu[0] * DDchi[0] + gtu[3] * DDchi[3] + gtu[5] * DDchi[5] +
        2.0 * (gtu[1] * DDchi[1] + gtu[2] * DDchi[2] + gtu[4] * DDchi[4]);
    double dchi2 = 0.0;
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int m = 0; m < 3; ++m) dchi2 += gtu[sy(l, m)] * fchi.d[l] * fchi.d[m];
    double Rs = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int ij = sy(i, j);
            const double rchi = c_half * (DDchi[ij] + gt[ij] * lapchi) -
                c_quart * (fchi.d[i] * fchi.d[j] - 3.0 * gt[ij] * dchi2);
            Rs += gtu[ij] * (Rt[ij] + rchi);
        }
    Rs *= chi;
    double Am[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Am[i][j] = gtu[sy(i, 0)] * At[sy(0, j)] + gtu[sy(i, 1)] * At[sy(1, j)] + gtu[sy(i, 2)] * At[sy(2, j)];
    double AtAt = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) AtAt += Am[i][j] * Am[j][i];
    H = Rs + (2.0 / 3.0) * K * K - AtAt;  // ccz4.cpp:1127 with rho = 0

    // momentum constraint, ccz4.cpp:1138-1155
    double dA[6][3], dK[3];
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        FieldDer<P> fd = field_der_noko<P, false>(B, FP(AXX + a), beta0, 0.0);
#pragma unroll
        for (int d = 0; d < 3; ++d) dA[a][d] = fd.d[d];
    }
    {
        FieldDer<P> fd = field_der_noko<P, false>(B, FP(KTR), beta0, 0.0);
#pragma unroll
        for (int d = 0; d < 3; ++d) dK[d] = fd.d[d];
    }
    const double c3 = 3.0 / (2.0 * chi + 1e-30);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double Mi = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double g_jk = gtu[sy(j, k)];
                double DA = dA[sy(k, i)][j];
#pragma unroll
                for (int m = 0; m < 3; ++m) DA -= ch[m][sy(j, k)] * At[sy(m, i)] + ch[m][sy(j, i)] * At[sy(k, m)];
                Mi += g_jk * DA - c3 * At[sy(i, j)] * g_jk * fchi.d[k];
            }
        M[i] = Mi - (2.0 / 3.0) * dK[i];
    }
#undef FP
}

constexpr int CT_X = 32, CT_Y = 4;

__global__ void __launch_bounds__(CT_X* CT_Y)
    constraints_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int sel,
                       double* __restrict__ ham, double* __restrict__ mom, double* __restrict__ partials) {
    const Tile t = tiles[blockIdx.x];
    const DevBlock& B = blocks[t.block];
    const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y, k = t.k0 + threadIdx.z;
    double h2 = 0.0, m2 = 0.0;
    if (i < B.n[0] && j < B.n[1] && k < B.n[2]) {
        const long long c = cell_index(B, i + NG, j + NG, k + NG);
        double H, M[3];
        constraint_point(B, B.buf[sel], c, H, M);
        if (ham) ham[c] = H;
        if (mom) {
            mom[3 * c] = M[0];
            mom[3 * c + 1] = M[1];
            mom[3 * c + 2] = M[2];
        }
        h2 = H * H;
        m2 = M[0] * M[0] + M[1] * M[1] + M[2] * M[2];
    }
    if (!partials) return;
    // fixed-shape CTA reduction (warp shuffles, then smem across warps)
    for (int o = 16; o > 0; o >>= 1) {
        h2 += __shfl_down_sync(0xffffffffu, h2, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
    }
    __shared__ double sh[2][CT_X * CT_Y / 32];
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    if (lane == 0) {
        sh[0][warp] = h2;
        sh[1][warp] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < CT_X * CT_Y / 32; ++w) {
            a += sh[0][w];
            b += sh[1][w];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// One CTA; thread t sums partials t, t+T, ... in order, then a fixed tree.
__global__ void sum_partials_kernel(const double* __restrict__ p, int n, double* out) {
    __shared__ double sa[256], sb[256];
    double a = 0.0, b = 0.0;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        a += p[2 * x];
        b += p[2 * x + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sa[0];
        out[1] = sb[0];
    }
}

}  // namespace

cudaError_t launch_constraints(const DevBlock* blocks, const Tile* tiles, int ntiles, int sel, double* ham,
                               double* mom, double* partials, cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    constraints_kernel<<<ntiles, dim3(CT_X, CT_Y, 1), 0, stream>>>(blocks, tiles, sel, ham, mom, partials);
    return cudaGetLastError();
}

cudaError_t launch_sum_partials(const double* partials, int n, double* out, cudaStream_t stream) {
    sum_partials_kernel<<<1, 256, 0, stream>>>(partials, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Regrid taggers (amr.cpp:653-731): a cell is tagged when |grad f| / (|f| + 1e-30)
// exceeds the threshold, grad f from centred differences (f[+1] - f[-1]) / (2 dx)
// summed as squares over x, y, z, in the reference's order with separately
// rounded operations (so the decision at the threshold is the reference's).
// ---------------------------------------------------------------------------
namespace {

__global__ void __launch_bounds__(CT_X* CT_Y)
    tag_count_kernel(const DevBlock* __restrict__ blocks, const Tile* __restrict__ tiles, int var, double threshold,
                     unsigned long long* count) {
    const Tile t = tiles[blockIdx.x];
    const DevBlock& B = blocks[t.block];
    const int w = t.w > 0 ? t.w : CT_X;
    const int tid = threadIdx.x + CT_X * threadIdx.y;
    const int i = t.i0 + tid % w, j = t.j0 + tid / w, k = t.k0;
    bool tag = false;
    if (i < B.n[0] && j < B.n[1] && k < B.n[2]) {
        const double* f = B.buf[0] + (long long)var * B.stride + cell_index(B, i + NG, j + NG, k + NG);
        const long long off[3] = {1, B.tx, (long long)B.tx * B.ty};
        double grad2 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double df = __ddiv_rn(__dsub_rn(__ldg(f + off[d]), __ldg(f - off[d])), __dmul_rn(2.0, B.dx[d]));
            grad2 = __dadd_rn(grad2, __dmul_rn(df, df));
        }
        tag = __ddiv_rn(__dsqrt_rn(grad2), __dadd_rn(fabs(__ldg(f)), 1e-30)) > threshold;
    }
    const unsigned n = __popc(__ballot_sync(0xffffffffu, tag));
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(count, (unsigned long long)n);
}

}  // namespace

cudaError_t launch_tag_count(const DevBlock* blocks, const Tile* tiles, int ntiles, int var, double threshold,
                             unsigned long long* count, cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    tag_count_kernel<<<ntiles, dim3(CT_X, CT_Y, 1), 0, stream>>>(blocks, tiles, var, threshold, count);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Constraint norms without any allocation (granite_ccz4_constraint_norms_noalloc)
//
// For callers that cannot allocate device memory themselves (see the header):
// the per-tile partial sums live in a fixed file-scope device array instead of
// context-owned scratch, the block descriptor travels as a kernel argument,
// and the tiles are derived from the grid instead of a device-side work-list.
// ---------------------------------------------------------------------------

// Capacity: one (sum H^2, sum |M|^2) pair per 32x4x1 tile of interior points.
constexpr int NOALLOC_MAX_TILES = 65536;  // 1 MiB; up to 8,388,608 interior points per call
static __device__ __align__(256) double g_noalloc_partials[2 * NOALLOC_MAX_TILES];

namespace {

__global__ void __launch_bounds__(CT_X* CT_Y)
    constraints_noalloc_kernel(DevBlock B, const double* __restrict__ u, int ntx, int nty, double* partials) {
    // tile index -> (i0, j0, k0) in the same order as the host work-lists (x fastest)
    const int t = blockIdx.x;
    const int i0 = (t % ntx) * CT_X, j0 = ((t / ntx) % nty) * CT_Y, k0 = t / (ntx * nty);
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y, k = k0;
    double h2 = 0.0, m2 = 0.0;
    if (i < B.n[0] && j < B.n[1] && k < B.n[2]) {
        const long long c = cell_index(B, i + NG, j + NG, k + NG);
        double H, M[3];
        constraint_point(B, u, c, H, M);
        h2 = H * H;
        m2 = M[0] * M[0] + M[1] * M[1] + M[2] * M[2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        h2 += __shfl_down_sync(0xffffffffu, h2, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
    }
    __shared__ double sh[2][CT_X * CT_Y / 32];
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    if (lane == 0) {
        sh[0][warp] = h2;
        sh[1][warp] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < CT_X * CT_Y / 32; ++w) {
            a += sh[0][w];
            b += sh[1][w];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// Fixed-order sum of the partials (same tree as sum_partials_kernel), then the
// RMS norms of main.cpp:1216-1254: norms[0] = sqrt(sum H^2 / N), norms[1] = sqrt(sum |M|^2 / N).
__global__ void noalloc_norms_kernel(const double* __restrict__ p, int n, double npts, double* norms) {
    __shared__ double sa[256], sb[256];
    double a = 0.0, b = 0.0;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        a += p[2 * x];
        b += p[2 * x + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sa[threadIdx.x] += sa[threadIdx.x + s];
            sb[threadIdx.x] += sb[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        norms[0] = sqrt(sa[0] / npts);
        norms[1] = sqrt(sb[0] / npts);
    }
}

constexpr int NOALLOC_MAX_DEVICES = 64;
// Device address of g_noalloc_partials per device, and the context it was looked
// up in: a device reset (or anything else that recreates the primary context)
// can load the module at a new address, so a changed context means a new lookup.
double* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
void* g_noalloc_ctx[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mutex;

// The current driver context (CUcontext as an opaque pointer), through the
// runtime's driver entry point (no link against libcuda); null if unavailable.
void* current_driver_context() {
    using GetCurrent = int (*)(void**);
    static GetCurrent fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<GetCurrent>(f);
    });
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

}  // namespace

// ---------------------------------------------------------------------------
// State comparison of two block lists of identical geometry (diagnostics):
// per field, the largest |a - b| and |a| over the interior cells of slot 0 of
// every block, as the bits of non-negative doubles (atomicMax on the bit
// patterns orders them as values), and the counts of non-finite values in a
// and in b (out[44], out[45]). NaN differences do not enter the maxima.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(256)
    compare_states_kernel(const DevBlock* __restrict__ A, const DevBlock* __restrict__ Bl, unsigned long long* out) {
    const DevBlock& a = A[blockIdx.y];
    const DevBlock& b = Bl[blockIdx.y];
    const long long n = (long long)a.n[0] * a.n[1] * a.n[2];
    double dev[NV], mag[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) dev[v] = mag[v] = 0.0;
    unsigned long long bad_a = 0, bad_b = 0;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % a.n[0]), j = (int)((p / a.n[0]) % a.n[1]), k = (int)(p / ((long long)a.n[0] * a.n[1]));
        const long long c = cell_index(a, i + NG, j + NG, k + NG);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double x = __ldg(a.buf[0] + (long long)v * a.stride + c);
            const double y = __ldg(b.buf[0] + (long long)v * b.stride + c);
            bad_a += !isfinite(x);
            bad_b += !isfinite(y);
            dev[v] = fmax(dev[v], fabs(x - y));
            mag[v] = fmax(mag[v], fabs(x));
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        for (int o = 16; o > 0; o >>= 1) {
            dev[v] = fmax(dev[v], __shfl_down_sync(0xffffffffu, dev[v], o));
            mag[v] = fmax(mag[v], __shfl_down_sync(0xffffffffu, mag[v], o));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        bad_a += __shfl_down_sync(0xffffffffu, bad_a, o);
        bad_b += __shfl_down_sync(0xffffffffu, bad_b, o);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            atomic_max_nonneg(out + v, dev[v]);
            atomic_max_nonneg(out + NV + v, mag[v]);
        }
        if (bad_a) atomicAdd(out + 2 * NV, bad_a);
        if (bad_b) atomicAdd(out + 2 * NV + 1, bad_b);
    }
}

}  // namespace

cudaError_t launch_compare_states(const DevBlock* a, const DevBlock* b, int nblocks, unsigned long long* out,
                                  cudaStream_t stream) {
    if (nblocks <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(out, 0, (2 * NV + 2) * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    compare_states_kernel<<<dim3(32, nblocks), 256, 0, stream>>>(a, b, out);
    return cudaGetLastError();
}

}  // namespace granite_b200

extern "C" GRANITE_API int granite_ccz4_constraint_norms_noalloc(const granite_block_desc* b, const double* u_dev,
                                                                  double* norms_dev, void* stream) {
    using namespace granite_b200;
    if (!b || !u_dev || !norms_dev) return GRANITE_ERR_INVALID;
    if (b->nghost != NG) return GRANITE_ERR_INVALID;
    for (int d = 0; d < 3; ++d)
        if (b->ncells[d] < NG || !(b->hi[d] > b->lo[d])) return GRANITE_ERR_INVALID;
    const int ntx = (b->ncells[0] + CT_X - 1) / CT_X, nty = (b->ncells[1] + CT_Y - 1) / CT_Y;
    const long long ntiles = (long long)ntx * nty * b->ncells[2];
    if (ntiles > NOALLOC_MAX_TILES) return GRANITE_ERR_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return GRANITE_ERR_NO_DEVICE;
    double* partials = nullptr;
    {
        // once per device (and again if its context was recreated), with that
        // device current: host code must not use the array's name as a device address
        const void* ctx = current_driver_context();
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_addr[dev] || g_noalloc_ctx[dev] != ctx) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return GRANITE_ERR_CUDA;
            g_noalloc_addr[dev] = static_cast<double*>(p);
            g_noalloc_ctx[dev] = const_cast<void*>(ctx);
        }
        partials = g_noalloc_addr[dev];
    }
    DevBlock B{};
    for (int d = 0; d < 3; ++d) B.n[d] = b->ncells[d];
    B.tx = b->ncells[0] + 2 * NG;
    B.ty = b->ncells[1] + 2 * NG;
    B.tz = b->ncells[2] + 2 * NG;
    B.stride = (long long)B.tx * B.ty * B.tz;
    for (int d = 0; d < 3; ++d) {
        B.lo[d] = b->lo[d];
        B.dx[d] = (b->hi[d] - b->lo[d]) / static_cast<double>(b->ncells[d]);  // grid.cpp:20-22
        B.inv12h[d] = 1.0 / (12.0 * B.dx[d]);
        B.inv12h2[d] = 1.0 / (12.0 * B.dx[d] * B.dx[d]);
    }
    B.inv4hh[0] = 1.0 / (4.0 * B.dx[0] * B.dx[1]);
    B.inv4hh[1] = 1.0 / (4.0 * B.dx[0] * B.dx[2]);
    B.inv4hh[2] = 1.0 / (4.0 * B.dx[1] * B.dx[2]);
    B.level = b->level;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // cudaLaunchKernel returns the status of each launch itself, so the result
    // reflects this call only (an error left by the caller's earlier work is
    // neither reported here nor cleared)
    {
        void* args[] = {&B, const_cast<double**>(&u_dev), const_cast<int*>(&ntx), const_cast<int*>(&nty),
                        &partials};
        if (cudaLaunchKernel(reinterpret_cast<const void*>(constraints_noalloc_kernel), dim3((unsigned)ntiles),
                             dim3(CT_X, CT_Y, 1), args, 0, s) != cudaSuccess)
            return GRANITE_ERR_CUDA;
    }
    double npts = (double)b->ncells[0] * b->ncells[1] * b->ncells[2];
    int n = (int)ntiles;
    void* args[] = {&partials, &n, &npts, &norms_dev};
    if (cudaLaunchKernel(reinterpret_cast<const void*>(noalloc_norms_kernel), dim3(1), dim3(256), args, 0, s) !=
        cudaSuccess)
        return GRANITE_ERR_CUDA;
    return GRANITE_OK;
}
