// ccz4_matter.cu -- the ADM matter sources of the CCZ4 RHS from GRMHD primitives.
//
// GRMHDEvolution::computeMatterSources (grmhd.cpp:1034-1103): per interior
// cell of a magnetised perfect fluid (PrimitiveVar order rho, v^x, v^y, v^z,
// p, B^x, B^y, B^z, eps, T, Ye; types.hpp:149-162)
//   h = 1 + eps + p / (rho + 1e-30)                     (grmhd.hpp:55)
//   W = 1 / sqrt(max(1 - v^2, 1e-10)),  b^2 = B^2 / W^2 + (B.v)^2
//   b_i = B_i / W^2 + (B.v) v_i
//   rho_ADM = rho h W^2 - p + b^2 / 2
//   S_i  = (rho h W^2 + b^2) v_i - (B.v) b_i
//   S_ij = (rho h W^2 + b^2) v_i v_j + (p + b^2/2) delta_ij - b_i b_j - B_i B_j / W^2
//   S    = S_xx + S_yy + S_zz
// Every operation is a separately rounded FP64 intrinsic in the reference's
// evaluation order (no contraction), so the sources equal the reference's bit
// for bit. Pointwise and HBM-bound: 72 B read, 88 B written per cell.
#include "ccz4_kernels.h"

namespace granite_b200 {
namespace {

// std::max(a, b) as the reference calls it: b when a < b, else a (a NaN stays).
__device__ __forceinline__ double std_max(double a, double b) { return a < b ? b : a; }

__global__ void __launch_bounds__(128)
    matter_sources_kernel(const DevBlock B, const double* __restrict__ prim, const MatterOut o) {
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y, k = blockIdx.z;
    if (i >= B.n[0] || j >= B.n[1]) return;
    const long long c = cell_index(B, i + NG, j + NG, k + NG), s = B.stride;
    const double rho = __ldg(prim + c), vx = __ldg(prim + s + c), vy = __ldg(prim + 2 * s + c),
                 vz = __ldg(prim + 3 * s + c), p = __ldg(prim + 4 * s + c);
    const double Bx = __ldg(prim + 5 * s + c), By = __ldg(prim + 6 * s + c), Bz = __ldg(prim + 7 * s + c);
    const double eps = __ldg(prim + 8 * s + c);

    const double h = __dadd_rn(__dadd_rn(1.0, eps), __ddiv_rn(p, __dadd_rn(rho, 1e-30)));
    const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy)), __dmul_rn(vz, vz));
    const double W = __ddiv_rn(1.0, __dsqrt_rn(std_max(__dsub_rn(1.0, v2), 1.0e-10)));
    const double W2 = __dmul_rn(W, W);
    const double Bv = __dadd_rn(__dadd_rn(__dmul_rn(Bx, vx), __dmul_rn(By, vy)), __dmul_rn(Bz, vz));
    const double B2 = __dadd_rn(__dadd_rn(__dmul_rn(Bx, Bx), __dmul_rn(By, By)), __dmul_rn(Bz, Bz));
    const double b2 = __dadd_rn(__ddiv_rn(B2, W2), __dmul_rn(Bv, Bv));
    const double rhoHW2 = __dmul_rn(__dmul_rn(rho, h), W2);
    const double e = __dadd_rn(rhoHW2, b2);
    const double ph = __dadd_rn(p, __dmul_rn(0.5, b2));
    o.rho[c] = __dadd_rn(__dsub_rn(rhoHW2, p), __dmul_rn(0.5, b2));

    const double vel[3] = {vx, vy, vz};
    const double Bco[3] = {Bx, By, Bz};
    double bco[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        bco[a] = __dadd_rn(__ddiv_rn(Bco[a], W2), __dmul_rn(Bv, vel[a]));
        o.Si[c * o.si_cell + a * o.si_comp] = __dsub_rn(__dmul_rn(e, vel[a]), __dmul_rn(Bv, bco[a]));
    }
    double tr = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b) {
            const double delta = a == b ? 1.0 : 0.0;
            const int q = a == 0 ? b : (a == 1 ? 2 + b : 5);  // symIdx (types.hpp:52-54)
            double v = __dadd_rn(__dmul_rn(__dmul_rn(e, vel[a]), vel[b]), __dmul_rn(ph, delta));
            v = __dsub_rn(v, __dmul_rn(bco[a], bco[b]));
            v = __dsub_rn(v, __ddiv_rn(__dmul_rn(Bco[a], Bco[b]), W2));
            o.Sij[c * o.sij_cell + q * o.sij_comp] = v;
            if (a == b) tr = __dadd_rn(tr, v);
        }
    o.S[c] = tr;
}

}  // namespace

cudaError_t launch_matter_sources(const DevBlock& B, const double* prim, const MatterOut& out, cudaStream_t stream) {
    if (B.n[0] <= 0 || B.n[1] <= 0 || B.n[2] <= 0) return cudaSuccess;
    const dim3 grid((B.n[0] + 31) / 32, (B.n[1] + 3) / 4, B.n[2]);
    matter_sources_kernel<<<grid, dim3(32, 4, 1), 0, stream>>>(B, prim, out);
    return cudaGetLastError();
}

}  // namespace granite_b200
