// ccz4_psi4.cu -- gravitational-wave extraction on coordinate spheres.
//
// Psi4Extractor::extract (postprocess.cpp:245-314) on one device-resident
// block: for every extraction radius r and sphere point (theta_i = (i + 1/2)
// pi / n_theta, phi_j = 2 pi j / n_phi) inside the block (one cell in from its
// faces), Psi4 ~ -(A~_ij / chi) mbar^i mbar^j from trilinearly interpolated
// chi and A~_ij with mbar = (theta-hat - i phi-hat) / sqrt 2
// (postprocess.cpp:61-99, 167-235), then the modes
//   Psi4^lm(r) = sum_points Psi4 conj(-2Y_lm(theta, phi)) sin(theta) dtheta dphi r
// for l = 2..l_max, m = -l..l, with the reference's -2Y_lm (l = 2 all m,
// l = 3 m = +-3, zero otherwise; postprocess.cpp:106-162).
//
// Two launches: one thread per sphere point writes Psi4 (zero outside the
// block) and counts the points inside, then one CTA per (mode, radius) sums the
// projections in a fixed order (deterministic; the reference sums point by
// point, so the two agree to rounding). Interpolation and contraction are
// separately rounded FP64 intrinsics in the reference's order; sin, cos and
// pow are CUDA's. A few thousand to a few hundred thousand points: latency-bound
// diagnostics whose point is to leave the state on the GPU.
#include "ccz4_kernels.h"

namespace granite_b200 {
namespace {

constexpr double PI_ = 3.14159265358979323846;  // constants::PI (types.hpp:71)

// postprocess.cpp:61-99: cell-centre trilinear interpolation with clamped indices.
__device__ double interp(const DevBlock& B, const double* __restrict__ u, int var, double px, double py, double pz) {
    const double ix = __dsub_rn(__dadd_rn(__ddiv_rn(__dsub_rn(px, B.lo[0]), B.dx[0]), (double)NG), 0.5);
    const double iy = __dsub_rn(__dadd_rn(__ddiv_rn(__dsub_rn(py, B.lo[1]), B.dx[1]), (double)NG), 0.5);
    const double iz = __dsub_rn(__dadd_rn(__ddiv_rn(__dsub_rn(pz, B.lo[2]), B.dx[2]), (double)NG), 0.5);
    const int nx = B.tx - 1, ny = B.ty - 1, nz = B.tz - 1;
    const int i0 = min(max((int)floor(ix), 0), nx - 1), j0 = min(max((int)floor(iy), 0), ny - 1),
              k0 = min(max((int)floor(iz), 0), nz - 1);
    const int i1 = min(i0 + 1, nx), j1 = min(j0 + 1, ny), k1 = min(k0 + 1, nz);
    const double wx = __dsub_rn(ix, floor(ix)), wy = __dsub_rn(iy, floor(iy)), wz = __dsub_rn(iz, floor(iz));
    const double* f = u + (long long)var * B.stride;
    auto d = [&](int i, int j, int k) { return __ldg(f + cell_index(B, i, j, k)); };
    const double ax = __dsub_rn(1.0, wx), ay = __dsub_rn(1.0, wy), az = __dsub_rn(1.0, wz);
    auto lx = [&](int j, int k) { return __dadd_rn(__dmul_rn(ax, d(i0, j, k)), __dmul_rn(wx, d(i1, j, k))); };
    const double z0 = __dadd_rn(__dmul_rn(ay, lx(j0, k0)), __dmul_rn(wy, lx(j1, k0)));
    const double z1 = __dadd_rn(__dmul_rn(ay, lx(j0, k1)), __dmul_rn(wy, lx(j1, k1)));
    return __dadd_rn(__dmul_rn(az, z0), __dmul_rn(wz, z1));
}

struct Cx {
    double re, im;
};
__device__ __forceinline__ Cx cmul(Cx a, Cx b) {
    return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
            __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ Cx cscale(Cx a, double s) { return {__dmul_rn(a.re, s), __dmul_rn(a.im, s)}; }
__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return {__dadd_rn(a.re, b.re), __dadd_rn(a.im, b.im)}; }

struct SphereArgs {
    double hi[3];     // the block's upper corner (GridBlock::upperCorner)
    double dth, dph;  // pi / n_theta, 2 pi / n_phi
    int nr, nth, nph;
};

__global__ void psi4_point_kernel(const DevBlock B, const double* __restrict__ u, const double* __restrict__ radii,
                                  const SphereArgs s, double2* __restrict__ psi4,
                                  unsigned int* __restrict__ inside_count) {
    const long long n = (long long)s.nr * s.nth * s.nph;
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int jp = (int)(p % s.nph), it = (int)((p / s.nph) % s.nth), r = (int)(p / ((long long)s.nph * s.nth));
    const double r_ext = radii[r];
    const double theta = __dmul_rn(__dadd_rn((double)it, 0.5), s.dth), phi = __dmul_rn((double)jp, s.dph);
    const double sth = sin(theta), cth = cos(theta), sph = sin(phi), cph = cos(phi);
    const double px = __dmul_rn(__dmul_rn(r_ext, sth), cph), py = __dmul_rn(__dmul_rn(r_ext, sth), sph),
                 pz = __dmul_rn(r_ext, cth);
    const double nx = __dmul_rn(sth, cph), ny = __dmul_rn(sth, sph), nz = cth;
    double2 out = make_double2(0.0, 0.0);
    const bool inside = px >= __dadd_rn(B.lo[0], B.dx[0]) && px <= __dsub_rn(s.hi[0], B.dx[0]) &&
        py >= __dadd_rn(B.lo[1], B.dx[1]) && py <= __dsub_rn(s.hi[1], B.dx[1]) &&
        pz >= __dadd_rn(B.lo[2], B.dx[2]) && pz <= __dsub_rn(s.hi[2], B.dx[2]);
    if (inside) {
        atomicAdd(inside_count + r, 1u);
        const double chi = interp(B, u, CHI, px, py, pz);
        if (!(chi < 1.0e-12)) {  // the reference returns zero below 1e-12 (a NaN goes on)
            const double rho = __dsqrt_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)));
            double tx = 1.0, ty = 0.0, tz = 0.0, phx = 0.0, phy = 1.0, phz = 0.0;
            if (rho > 1.0e-10) {
                tx = __ddiv_rn(__dmul_rn(nx, nz), rho);
                ty = __ddiv_rn(__dmul_rn(ny, nz), rho);
                tz = -rho;
                phx = __ddiv_rn(-ny, rho);
                phy = __ddiv_rn(nx, rho);
                phz = 0.0;
            }
            const double sq2 = __dsqrt_rn(2.0);
            const Cx mx = {__ddiv_rn(tx, sq2), __ddiv_rn(-phx, sq2)}, my = {__ddiv_rn(ty, sq2), __ddiv_rn(-phy, sq2)},
                     mz = {__ddiv_rn(tz, sq2), __ddiv_rn(-phz, sq2)};
            const double fac = __ddiv_rn(1.0, chi);
            const double Bxx = __dmul_rn(interp(B, u, AXX, px, py, pz), fac);
            const double Bxy = __dmul_rn(interp(B, u, AXY, px, py, pz), fac);
            const double Bxz = __dmul_rn(interp(B, u, AXZ, px, py, pz), fac);
            const double Byy = __dmul_rn(interp(B, u, AYY, px, py, pz), fac);
            const double Byz = __dmul_rn(interp(B, u, AYZ, px, py, pz), fac);
            const double Bzz = __dmul_rn(interp(B, u, AZZ, px, py, pz), fac);
            Cx q = cmul(cscale(mx, Bxx), mx);
            q = cadd(q, cmul(cscale(my, Byy), my));
            q = cadd(q, cmul(cscale(mz, Bzz), mz));
            q = cadd(q, cmul(cscale(mx, __dmul_rn(2.0, Bxy)), my));
            q = cadd(q, cmul(cscale(mx, __dmul_rn(2.0, Bxz)), mz));
            q = cadd(q, cmul(cscale(my, __dmul_rn(2.0, Byz)), mz));
            out = make_double2(-q.re, -q.im);
        }
    }
    psi4[p] = out;
}

// -2Y_lm of postprocess.cpp:106-162 (zero for the modes the reference omits).
__device__ Cx sw_ylm(int l, int m, double theta, double phi) {
    const double c2th = cos(theta / 2.0), s2th = sin(theta / 2.0);
    const Cx e = {cos(__dmul_rn((double)m, phi)), sin(__dmul_rn((double)m, phi))};
    if (l == 2) {
        if (m == 2) return cscale(e, __dmul_rn(__dsqrt_rn(5.0 / (4.0 * PI_)), pow(c2th, 4.0)));
        if (m == 1) return cscale(e, __dmul_rn(__dmul_rn(__dsqrt_rn(5.0 / PI_), pow(c2th, 3.0)), s2th));
        if (m == 0)  // pow(x, 2) is x * x, as the compiler evaluates it
            return {__dmul_rn(__dmul_rn(__dsqrt_rn(15.0 / (2.0 * PI_)), __dmul_rn(c2th, c2th)), __dmul_rn(s2th, s2th)),
                    0.0};
        if (m == -1) return cscale(e, __dmul_rn(__dmul_rn(__dsqrt_rn(5.0 / PI_), c2th), pow(s2th, 3.0)));
        if (m == -2) return cscale(e, __dmul_rn(__dsqrt_rn(5.0 / (4.0 * PI_)), pow(s2th, 4.0)));
    }
    if (l == 3) {
        const double N33 = __dsqrt_rn(21.0 / (2.0 * PI_));
        if (m == 3) return cscale(e, __ddiv_rn(__dmul_rn(__dmul_rn(__ddiv_rn(-N33, 4.0), pow(c2th, 5.0)), s2th), 2.0));
        if (m == -3) return cscale(e, __ddiv_rn(__dmul_rn(__dmul_rn(__ddiv_rn(N33, 4.0), c2th), pow(s2th, 5.0)), 2.0));
    }
    return {0.0, 0.0};
}

constexpr int MODE_THREADS = 256;

__global__ void __launch_bounds__(MODE_THREADS)
    psi4_modes_kernel(const double* __restrict__ radii, const SphereArgs s, const double2* __restrict__ psi4,
                      double2* __restrict__ modes) {
    const int q = blockIdx.x, r = blockIdx.y, nm = gridDim.x;
    int l = 2;
    while (q >= (l + 1) * (l + 1) - 4) ++l;
    const int m = q - (l * l - 4) - l;
    const double r_ext = radii[r];
    const int npts = s.nth * s.nph;
    const double2* P = psi4 + (long long)r * npts;
    double re = 0.0, im = 0.0;
    for (int p = threadIdx.x; p < npts; p += MODE_THREADS) {
        const double2 v = P[p];
        if (v.x == 0.0 && v.y == 0.0) continue;  // outside the block (or zero): adds nothing
        const int it = p / s.nph, jp = p % s.nph;
        const double theta = __dmul_rn(__dadd_rn((double)it, 0.5), s.dth), phi = __dmul_rn((double)jp, s.dph);
        Cx y = sw_ylm(l, m, theta, phi);
        y.im = -y.im;
        const Cx c = cscale(cscale(cscale(cscale(cmul({v.x, v.y}, y), sin(theta)), s.dth), s.dph), r_ext);
        re = __dadd_rn(re, c.re);
        im = __dadd_rn(im, c.im);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    __shared__ double sre[MODE_THREADS / 32], sim[MODE_THREADS / 32];
    if ((threadIdx.x & 31) == 0) {
        sre[threadIdx.x >> 5] = re;
        sim[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < MODE_THREADS / 32; ++w) {
            a += sre[w];
            b += sim[w];
        }
        modes[(long long)r * nm + q] = make_double2(a, b);
    }
}

}  // namespace

cudaError_t launch_psi4_modes(const DevBlock& B, const double* u, const double hi[3], const double* radii, int nr,
                              int n_theta, int n_phi, int l_max, double2* psi4_scratch, double2* modes,
                              unsigned int* inside_count, cudaStream_t stream) {
    SphereArgs s;
    for (int d = 0; d < 3; ++d) s.hi[d] = hi[d];
    s.dth = PI_ / n_theta;
    s.dph = 2.0 * PI_ / n_phi;
    s.nr = nr;
    s.nth = n_theta;
    s.nph = n_phi;
    const long long n = (long long)nr * n_theta * n_phi;
    cudaError_t e = cudaMemsetAsync(inside_count, 0, (size_t)nr * sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    psi4_point_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(B, u, radii, s, psi4_scratch, inside_count);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int nm = (l_max + 1) * (l_max + 1) - 4;
    psi4_modes_kernel<<<dim3(nm, nr), MODE_THREADS, 0, stream>>>(radii, s, psi4_scratch, modes);
    return cudaGetLastError();
}

}  // namespace granite_b200
