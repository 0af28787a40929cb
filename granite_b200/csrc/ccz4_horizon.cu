// ccz4_horizon.cu -- apparent-horizon flow on the device.
//
// ApparentHorizonFinder::findHorizon (horizon_finder.cpp:310-449): a trial
// surface r = h(theta_i, phi_j) around a centre flows as h <- max(h - 0.05 dx
// Theta, 1e-6 dx), Theta the null expansion at the surface point for the
// coordinate radial normal (computeExpansion, :114-281: interpolated chi,
// gamma~_ij, A~_ij, K; D_i s^i from centred differences of the unit normal at
// +-dx). Every surface point flows on its own: Theta at a point depends on its
// own radius only. The reference stops at the first iteration whose largest
// |Theta| is below the tolerance, after that iteration's update.
//
// One thread per surface point runs a chunk of iterations, keeps its radius
// after each one and folds |Theta| into a per-iteration maximum (atomicMax on
// the bits of a non-negative double; a NaN is skipped, as std::max skips it);
// the host finds the first converged iteration of the chunk and takes that
// iteration's radii. The arithmetic is the reference's, operation for
// operation, in separately rounded FP64 intrinsics, and the angular tables
// come from the host's libm, so the flow equals the reference bit for bit.
// The surface integrals (area, J_z) are evaluated per point here and summed on
// the host in the reference's order.
#include "ccz4_kernels.h"

namespace granite_b200 {
namespace {

// horizon_finder.cpp:55-98: trilinear, indices clamped at each access.
__device__ double hz_interp(const DevBlock& B, const double* __restrict__ u, int var, double px, double py,
                            double pz) {
    const double ix = __dsub_rn(__dadd_rn(__ddiv_rn(__dsub_rn(px, B.lo[0]), B.dx[0]), (double)NG), 0.5);
    const double iy = __dsub_rn(__dadd_rn(__ddiv_rn(__dsub_rn(py, B.lo[1]), B.dx[1]), (double)NG), 0.5);
    const double iz = __dsub_rn(__dadd_rn(__ddiv_rn(__dsub_rn(pz, B.lo[2]), B.dx[2]), (double)NG), 0.5);
    const int i0 = (int)floor(ix), j0 = (int)floor(iy), k0 = (int)floor(iz);
    const int nx = B.tx - 1, ny = B.ty - 1, nz = B.tz - 1;
    const int i1 = min(i0 + 1, nx), j1 = min(j0 + 1, ny), k1 = min(k0 + 1, nz);
    const double wx = __dsub_rn(ix, floor(ix)), wy = __dsub_rn(iy, floor(iy)), wz = __dsub_rn(iz, floor(iz));
    const double* f = u + (long long)var * B.stride;
    auto d = [&](int i, int j, int k) {
        return __ldg(f + cell_index(B, max(0, min(i, nx)), max(0, min(j, ny)), max(0, min(k, nz))));
    };
    const double ax = __dsub_rn(1.0, wx), ay = __dsub_rn(1.0, wy), az = __dsub_rn(1.0, wz);
    auto lx = [&](int j, int k) { return __dadd_rn(__dmul_rn(ax, d(i0, j, k)), __dmul_rn(wx, d(i1, j, k))); };
    const double z0 = __dadd_rn(__dmul_rn(ay, lx(j0, k0)), __dmul_rn(wy, lx(j1, k0)));
    const double z1 = __dadd_rn(__dmul_rn(ay, lx(j0, k1)), __dmul_rn(wy, lx(j1, k1)));
    return __dadd_rn(__dmul_rn(az, z0), __dmul_rn(wz, z1));
}

#define M(a, b) __dmul_rn(a, b)
#define A(a, b) __dadd_rn(a, b)
#define S(a, b) __dsub_rn(a, b)
#define Q(a, b) __ddiv_rn(a, b)

// gamma~ determinant as horizon_finder.cpp:145-146 writes it
__device__ __forceinline__ double det3(double gxx, double gxy, double gxz, double gyy, double gyz, double gzz) {
    return A(S(M(gxx, S(M(gyy, gzz), M(gyz, gyz))), M(gxy, S(M(gxy, gzz), M(gyz, gxz)))),
             M(gxz, S(M(gxy, gyz), M(gyy, gxz))));
}

// the scomp lambda of horizon_finder.cpp:222-276: component dir of s^i at the displaced point
__device__ double hz_scomp(const DevBlock& B, const double* __restrict__ u, double px, double py, double pz, double snx,
                           double sny, double snz, int dir, double delta) {
    const double ppx = A(px, dir == 0 ? delta : 0.0), ppy = A(py, dir == 1 ? delta : 0.0),
                 ppz = A(pz, dir == 2 ? delta : 0.0);
    const double chi = hz_interp(B, u, CHI, ppx, ppy, ppz);
    if (chi < 1.0e-12) return 0.0;
    const double gxx = hz_interp(B, u, GXX, ppx, ppy, ppz), gxy = hz_interp(B, u, GXY, ppx, ppy, ppz),
                 gxz = hz_interp(B, u, GXZ, ppx, ppy, ppz), gyy = hz_interp(B, u, GYY, ppx, ppy, ppz),
                 gyz = hz_interp(B, u, GYZ, ppx, ppy, ppz), gzz = hz_interp(B, u, GZZ, ppx, ppy, ppz);
    const double det = det3(gxx, gxy, gxz, gyy, gyz, gzz);
    if (fabs(det) < 1.0e-14) return 0.0;
    const double idet = Q(1.0, det);
    const double hxx = Q(gxx, chi), hxy = Q(gxy, chi), hxz = Q(gxz, chi), hyy = Q(gyy, chi), hyz = Q(gyz, chi),
                 hzz = Q(gzz, chi);
    const double sx = A(A(M(hxx, snx), M(hxy, sny)), M(hxz, snz));
    const double sy = A(A(M(hxy, snx), M(hyy, sny)), M(hyz, snz));
    const double sz = A(A(M(hxz, snx), M(hyz, sny)), M(hzz, snz));
    const double n2 = A(A(M(snx, sx), M(sny, sy)), M(snz, sz));
    if (n2 < 1.0e-14) return 0.0;
    const double nm = __dsqrt_rn(n2);
    if (dir == 0) {
        const double ixx = M(chi, M(S(M(gyy, gzz), M(gyz, gyz)), idet));
        const double ixy = M(chi, M(S(M(gxz, gyz), M(gxy, gzz)), idet));
        const double ixz = M(chi, M(S(M(gxy, gyz), M(gxz, gyy)), idet));
        return Q(A(A(M(ixx, sx), M(ixy, sy)), M(ixz, sz)), nm);
    }
    if (dir == 1) {
        const double ixy = M(chi, M(S(M(gxz, gyz), M(gxy, gzz)), idet));
        const double iyy = M(chi, M(S(M(gxx, gzz), M(gxz, gxz)), idet));
        const double iyz = M(chi, M(S(M(gxy, gxz), M(gxx, gyz)), idet));
        return Q(A(A(M(ixy, sx), M(iyy, sy)), M(iyz, sz)), nm);
    }
    const double ixz = M(chi, M(S(M(gxy, gyz), M(gxz, gyy)), idet));
    const double iyz = M(chi, M(S(M(gxy, gxz), M(gxx, gyz)), idet));
    const double izz = M(chi, M(S(M(gxx, gyy), M(gxy, gxy)), idet));
    return Q(A(A(M(ixz, sx), M(iyz, sy)), M(izz, sz)), nm);
}

// computeExpansion, horizon_finder.cpp:114-281
__device__ double hz_expansion(const DevBlock& B, const double* __restrict__ u, double px, double py, double pz,
                               double snx, double sny, double snz) {
    const double chi = hz_interp(B, u, CHI, px, py, pz);
    const double gxx = hz_interp(B, u, GXX, px, py, pz), gxy = hz_interp(B, u, GXY, px, py, pz),
                 gxz = hz_interp(B, u, GXZ, px, py, pz), gyy = hz_interp(B, u, GYY, px, py, pz),
                 gyz = hz_interp(B, u, GYZ, px, py, pz), gzz = hz_interp(B, u, GZZ, px, py, pz);
    if (chi < 1.0e-12) return 0.0;
    const double det = det3(gxx, gxy, gxz, gyy, gyz, gzz);
    if (fabs(det) < 1.0e-14) return 0.0;
    const double hxx = Q(gxx, chi), hxy = Q(gxy, chi), hxz = Q(gxz, chi), hyy = Q(gyy, chi), hyz = Q(gyz, chi),
                 hzz = Q(gzz, chi);
    const double sx = A(A(M(hxx, snx), M(hxy, sny)), M(hxz, snz));
    const double sy = A(A(M(hxy, snx), M(hyy, sny)), M(hyz, snz));
    const double sz = A(A(M(hxz, snx), M(hyz, sny)), M(hzz, snz));
    const double norm2 = A(A(M(snx, sx), M(sny, sy)), M(snz, sz));
    if (norm2 < 1.0e-14) return 0.0;
    const double norm = __dsqrt_rn(norm2);
    const double ux = Q(snx, norm), uy = Q(sny, norm), uz = Q(snz, norm);
    const double K = hz_interp(B, u, KTR, px, py, pz);
    auto kij = [&](int a, double g) { return Q(A(hz_interp(B, u, a, px, py, pz), Q(M(g, K), 3.0)), chi); };
    const double Kxx = kij(AXX, gxx), Kxy = kij(AXY, gxy), Kxz = kij(AXZ, gxz), Kyy = kij(AYY, gyy),
                 Kyz = kij(AYZ, gyz), Kzz = kij(AZZ, gzz);
    const double Kss = A(A(A(M(M(Kxx, ux), ux), M(M(Kyy, uy), uy)), M(M(Kzz, uz), uz)),
                         M(2.0, A(A(M(M(Kxy, ux), uy), M(M(Kxz, ux), uz)), M(M(Kyz, uy), uz))));
    const double eps = B.dx[0], e2 = M(2.0, eps);
    const double d0 = Q(S(hz_scomp(B, u, px, py, pz, snx, sny, snz, 0, eps), hz_scomp(B, u, px, py, pz, snx, sny, snz, 0, -eps)), e2);
    const double d1 = Q(S(hz_scomp(B, u, px, py, pz, snx, sny, snz, 1, eps), hz_scomp(B, u, px, py, pz, snx, sny, snz, 1, -eps)), e2);
    const double d2 = Q(S(hz_scomp(B, u, px, py, pz, snx, sny, snz, 2, eps), hz_scomp(B, u, px, py, pz, snx, sny, snz, 2, -eps)), e2);
    return S(A(A(A(d0, d1), d2), K), Kss);
}

__global__ void horizon_flow_kernel(const DevBlock B, const double* __restrict__ u, const HorizonArgs a,
                                    const double* __restrict__ tab, double* __restrict__ h, int iters,
                                    double* __restrict__ hist, unsigned long long* __restrict__ itmax) {
    const int N = a.nth * a.nph;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int i = p / a.nph, j = p % a.nph;
    const double sth = tab[i], cth = tab[a.nth + i], sph = tab[2 * a.nth + j], cph = tab[2 * a.nth + a.nph + j];
    const double nx = M(sth, cph), ny = M(sth, sph), nz = cth;
    double r = h[p];
    for (int k = 0; k < iters; ++k) {
        const double px = A(a.center[0], M(M(r, sth), cph)), py = A(a.center[1], M(M(r, sth), sph)),
                     pz = A(a.center[2], M(r, cth));
        const double th = hz_expansion(B, u, px, py, pz, nx, ny, nz);
        r = S(r, M(a.flow_step, th));
        r = r < a.rmin ? a.rmin : r;
        hist[(long long)k * N + p] = r;
        const double at = fabs(th);
        if (!isnan(at)) atomicMax(itmax + k, (unsigned long long)__double_as_longlong(at));
    }
    h[p] = r;
}

// per-point terms of the area and J_z sums (horizon_finder.cpp:381-412); flag 0 where chi < 1e-12
__global__ void horizon_surface_kernel(const DevBlock B, const double* __restrict__ u, const HorizonArgs a,
                                       const double* __restrict__ tab, const double* __restrict__ h,
                                       double* __restrict__ terms) {
    const int N = a.nth * a.nph;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int i = p / a.nph, j = p % a.nph;
    const double sth = tab[i], cth = tab[a.nth + i], sph = tab[2 * a.nth + j], cph = tab[2 * a.nth + a.nph + j];
    const double r = h[p];
    const double px = A(a.center[0], M(M(r, sth), cph)), py = A(a.center[1], M(M(r, sth), sph)),
                 pz = A(a.center[2], M(r, cth));
    const double chi = hz_interp(B, u, CHI, px, py, pz);
    double ar = 0.0, jz = 0.0, ok = 0.0;
    if (!(chi < 1.0e-12)) {
        const double gxx = hz_interp(B, u, GXX, px, py, pz), gyy = hz_interp(B, u, GYY, px, py, pz),
                     gzz = hz_interp(B, u, GZZ, px, py, pz);
        const double sg = Q(__dsqrt_rn(fabs(M(M(gxx, gyy), gzz))), M(chi, __dsqrt_rn(chi)));
        ar = M(M(M(M(M(sg, r), r), sth), a.dth), a.dph);
        jz = M(M(M(M(M(A(M(-sph, px), M(cph, py)), sg), r), sth), a.dth), a.dph);
        ok = 1.0;
    }
    terms[3 * p] = ar;
    terms[3 * p + 1] = jz;
    terms[3 * p + 2] = ok;
}

// findAllHorizons' scan (horizon_finder.cpp:458-477): interior cells two in from
// the faces whose lapse is below 0.5 and below all six neighbours
__global__ void lapse_minima_kernel(const DevBlock B, const double* __restrict__ u, long long* __restrict__ out,
                                    unsigned int* __restrict__ count, unsigned int cap) {
    const int i = NG + 2 + blockIdx.x * blockDim.x + threadIdx.x, j = NG + 2 + blockIdx.y, k = NG + 2 + blockIdx.z;
    if (i >= NG + B.n[0] - 2) return;
    const double* f = u + (long long)ALPHA * B.stride;
    const long long c = cell_index(B, i, j, k), sy = B.tx, sz = (long long)B.tx * B.ty;
    const double al = __ldg(f + c);
    if (al < __ldg(f + c - 1) && al < __ldg(f + c + 1) && al < __ldg(f + c - sy) && al < __ldg(f + c + sy) &&
        al < __ldg(f + c - sz) && al < __ldg(f + c + sz) && al < 0.5) {
        const unsigned int q = atomicAdd(count, 1u);
        if (q < cap) out[q] = c;
    }
}

#undef M
#undef A
#undef S
#undef Q

}  // namespace

cudaError_t launch_horizon_flow(const DevBlock& B, const double* u, const HorizonArgs& a, const double* tab,
                                double* h, int iters, double* hist, unsigned long long* itmax, cudaStream_t stream) {
    const int N = a.nth * a.nph;
    cudaError_t e = cudaMemsetAsync(itmax, 0, (size_t)iters * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return e;
    horizon_flow_kernel<<<(N + 127) / 128, 128, 0, stream>>>(B, u, a, tab, h, iters, hist, itmax);
    return cudaGetLastError();
}

cudaError_t launch_horizon_surface(const DevBlock& B, const double* u, const HorizonArgs& a, const double* tab,
                                   const double* h, double* terms, cudaStream_t stream) {
    const int N = a.nth * a.nph;
    horizon_surface_kernel<<<(N + 127) / 128, 128, 0, stream>>>(B, u, a, tab, h, terms);
    return cudaGetLastError();
}

cudaError_t launch_lapse_minima(const DevBlock& B, const double* u, long long* out, unsigned int* count,
                                unsigned int cap, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned int), stream);
    if (e != cudaSuccess) return e;
    const int ni = B.n[0] - 4, nj = B.n[1] - 4, nk = B.n[2] - 4;
    if (ni <= 0 || nj <= 0 || nk <= 0) return cudaSuccess;
    lapse_minima_kernel<<<dim3((ni + 127) / 128, nj, nk), 128, 0, stream>>>(B, u, out, count, cap);
    return cudaGetLastError();
}

}  // namespace granite_b200
