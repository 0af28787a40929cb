// ccz4_stencil.cuh -- finite-difference stencils of the CCZ4 operator
// (ccz4.cpp:71-223) and the Kreiss-Oliger operator (ccz4.cpp:871-935).
//
// Two evaluation modes, chosen by the algebra type P:
//
//  P = double (plain FP64): every stencil is evaluated in the reference's
//    operation order with explicitly rounded products and sums, so the
//    derivatives and the KO term are bit-identical to the host code. This
//    matters where a field is O(1) and its RHS is ~1e-6 of that (noisy flat
//    regions): there the rounding of the reference's own stencil sums is the
//    size of the result, and only the same rounding reproduces it.
//
//  P = float (mixed): stencils are evaluated from FP64 pair differences
//    (f[+k] - f[-k], f[+k] + f[-k] - 2 f[0], ...) that cancel exactly, and only
//    the small differences are rounded to FP32; the algebra downstream runs in
//    FP32 without losing the cancellation.
#pragma once

#include "ccz4_common.cuh"

namespace granite_b200 {
namespace {

#define RN_MUL __dmul_rn
#define RN_ADD __dadd_rn
#define RN_SUB __dsub_rn

// Value loaders: offset (in cells) from a centre pointer.
struct GlobalLoad {  // read-only global memory through the non-coherent path
    const double* __restrict__ p;
    __device__ __forceinline__ double operator()(long long o) const { return __ldg(p + o); }
};
struct SharedLoad {  // a CTA-staged tile in shared memory
    const double* p;
    __device__ __forceinline__ double operator()(long long o) const { return p[o]; }
};

template <typename P>
struct AxisDer {
    P d1;  // 4th-order centred first derivative, ccz4.cpp:71-99
    P up;  // 4th-order one-sided derivative on the upwind side, ccz4.cpp:109-152
    P d2;  // 4th-order second derivative, ccz4.cpp:156-184
};

// Reference-order evaluation (P = double). `ko` accumulates the KO sum across
// the three axes exactly as ccz4.cpp:912-926 does.
//
// The upwind derivative is evaluated without a branch: both +-4 arms are
// loaded and the side is selected. The beta < 0 form of ccz4.cpp:109-152,
// inv12h (-25 f0 + 48 f+1 - 36 f+2 + 16 f+3 - 3 f+4), rounded left to right,
// is bit for bit the negation of the beta >= 0 form applied to the + side
// (round-to-nearest is odd-symmetric; only the sign of an exact zero differs).
template <bool WANT_D2, bool WANT_KO, typename L>
__device__ __forceinline__ AxisDer<double> axis_exact(const L& f, long long s, double f0,
                                                     double beta, double inv12h, double inv12h2,
                                                     const double* kw, double& ko) {
    const double fm1 = f(-s), fp1 = f(s);
    const double fm2 = f(-2 * s), fp2 = f(2 * s);
    const double fm3 = f(-3 * s), fp3 = f(3 * s);
    const double fm4 = f(-4 * s), fp4 = f(4 * s);
    AxisDer<double> r;
    // inv12h * (-f[+2] + 8 f[+1] - 8 f[-1] + f[-2])
    r.d1 = RN_MUL(inv12h, RN_ADD(RN_SUB(RN_ADD(-fp2, RN_MUL(8.0, fp1)), RN_MUL(8.0, fm1)), fm2));
    const bool pos = beta >= 0.0;
    const double g1 = pos ? fm1 : fp1, g2 = pos ? fm2 : fp2, g3 = pos ? fm3 : fp3, g4 = pos ? fm4 : fp4;
    // inv12h * (25 f0 - 48 g1 + 36 g2 - 16 g3 + 3 g4), g = the - side for beta >= 0
    const double up = RN_MUL(inv12h, RN_ADD(RN_SUB(RN_ADD(RN_SUB(RN_MUL(25.0, f0), RN_MUL(48.0, g1)), RN_MUL(36.0, g2)),
                                                   RN_MUL(16.0, g3)),
                                            RN_MUL(3.0, g4)));
    r.up = pos ? up : -up;
    if (WANT_D2) {
        // inv12h2 * (-f[+2] + 16 f[+1] - 30 f0 + 16 f[-1] - f[-2])
        r.d2 = RN_MUL(inv12h2, RN_SUB(RN_ADD(RN_SUB(RN_ADD(-fp2, RN_MUL(16.0, fp1)), RN_MUL(30.0, f0)),
                                             RN_MUL(16.0, fm1)),
                                      fm2));
    } else {
        r.d2 = 0.0;
    }
    if (WANT_KO) {
        // diss += (cf w_s) u(x + s e_d), s = -3..3, w = {1,-6,15,-20,15,-6,1}
        ko = RN_ADD(ko, RN_MUL(kw[0], fm3));
        ko = RN_ADD(ko, RN_MUL(kw[1], fm2));
        ko = RN_ADD(ko, RN_MUL(kw[2], fm1));
        ko = RN_ADD(ko, RN_MUL(kw[3], f0));
        ko = RN_ADD(ko, RN_MUL(kw[2], fp1));
        ko = RN_ADD(ko, RN_MUL(kw[1], fp2));
        ko = RN_ADD(ko, RN_MUL(kw[0], fp3));
    }
    return r;
}

// Pair-difference evaluation (P = float: the mixed form; P = double: the FP64
// pass of the per-tile precision, equal to the reference-order form to
// rounding). The pair differences and their weighted sums stay FP64 (small,
// exactly cancelled numbers) and each derivative the algebra uses is rounded
// to P once. The advection and KO terms are sums over the three axes: they
// are accumulated in FP64 (upd, kod) and rounded once per field by the caller,
// which saves two conversions per axis.
//
// The upwind stencil (ccz4.cpp:109-152) takes the side of the shift: for
// beta >= 0, e = 25 f0 - 48 g1 + 36 g2 - 16 g3 + 3 g4 with g_k = f[-k], and
// beta e goes into the advection sum; for beta < 0 the mirror (g_k = f[+k])
// with -e, so the term is |beta| e either way and needs no select of e. The
// fourth neighbour is loaded once from the selected side (sgn_s = -s or +s).
template <bool WANT_D2, bool WANT_KO, typename P, typename L>
__device__ __forceinline__ void axis_pairs(const L& f, long long s, long long sgn_s, double f0, double beta,
                                           double inv12h, double inv12h2, double kocf, P& d1, P& d2,
                                           double& upd, double& kod) {
    // differences from the centre, a_k = f[-k] - f0 and b_k = f[+k] - f0, shared by
    // every stencil below
    const double a1 = f(-s) - f0, b1 = f(s) - f0;
    const double a2 = f(-2 * s) - f0, b2 = f(2 * s) - f0;
    const double a3 = f(-3 * s) - f0, b3 = f(3 * s) - f0;
    const double c4 = f(4 * sgn_s) - f0;
    // 8 (f+1 - f-1) - (f+2 - f-2)
    d1 = (P)inv12h * (P)(8.0 * (b1 - a1) - (b2 - a2));
    const bool pos = beta >= 0.0;
    const double x1 = pos ? a1 : b1, x2 = pos ? a2 : b2, x3 = pos ? a3 : b3;
    // 25 f0 - 48 g1 + 36 g2 - 16 g3 + 3 g4 (g: the upwind side), weights summing to zero
    const double e = -48.0 * x1 + 36.0 * x2 - 16.0 * x3 + 3.0 * c4;
    upd += (fabs(beta) * inv12h) * e;
    const double t1 = b1 + a1;
    const double t2 = b2 + a2;
    d2 = WANT_D2 ? (P)inv12h2 * (P)(16.0 * t1 - t2) : (P)0;
    if (WANT_KO) {
        // (f-3 + f+3) - 6 (f-2 + f+2) + 15 (f-1 + f+1) - 20 f0
        kod += kocf * ((b3 + a3) - 6.0 * t2 + 15.0 * t1);
    }
}

// 2nd-order mixed derivative, ccz4.cpp:185-222: inv4hh * (f++ - f+- - f-+ + f--),
// in the reference's order (EXACT) or from pair differences.
template <typename P, bool EXACT, typename L>
__device__ __forceinline__ P dmix(const L& f, long long sa, long long sb, double inv4hh) {
    const double pp = f(sa + sb), pm = f(sa - sb);
    const double mp = f(-sa + sb), mm = f(-sa - sb);
    if constexpr (EXACT)
        return RN_MUL(inv4hh, RN_ADD(RN_SUB(RN_SUB(pp, pm), mp), mm));
    else
        return (P)inv4hh * (P)((pp - pm) - (mp - mm));
}

// Everything one field contributes: gradient, blended advection, KO, and
// (optionally) its Hessian.
template <typename P>
struct FieldDer {
    P d[3];
    P adv;  // w sum beta_d up_d + (1-w) sum beta_d d1_d, ccz4.cpp:567-574
    P ko;   // KO term of the field (added after the rest of its RHS)
    P h[6]; // xx xy xz yy yz zz
};

// EXACT (P = double only): every stencil in the reference's operation order.
template <typename P, bool HESS, bool KO, typename L, bool EXACT = (sizeof(P) == 8)>
__device__ __forceinline__ FieldDer<P> field_der_l(const DevBlock& B, const L& f, const long long off[3],
                                                   const double beta[3], P w) {
    static_assert(!EXACT || sizeof(P) == 8, "reference-order stencils are FP64");
    const double f0 = f(0);
    FieldDer<P> r;
    const P b0 = (P)beta[0], b1 = (P)beta[1], b2 = (P)beta[2];
    if constexpr (EXACT) {
        P up[3];
        P ko = (P)0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const AxisDer<P> a = axis_exact<HESS, KO>(f, off[d], f0, beta[d], B.inv12h[d], B.inv12h2[d], B.kow[d], ko);
            r.d[d] = a.d1;
            up[d] = a.up;
            if (HESS) r.h[d == 0 ? 0 : (d == 1 ? 3 : 5)] = a.d2;
        }
        const P up_sum = b0 * up[0] + b1 * up[1] + b2 * up[2];
        const P cen_sum = b0 * r.d[0] + b1 * r.d[1] + b2 * r.d[2];
        r.adv = w * up_sum + ((P)1 - w) * cen_sum;
        r.ko = ko;
    } else {
        double upd = 0.0, kod = 0.0;  // sum_d beta_d up_d and the KO sum, FP64
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            P d2;
            axis_pairs<HESS, KO, P>(f, off[d], beta[d] >= 0.0 ? -off[d] : off[d], f0, beta[d], B.inv12h[d],
                                    B.inv12h2[d], B.kocf[d], r.d[d], d2, upd, kod);
            if (HESS) r.h[d == 0 ? 0 : (d == 1 ? 3 : 5)] = d2;
        }
        const P cen_sum = b0 * r.d[0] + b1 * r.d[1] + b2 * r.d[2];
        r.adv = w * (P)upd + ((P)1 - w) * cen_sum;
        r.ko = (P)kod;
    }
    if (HESS) {
        r.h[1] = dmix<P, EXACT, L>(f, off[0], off[1], B.inv4hh[0]);
        r.h[2] = dmix<P, EXACT, L>(f, off[0], off[2], B.inv4hh[1]);
        r.h[4] = dmix<P, EXACT, L>(f, off[1], off[2], B.inv4hh[2]);
    } else {
#pragma unroll
        for (int a = 0; a < 6; ++a) r.h[a] = (P)0;
    }
    return r;
}

// Field derivatives straight from global memory, without the KO term.
template <typename P, bool HESS>
__device__ __forceinline__ FieldDer<P> field_der_noko(const DevBlock& B, const double* __restrict__ f,
                                                      const double beta[3], P w) {
    const long long off[3] = {1, B.tx, (long long)B.tx * B.ty};
    return field_der_l<P, HESS, false>(B, GlobalLoad{f}, off, beta, w);
}

__device__ __forceinline__ int sy(int a, int b) {
    // symmetric pair -> packed index (types.hpp:52-54)
    return (a <= b) ? (a * 3 - a * (a - 1) / 2 + b - a) : (b * 3 - b * (b - 1) / 2 + a - b);
}

}  // namespace
}  // namespace granite_b200
