// ccz4_stencil.cuh -- finite-difference stencils of the CCZ4 operator
// (ccz4.cpp:71-223 and the KO operator of ccz4.cpp:871-935), evaluated from
// FP64 pair differences so a reduced-precision algebra type P loses nothing
// to cancellation.
#pragma once

#include "ccz4_common.cuh"

namespace granite_b200 {
namespace {

template <typename T>
__device__ __forceinline__ T ld(const double* p) {
    return (T)__ldg(p);
}

// ---------------------------------------------------------------------------
// Stencil evaluation. `f` points at the centre value; `s` is one cell along
// the axis. Pair differences are taken in FP64 and rounded to P afterwards.
// ---------------------------------------------------------------------------
template <typename P>
struct AxisDer {
    P d1;   // 4th-order centred first derivative, ccz4.cpp:71-99
    P up;   // 4th-order one-sided derivative on the upwind side, ccz4.cpp:109-152
    P ko;   // sigma/(64 dx) x undivided 6th difference, ccz4.cpp:886-931
    P d2;   // 4th-order second derivative, ccz4.cpp:156-184
};

template <typename P, bool WANT_D2, bool WANT_KO>
__device__ __forceinline__ AxisDer<P> axis_der(const double* __restrict__ f, long long s, double f0,
                                              double beta, double inv12h, double inv12h2,
                                              double kocf) {
    const double fm1 = __ldg(f - s), fp1 = __ldg(f + s);
    const double fm2 = __ldg(f - 2 * s), fp2 = __ldg(f + 2 * s);
    const double fm3 = __ldg(f - 3 * s), fp3 = __ldg(f + 3 * s);
    AxisDer<P> r;
    // pair differences in FP64
    const double a1 = fp1 - fm1, a2 = fp2 - fm2;
    r.d1 = (P)inv12h * ((P)8.0 * (P)a1 - (P)a2);
    double e;
    if (beta >= 0.0) {
        const double fm4 = __ldg(f - 4 * s);
        // 25 f0 - 48 f-1 + 36 f-2 - 16 f-3 + 3 f-4 (weights sum to zero): differences vs f0
        e = 48.0 * (f0 - fm1) - 36.0 * (f0 - fm2) + 16.0 * (f0 - fm3) - 3.0 * (f0 - fm4);
    } else {
        const double fp4 = __ldg(f + 4 * s);
        e = -48.0 * (f0 - fp1) + 36.0 * (f0 - fp2) - 16.0 * (f0 - fp3) + 3.0 * (f0 - fp4);
    }
    r.up = (P)inv12h * (P)e;
    if (WANT_D2) {
        const double s1 = (fp1 - f0) + (fm1 - f0), s2 = (fp2 - f0) + (fm2 - f0);
        r.d2 = (P)inv12h2 * ((P)16.0 * (P)s1 - (P)s2);
    } else {
        r.d2 = (P)0;
    }
    if (WANT_KO) {
        const double t1 = (fp1 - f0) + (fm1 - f0);
        const double t2 = (fp2 - f0) + (fm2 - f0);
        const double t3 = (fp3 - f0) + (fm3 - f0);
        // (f-3 + f+3) - 6 (f-2 + f+2) + 15 (f-1 + f+1) - 20 f0 in differences vs f0
        r.ko = (P)kocf * ((P)t3 - (P)6.0 * (P)t2 + (P)15.0 * (P)t1);
    } else {
        r.ko = (P)0;
    }
    return r;
}

// 2nd-order mixed derivative, ccz4.cpp:185-222
template <typename P>
__device__ __forceinline__ P dmix(const double* __restrict__ f, long long sa, long long sb,
                                  double inv4hh) {
    const double pp = __ldg(f + sa + sb), pm = __ldg(f + sa - sb);
    const double mp = __ldg(f - sa + sb), mm = __ldg(f - sa - sb);
    return (P)inv4hh * (P)((pp - pm) - (mp - mm));
}

// Everything one field contributes: gradient, blended advection, KO, and
// (optionally) its Hessian.
template <typename P>
struct FieldDer {
    P d[3];
    P adv;   // w sum beta_d up_d + (1-w) sum beta_d d1_d, ccz4.cpp:567-574
    P ko;
    P h[6];  // xx xy xz yy yz zz
};

template <typename P, bool HESS>
__device__ __forceinline__ FieldDer<P> field_der(const DevBlock& B, const double* __restrict__ f,
                                                 const double beta[3], P w, bool ko_on) {
    const long long off[3] = {1, B.tx, (long long)B.tx * B.ty};
    const double f0 = __ldg(f);
    FieldDer<P> r;
    P up_sum = (P)0, cen_sum = (P)0, ko = (P)0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        AxisDer<P> a;
        if (ko_on)
            a = axis_der<P, HESS, true>(f, off[d], f0, beta[d], B.inv12h[d], B.inv12h2[d], B.kocf[d]);
        else
            a = axis_der<P, HESS, false>(f, off[d], f0, beta[d], B.inv12h[d], B.inv12h2[d], B.kocf[d]);
        r.d[d] = a.d1;
        up_sum += (P)beta[d] * a.up;
        cen_sum += (P)beta[d] * a.d1;
        ko += a.ko;
        if (HESS) r.h[d == 0 ? 0 : (d == 1 ? 3 : 5)] = a.d2;
    }
    r.adv = w * up_sum + ((P)1 - w) * cen_sum;
    r.ko = ko;
    if (HESS) {
        r.h[1] = dmix<P>(f, off[0], off[1], B.inv4hh[0]);
        r.h[2] = dmix<P>(f, off[0], off[2], B.inv4hh[1]);
        r.h[4] = dmix<P>(f, off[1], off[2], B.inv4hh[2]);
    } else {
#pragma unroll
        for (int a = 0; a < 6; ++a) r.h[a] = (P)0;
    }
    return r;
}

__device__ __forceinline__ int sy(int a, int b) {
    // symmetric pair -> packed index (types.hpp:52-54)
    return (a <= b) ? (a * 3 - a * (a - 1) / 2 + b - a) : (b * 3 - b * (b - 1) / 2 + a - b);
}

}  // namespace
}  // namespace granite_b200
