// ccz4_point.cuh -- the CCZ4 right-hand side at one interior point, shared by
// every stage kernel (global-load, cp.async and TMA variants).
//
// Physics: CCZ4Evolution::computeRHS (ccz4.cpp:251-865) plus applyDissipation
// (ccz4.cpp:871-935). The algebra is regrouped (first-kind Christoffels reused
// in the Ricci tensor, mixed-index A and Christoffel contractions computed
// once) but every term of the reference is kept with the same coefficients,
// regularisers and blend, so results agree with the reference to rounding.
//
// Epilogues (stage_epilogue):
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
// stay FP64.
//
// A stencil source S provides der<HESS, EXACT>(v, beta, w), the derivatives of
// field v, called for the fields in FIELD_ORDER; S::HS says whether it also
// provides per-thread shared-memory slots (hess_slots, stride S::NT) for the
// values of the Hessian-field loop, and S::UNROLL whether that loop may be
// unrolled (a source whose der() is short).
#pragma once

#include <type_traits>

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
    static constexpr bool HS = false;      // the Hessian-field loop's values stay in (local) registers
    static constexpr bool UNROLL = false;  // and the loop stays rolled (stencil code is long)
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

// ---------------------------------------------------------------------------
// RHS at one interior point. Returns L(u) for the 22 fields in `out` (FP64).
// ---------------------------------------------------------------------------
// EXACT: FP64 stencils in the reference's operation order (P = double only).
template <typename P, bool EXACT, typename Src>
__device__ __forceinline__ void ccz4_point(const DevBlock& B, const double* __restrict__ u,
                                           long long c, const StageArgs& A, Src& S, P out[NV]) {
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
    // hold, and instruction fetch stalls the warps. The 36 values it produces
    // go to this thread's column of shared memory when the source provides one
    // (Src::HS: slot q of the thread at hs[q * Src::NT]), else to an array in
    // L1-cached local memory.
    P* hs = nullptr;
    if constexpr (Src::HS) {
        hs = S.template hess_slots<P>();
        constexpr int T = Src::HS ? Src::NT : 1;
#pragma unroll 1
        for (int a = 0; a < 6; ++a) {
            FieldDer<P> fd = S.template der<true, EXACT>(GXX + a, beta, w);
#pragma unroll
            for (int d = 0; d < 3; ++d) hs[(3 * a + d) * T] = fd.d[d];
            hs[(18 + a) * T] = (P)-0.5 * (gtu[0] * fd.h[0] + gtu[3] * fd.h[3] + gtu[5] * fd.h[5] +
                                          (P)2 * (gtu[1] * fd.h[1] + gtu[2] * fd.h[2] + gtu[4] * fd.h[4]));
            hs[(24 + a) * T] = fd.adv;
            hs[(30 + a) * T] = fd.ko;
        }
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int d = 0; d < 3; ++d) dg[a][d] = hs[(3 * a + d) * T];
    } else if constexpr (Src::UNROLL) {
        // a source that evaluates no stencils has a short loop body: unrolled, in registers
#pragma unroll
        for (int a = 0; a < 6; ++a) {
            FieldDer<P> fd = S.template der<true, EXACT>(GXX + a, beta, w);
#pragma unroll
            for (int d = 0; d < 3; ++d) dg[a][d] = fd.d[d];
            Rt[a] = (P)-0.5 * (gtu[0] * fd.h[0] + gtu[3] * fd.h[3] + gtu[5] * fd.h[5] +
                               (P)2 * (gtu[1] * fd.h[1] + gtu[2] * fd.h[2] + gtu[4] * fd.h[4]));
            agt[a] = fd.adv;
            kgt[a] = fd.ko;
        }
    } else {
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
    if constexpr (Src::HS) {
#pragma unroll
        for (int a = 0; a < 6; ++a) Rt[a] = hs[(18 + a) * (Src::HS ? Src::NT : 1)];
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
    out[CHI] = (((P)(2.0 / 3.0) * chiP * (alpha * K - divb) + fchi.adv) + fchi.ko);
    // gt (ccz4.cpp:586-607)
    if constexpr (Src::HS) {
#pragma unroll
        for (int a = 0; a < 6; ++a) {
            agt[a] = hs[(24 + a) * (Src::HS ? Src::NT : 1)];
            kgt[a] = hs[(30 + a) * (Src::HS ? Src::NT : 1)];
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const int ij = sy(i, j);
            P lie = agt[ij];
#pragma unroll
            for (int d = 0; d < 3; ++d) lie += gt[sy(i, d)] * db[d][j] + gt[sy(j, d)] * db[d][i];
            out[GXX + ij] = (((P)-2 * alpha * At[ij] + lie - (P)(2.0 / 3.0) * gt[ij] * divb) + kgt[ij]);
        }
    // K (ccz4.cpp:650-652)
    {
        FieldDer<P> fK = S.template der<false, EXACT>(KTR, beta, w);
        const P k1 = (P)A.kappa1, k2 = (P)A.kappa2;
        out[KTR] = ((-phys_lap_alpha + alpha * (AtAt + K * K / (P)3) + (P)4 * PI * alpha * (rho + Str) +
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
            out[GHX + i] = ((T1 + T2 + T3 + T4 + T5[i] + T6 + T7 + T8) + kGh[i]);
        }
    }
    // Theta (ccz4.cpp:662-665)
    {
        FieldDer<P> fT = S.template der<false, EXACT>(THETA, beta, w);
        const P k1 = (P)A.kappa1, k2 = (P)A.kappa2;
        out[THETA] = (((P)0.5 * alpha * (Rs - AtAt + (P)2 * K * K / (P)3 - (P)16 * PI * rho) -
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
        for (int a = 0; a < 6; ++a) out[AXX + a] = (raw[a] - (P)(1.0 / 3.0) * gt[a] * tr + koA[a]);
    }
    // lapse (ccz4.cpp:820) and shift (ccz4.cpp:825-831)
    out[ALPHA] = (((P)-2 * alpha * K + fal.adv) + fal.ko);
    {
        const P eta = (P)A.eta;
#pragma unroll
        for (int d = 0; d < 3; ++d) out[BETAX + d] = (((P)0.75 * Gh[d] - eta * (P)beta[d] + abe[d]) + kbe[d]);
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
// The algebra's type of precision mode PM; the RHS values stay in it until the
// epilogue widens them to FP64 (exact), so the FP32 form keeps 22 registers
// instead of 44 for them.
template <int PM>
using AlgebraT = typename std::conditional<PM == PM_MIXED, float, double>::type;

template <int PM, typename Src>
__device__ __forceinline__ void point_pm(const DevBlock& B, const double* __restrict__ u, long long c,
                                         const StageArgs& A, Src& S, AlgebraT<PM> L[NV]) {
    if constexpr (PM == PM_FP64)
        ccz4_point<double, true>(B, u, c, A, S, L);
    else if constexpr (PM == PM_FP64F)
        ccz4_point<double, false>(B, u, c, A, S, L);
    else
        ccz4_point<float, false>(B, u, c, A, S, L);
}

// Shared epilogue: store L, or RK combine + floors (+ algebraic constraints).
// u_in: the stage input at the point, from global memory, or (tin != nullptr)
// from a per-thread column of shared memory that the stencil source filled with
// each field's centre value, field v at tin[v * tin_stride].
// The new state of interior point (i, j, k) into the ghost cells of the
// same-level neighbours that hold it (the tile's npush boxes, slot out_sel);
// the containment test is per point.
__device__ __forceinline__ void push_copies(const PushBox* boxes, int npush, int out_sel, int i, int j, int k,
                                            const double r[NV]) {
    for (int q = 0; q < npush; ++q) {
        const PushBox& P = boxes[q];
        if (i < P.lo[0] || i >= P.hi[0] || j < P.lo[1] || j >= P.hi[1] || k < P.lo[2] || k >= P.hi[2]) continue;
        double* o = P.buf[out_sel] + (P.base + i + (long long)P.tx * j + (long long)P.txy * k);
#pragma unroll
        for (int v = 0; v < NV; ++v) o[(long long)v * P.stride] = r[v];
    }
}

// pushes, npush, (i, j, k): the tile's push boxes (A.push set) and the point's
// interior indices, for the pushed ghost copies.
template <int EPI, typename T>
__device__ __forceinline__ void stage_epilogue(const DevBlock& B, const StageArgs& A, long long c, const T L[NV],
                                               const double* tin = nullptr, int tin_stride = 0,
                                               const PushBox* pushes = nullptr, int npush = 0, int i = 0, int j = 0,
                                               int k = 0) {
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
    if (tin) {
        if (A.in_sel == A.n_sel) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const double unv = tin[v * tin_stride];
                r[v] = rk_combine(A.a1, unv, A.a2, unv, A.a3dt, L[v]);
            }
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v)
                r[v] = rk_combine(A.a1, __ldg(un + (long long)v * st + c), A.a2, tin[v * tin_stride], A.a3dt, L[v]);
        }
    } else if (A.in_sel == A.n_sel) {  // stage 1 reads u^n as both the stage input and u^n: load it once
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
    if (npush > 0) push_copies(pushes, npush, A.out_sel, i, j, k, r);
}

}  // namespace granite_b200
