/*
 * ccz4_oracle.c -- CPU oracle (test infrastructure, see ccz4_oracle.h).
 *
 * Restates GRANITE v0.6.7's CCZ4 hot path in plain C. The floating-point
 * evaluation order of every expression follows the reference so the oracle
 * is bit-identical to the compiled reference under -ffp-contract=off; the
 * code structure (flat indexing, stencil helpers taking a linear offset,
 * lookup tables for the symmetric index) is this project's own.
 *
 * Reference files (paths inside the GRANITE tree):
 *   src/spacetime/ccz4.cpp        RHS, stencils, KO, constraints, flat/gauge-wave data
 *   src/main.cpp                  SSP-RK3 stage sequence, floors, algebraic constraints,
 *                                 1/r outer boundary
 *   src/amr/amr.cpp               zero-gradient ghost fill, prolongation, restriction
 *   src/initial_data/initial_data.cpp   Brill-Lindquist data
 */
#include "ccz4_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum {
    CHI = 0, GXX, GXY, GXZ, GYY, GYZ, GZZ, AXX, AXY, AXZ, AYY, AYZ, AZZ,
    KTR, GHX, GHY, GHZ, THETA, ALPHA, BETAX, BETAY, BETAZ
};

static const double PI_ = 3.14159265358979323846; /* types.hpp:72 */

/* symmetric (a,b) -> packed index, types.hpp:52-54 */
static const int SY[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static inline int tx_(const orc_geom* g) { return g->n[0] + 2 * g->ng; }
static inline int ty_(const orc_geom* g) { return g->n[1] + 2 * g->ng; }
static inline int tz_(const orc_geom* g) { return g->n[2] + 2 * g->ng; }

long orc_stride(const orc_geom* g) { return (long)tx_(g) * ty_(g) * tz_(g); }

/* cell-centre coordinate, grid.hpp:92-94 */
static inline double xc(const orc_geom* g, int d, int idx) {
    return g->lo[d] + ((double)idx - g->ng + 0.5) * g->dx[d];
}

/* ---------------------------------------------------------------------------
 * Stencils. `f` points at the field value of the centre cell; `s` is the
 * linear offset of one cell along the stencil axis.
 * ------------------------------------------------------------------------- */

/* 4th-order centred first derivative, ccz4.cpp:71-99 */
static inline double st_d1(const double* f, long s, double inv12h) {
    return inv12h * (-f[2 * s] + 8.0 * f[s] - 8.0 * f[-s] + f[-2 * s]);
}

/* 4th-order one-sided upwind derivative, side picked by beta >= 0, ccz4.cpp:109-152 */
static inline double st_d1up(const double* f, long s, double beta, double inv12h) {
    if (beta >= 0.0)
        return inv12h *
            (25.0 * f[0] - 48.0 * f[-s] + 36.0 * f[-2 * s] - 16.0 * f[-3 * s] + 3.0 * f[-4 * s]);
    return inv12h *
        (-25.0 * f[0] + 48.0 * f[s] - 36.0 * f[2 * s] + 16.0 * f[3 * s] - 3.0 * f[4 * s]);
}

/* 4th-order same-axis second derivative, ccz4.cpp:156-184 */
static inline double st_d2(const double* f, long s, double inv12h2) {
    return inv12h2 * (-f[2 * s] + 16.0 * f[s] - 30.0 * f[0] + 16.0 * f[-s] - f[-2 * s]);
}

/* 2nd-order mixed derivative, ccz4.cpp:185-222; sa along dir1, sb along dir2 */
static inline double st_dmix(const double* f, long sa, long sb, double inv4hh) {
    return inv4hh * (f[sa + sb] - f[sa - sb] - f[-sa + sb] + f[-sa - sb]);
}

typedef struct {
    long off[3];          /* linear offset of one cell per axis */
    double inv12h[3];     /* 1/(12 dx_d) */
    double inv12h2[3];    /* 1/(12 dx_d^2) */
    double inv4hh[3][3];  /* 1/(4 dx_a dx_b) */
} stencil_geom;

static void make_sg(const orc_geom* g, stencil_geom* sg) {
    sg->off[0] = 1;
    sg->off[1] = tx_(g);
    sg->off[2] = (long)tx_(g) * ty_(g);
    for (int d = 0; d < 3; ++d) {
        sg->inv12h[d] = 1.0 / (12.0 * g->dx[d]);
        sg->inv12h2[d] = 1.0 / (12.0 * g->dx[d] * g->dx[d]);
        for (int e = 0; e < 3; ++e) sg->inv4hh[d][e] = 1.0 / (4.0 * g->dx[d] * g->dx[e]);
    }
}

/* symmetric second-derivative matrix of one field, ccz4.cpp:377-399 */
static void hess(const double* f, const stencil_geom* sg, double out[3][3]) {
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b) {
            double v = (a == b) ? st_d2(f, sg->off[a], sg->inv12h2[a])
                                : st_dmix(f, sg->off[a], sg->off[b], sg->inv4hh[a][b]);
            out[a][b] = v;
            out[b][a] = v;
        }
}

/* inverse conformal metric by cofactors, ccz4.cpp:318-330 */
static void inverse_metric(const double gt[6], double gtu[6]) {
    double det = gt[0] * (gt[3] * gt[5] - gt[4] * gt[4]) - gt[1] * (gt[1] * gt[5] - gt[4] * gt[2]) +
        gt[2] * (gt[1] * gt[4] - gt[3] * gt[2]);
    double inv = 1.0 / (det + 1.0e-30);
    gtu[0] = (gt[3] * gt[5] - gt[4] * gt[4]) * inv;
    gtu[1] = (gt[2] * gt[4] - gt[1] * gt[5]) * inv;
    gtu[2] = (gt[1] * gt[4] - gt[2] * gt[3]) * inv;
    gtu[3] = (gt[0] * gt[5] - gt[2] * gt[2]) * inv;
    gtu[4] = (gt[1] * gt[2] - gt[0] * gt[4]) * inv;
    gtu[5] = (gt[0] * gt[3] - gt[1] * gt[1]) * inv;
}

/* ---------------------------------------------------------------------------
 * Point RHS, ccz4.cpp:251-858
 * ------------------------------------------------------------------------- */
static void rhs_point(const orc_params* p, const stencil_geom* sg, const double* u, long stride,
                      long c, double out[ORC_NV], const double* rho_m, const double* Si_m,
                      const double* Sij_m, const double* S_m) {
#define F(v) (u + (long)(v) * stride + c)
    const double kappa1 = p->kappa1, kappa2 = p->kappa2, eta = p->eta;

    double chi_raw = *F(CHI);
    double chi = (isfinite(chi_raw) && chi_raw >= 1.0e-4) ? chi_raw : 1.0e-4; /* :279-280 */
    double alpha = *F(ALPHA), K = *F(KTR), Theta = *F(THETA);
    double gt[6], At[6], Gh[3], beta[3];
    for (int a = 0; a < 6; ++a) {
        gt[a] = *F(GXX + a);
        At[a] = *F(AXX + a);
    }
    for (int a = 0; a < 3; ++a) {
        Gh[a] = *F(GHX + a);
        beta[a] = *F(BETAX + a);
    }
    double gtu[6];
    inverse_metric(gt, gtu);

    /* first derivatives, :342-369 */
    double d_chi[3], d_alpha[3], d_K[3], d_gt[6][3], d_At[6][3], d_Gh[3][3], d_beta[3][3];
    for (int d = 0; d < 3; ++d) {
        long s = sg->off[d];
        double h = sg->inv12h[d];
        d_chi[d] = st_d1(F(CHI), s, h);
        d_alpha[d] = st_d1(F(ALPHA), s, h);
        d_K[d] = st_d1(F(KTR), s, h);
        for (int a = 0; a < 6; ++a) {
            d_gt[a][d] = st_d1(F(GXX + a), s, h);
            d_At[a][d] = st_d1(F(AXX + a), s, h);
        }
        for (int a = 0; a < 3; ++a) {
            d_Gh[a][d] = st_d1(F(GHX + a), s, h);
            d_beta[a][d] = st_d1(F(BETAX + a), s, h);
        }
    }

    /* second derivatives, :374-399 */
    double dd_chi[3][3], dd_alpha[3][3], dd_gt[6][3][3];
    hess(F(CHI), sg, dd_chi);
    hess(F(ALPHA), sg, dd_alpha);
    for (int a = 0; a < 6; ++a) hess(F(GXX + a), sg, dd_gt[a]);

    /* Christoffels chris[i][jk], :408-444 */
    double chris[3][6];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = j; k < 3; ++k) {
                double val = 0.0;
                for (int l = 0; l < 3; ++l)
                    val += 0.5 * gtu[SY[i][l]] *
                        (d_gt[SY[l][k]][j] + d_gt[SY[l][j]][k] - d_gt[SY[j][k]][l]);
                chris[i][SY[j][k]] = val;
            }

    /* Ricci tensor, :460-543 */
    double Rt[6] = {0}, Rchi[6] = {0};
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            int ij = SY[i][j];
            double R = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) R += -0.5 * gtu[SY[l][m]] * dd_gt[ij][l][m];
            for (int k = 0; k < 3; ++k)
                R += 0.5 * (gt[SY[k][i]] * d_Gh[k][j] + gt[SY[k][j]] * d_Gh[k][i]);
            for (int k = 0; k < 3; ++k) {
                double G = 0.0;
                for (int m = 0; m < 3; ++m) G += gt[SY[k][m]] * chris[m][ij];
                R += Gh[k] * G;
            }
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) {
                    double g_lm = gtu[SY[l][m]];
                    for (int k = 0; k < 3; ++k) {
                        double Gjkm = 0.0, Gikm = 0.0;
                        for (int n = 0; n < 3; ++n) {
                            Gjkm += gt[SY[k][n]] * chris[n][SY[j][m]];
                            Gikm += gt[SY[k][n]] * chris[n][SY[i][m]];
                        }
                        R += g_lm * (chris[k][SY[l][i]] * Gjkm + chris[k][SY[l][j]] * Gikm);
                        double Gkij = 0.0;
                        for (int n = 0; n < 3; ++n) Gkij += gt[SY[k][n]] * chris[n][ij];
                        R -= g_lm * chris[k][SY[l][m]] * Gkij;
                    }
                }
            Rt[ij] = R;

            double DDchi = dd_chi[i][j];
            for (int k = 0; k < 3; ++k) DDchi -= chris[k][ij] * d_chi[k];
            double lap_chi = 0.0, dchi2 = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) {
                    double g_lm = gtu[SY[l][m]];
                    double Dlm = dd_chi[l][m];
                    for (int k = 0; k < 3; ++k) Dlm -= chris[k][SY[l][m]] * d_chi[k];
                    lap_chi += g_lm * Dlm;
                    dchi2 += g_lm * d_chi[l] * d_chi[m];
                }
            double t1 = (0.5 / (chi + 1e-30)) * (DDchi + gt[ij] * lap_chi);
            double t2 = (0.25 / ((chi * chi) + 1e-30)) * (d_chi[i] * d_chi[j] - 3.0 * gt[ij] * dchi2);
            Rchi[ij] = t1 - t2;
        }

    double div_beta = d_beta[0][0] + d_beta[1][1] + d_beta[2][2]; /* :548 */
    double w = 0.5 * (1.0 + tanh((chi - p->chi_blend_center) / p->chi_blend_width)); /* :565 */

    /* blended advection beta^k d_k f of field v given its centred gradient, :567-574 */
#define UPW(v, d) st_d1up(F(v), sg->off[d], beta[d], sg->inv12h[d])
#define ADVEC(v)                                                                              \
    (w * (beta[0] * UPW(v, 0) + beta[1] * UPW(v, 1) + beta[2] * UPW(v, 2)) +                  \
     (1.0 - w) *                                                                              \
         (beta[0] * st_d1(F(v), sg->off[0], sg->inv12h[0]) +                                  \
          beta[1] * st_d1(F(v), sg->off[1], sg->inv12h[1]) +                                  \
          beta[2] * st_d1(F(v), sg->off[2], sg->inv12h[2])))

    double rhs_chi = (2.0 / 3.0) * chi * (alpha * K - div_beta) + ADVEC(CHI); /* :580 */

    double rhs_gt[6]; /* :586-607 */
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            int ij = SY[i][j];
            double up = 0.0, cen = 0.0;
            for (int d = 0; d < 3; ++d) {
                up += beta[d] * UPW(GXX + ij, d);
                cen += beta[d] * d_gt[ij][d];
            }
            double lie = w * up + (1.0 - w) * cen;
            for (int d = 0; d < 3; ++d)
                lie += gt[SY[i][d]] * d_beta[d][j] + gt[SY[j][d]] * d_beta[d][i];
            rhs_gt[ij] = -2.0 * alpha * At[ij] + lie - (2.0 / 3.0) * gt[ij] * div_beta;
        }

    double AtAt = 0.0; /* :609-619 */
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l)
                    AtAt += gtu[SY[i][k]] * gtu[SY[j][l]] * At[SY[i][j]] * At[SY[k][l]];

    double lap_alpha = 0.0; /* :621-632 */
    for (int a = 0; a < 3; ++a)
        for (int b = a; b < 3; ++b) {
            double g_ab = gtu[SY[a][b]];
            double fac = (a == b) ? 1.0 : 2.0;
            lap_alpha += fac * g_ab * dd_alpha[a][b];
            for (int k = 0; k < 3; ++k) lap_alpha -= fac * g_ab * chris[k][SY[a][b]] * d_alpha[k];
        }
    double cga = 0.0; /* :643-646 */
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) cga += gtu[SY[a][b]] * d_chi[a] * d_alpha[b];
    double phys_lap_alpha = chi * lap_alpha - 0.5 * cga;

    const double rho = rho_m ? rho_m[c] : 0.0;
    const double Str = S_m ? S_m[c] : 0.0;
    double rhs_K = -phys_lap_alpha + alpha * (AtAt + K * K / 3.0) +
        4.0 * PI_ * alpha * (rho + Str) + kappa1 * (1.0 - kappa2) * alpha * Theta + ADVEC(KTR);

    double Rs = 0.0; /* :654-660 */
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rs += chi * gtu[SY[i][j]] * (Rt[SY[i][j]] + Rchi[SY[i][j]]);

    double rhs_Theta = 0.5 * alpha * (Rs - AtAt + 2.0 * K * K / 3.0 - 16.0 * PI_ * rho) -
        alpha * kappa1 * (2.0 + kappa2) * Theta + ADVEC(THETA); /* :662-665 */

    double raw[6]; /* :671-726 */
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            int ij = SY[i][j];
            double DDa = dd_alpha[i][j];
            for (int k = 0; k < 3; ++k) DDa -= chris[k][ij] * d_alpha[k];
            double Sij = Sij_m ? Sij_m[6 * c + ij] : 0.0;
            double Rij = Rt[ij] + Rchi[ij];
            double t1 = chi * (-DDa + alpha * (Rij - 8.0 * PI_ * Sij));
            double Asq = 0.0;
            for (int k = 0; k < 3; ++k) {
                double Au = 0.0;
                for (int l = 0; l < 3; ++l) Au += gtu[SY[k][l]] * At[SY[l][j]];
                Asq += At[SY[i][k]] * Au;
            }
            double t2 = alpha * (K * At[ij] - 2.0 * Asq);
            double up = 0.0, cen = 0.0;
            for (int d = 0; d < 3; ++d) {
                up += beta[d] * UPW(AXX + ij, d);
                cen += beta[d] * d_At[ij][d];
            }
            double lie = w * up + (1.0 - w) * cen;
            for (int d = 0; d < 3; ++d)
                lie += At[SY[i][d]] * d_beta[d][j] + At[SY[j][d]] * d_beta[d][i];
            lie -= (2.0 / 3.0) * At[ij] * div_beta;
            raw[ij] = t1 + t2 + lie;
        }
    double trA = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) trA += gtu[SY[i][j]] * raw[SY[i][j]];
    double rhs_At[6];
    for (int a = 0; a < 6; ++a) rhs_At[a] = raw[a] - (1.0 / 3.0) * gt[a] * trA;

    double dd_beta[3][3][3]; /* :733-745 */
    for (int a = 0; a < 3; ++a) hess(F(BETAX + a), sg, dd_beta[a]);

    double rhs_Gh[3]; /* :747-815 */
    for (int i = 0; i < 3; ++i) {
        double T1 = 0.0;
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) T1 += chris[i][SY[j][k]] * At[SY[j][k]];
        T1 *= 2.0 * alpha;
        double T2 = 0.0;
        for (int j = 0; j < 3; ++j) T2 += gtu[SY[i][j]] * d_K[j];
        T2 *= -(4.0 / 3.0) * alpha;
        double T3 = 0.0;
        for (int j = 0; j < 3; ++j) T3 += gtu[SY[i][j]] * (Si_m ? Si_m[3 * c + j] : 0.0);
        T3 *= -16.0 * PI_ * alpha;
        double T4 = 0.0;
        for (int j = 0; j < 3; ++j) {
            double Au = 0.0;
            for (int k = 0; k < 3; ++k) Au += gtu[SY[i][k]] * At[SY[k][j]];
            T4 += Au * d_chi[j];
        }
        T4 *= 3.0 * alpha / (chi + 1e-30);
        double T5 = 0.0;
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) T5 += gtu[SY[j][k]] * dd_beta[i][j][k];
        double T6 = 0.0;
        for (int j = 0; j < 3; ++j) {
            double ddiv = 0.0;
            for (int k = 0; k < 3; ++k) ddiv += dd_beta[k][k][j];
            T6 += gtu[SY[i][j]] * ddiv;
        }
        T6 *= (1.0 / 3.0);
        double T7 = 0.0;
        for (int j = 0; j < 3; ++j) T7 -= Gh[j] * d_beta[i][j];
        double up = 0.0, cen = 0.0;
        for (int j = 0; j < 3; ++j) {
            up += beta[j] * UPW(GHX + i, j);
            cen += beta[j] * d_Gh[i][j];
        }
        T7 += w * up + (1.0 - w) * cen;
        T7 += (2.0 / 3.0) * Gh[i] * div_beta;
        double T8 = -2.0 * kappa1 * alpha * Gh[i];
        rhs_Gh[i] = T1 + T2 + T3 + T4 + T5 + T6 + T7 + T8;
    }

    double rhs_alpha = -2.0 * alpha * K + ADVEC(ALPHA); /* :820 */
    double rhs_beta[3];
    for (int d = 0; d < 3; ++d) rhs_beta[d] = 0.75 * Gh[d] - eta * beta[d] + ADVEC(BETAX + d);

    out[CHI] = rhs_chi;
    for (int a = 0; a < 6; ++a) {
        out[GXX + a] = rhs_gt[a];
        out[AXX + a] = rhs_At[a];
    }
    out[KTR] = rhs_K;
    for (int a = 0; a < 3; ++a) {
        out[GHX + a] = rhs_Gh[a];
        out[BETAX + a] = rhs_beta[a];
    }
    out[THETA] = rhs_Theta;
    out[ALPHA] = rhs_alpha;
#undef ADVEC
#undef UPW
#undef F
}

void orc_rhs(const orc_params* p, const orc_geom* g, const double* u, double* rhs,
             const double* rho, const double* Si, const double* Sij, const double* S) {
    stencil_geom sg;
    make_sg(g, &sg);
    const long stride = orc_stride(g);
    const int ng = g->ng, tx = tx_(g), ty = ty_(g);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng; k < ng + g->n[2]; ++k)
        for (int j = ng; j < ng + g->n[1]; ++j)
            for (int i = ng; i < ng + g->n[0]; ++i) {
                long c = i + (long)tx * (j + (long)ty * k);
                double out[ORC_NV];
                rhs_point(p, &sg, u, stride, c, out, rho, Si, Sij, S);
                for (int v = 0; v < ORC_NV; ++v) rhs[(long)v * stride + c] = out[v];
            }
    orc_dissipation(p, g, u, rhs);
}

/* KO dissipation, ccz4.cpp:871-935 */
void orc_dissipation(const orc_params* p, const orc_geom* g, const double* u, double* rhs) {
    const double sigma = p->ko_sigma;
    if (sigma <= 0.0) return;
    static const double wts[7] = {1.0, -6.0, 15.0, -20.0, 15.0, -6.0, 1.0};
    const double cf[3] = {sigma / (64.0 * g->dx[0]), sigma / (64.0 * g->dx[1]),
                          sigma / (64.0 * g->dx[2])};
    const long stride = orc_stride(g);
    const int ng = g->ng, tx = tx_(g), ty = ty_(g);
    const long off[3] = {1, tx, (long)tx * ty};
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng; k < ng + g->n[2]; ++k)
        for (int j = ng; j < ng + g->n[1]; ++j)
            for (int i = ng; i < ng + g->n[0]; ++i) {
                long c = i + (long)tx * (j + (long)ty * k);
                double diss[ORC_NV] = {0};
                for (int d = 0; d < 3; ++d)
                    for (int s = 0; s < 7; ++s) {
                        double wt = cf[d] * wts[s];
                        long cs = c + (long)(s - 3) * off[d];
                        for (int v = 0; v < ORC_NV; ++v) diss[v] += wt * u[(long)v * stride + cs];
                    }
                for (int v = 0; v < ORC_NV; ++v) rhs[(long)v * stride + c] += diss[v];
            }
}

/* ---------------------------------------------------------------------------
 * Constraints, ccz4.cpp:941-1159
 * ------------------------------------------------------------------------- */
static void constraint_point(const stencil_geom* sg, const double* u, long stride, long c,
                             double* H, double M[3]) {
#define F(v) (u + (long)(v) * stride + c)
    double chi = *F(CHI); /* not clamped here, :963 */
    double K = *F(KTR);
    double gt[6], At[6], gtu[6];
    for (int a = 0; a < 6; ++a) {
        gt[a] = *F(GXX + a);
        At[a] = *F(AXX + a);
    }
    inverse_metric(gt, gtu);

    double AtAt = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l)
                    AtAt += gtu[SY[i][k]] * gtu[SY[j][l]] * At[SY[i][j]] * At[SY[k][l]];

    double d_gt[6][3], dd_gt[6][3][3], d_chi[3], dd_chi[3][3];
    for (int a = 0; a < 6; ++a)
        for (int d = 0; d < 3; ++d) {
            d_gt[a][d] = st_d1(F(GXX + a), sg->off[d], sg->inv12h[d]);
            for (int e = d; e < 3; ++e) {
                double v = (d == e) ? st_d2(F(GXX + a), sg->off[d], sg->inv12h2[d])
                                    : st_dmix(F(GXX + a), sg->off[d], sg->off[e], sg->inv4hh[d][e]);
                dd_gt[a][d][e] = v;
                dd_gt[a][e][d] = v;
            }
        }
    for (int d = 0; d < 3; ++d) d_chi[d] = st_d1(F(CHI), sg->off[d], sg->inv12h[d]);
    hess(F(CHI), sg, dd_chi);

    double chris[3][6];
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i)
            for (int j = i; j < 3; ++j) {
                double sum = 0.0;
                for (int m = 0; m < 3; ++m)
                    sum += 0.5 * gtu[SY[k][m]] *
                        (d_gt[SY[m][i]][j] + d_gt[SY[m][j]][i] - d_gt[SY[i][j]][m]);
                chris[k][SY[i][j]] = sum;
            }

    double Gh[3], d_Gh[3][3];
    for (int a = 0; a < 3; ++a) Gh[a] = *F(GHX + a);
    for (int d = 0; d < 3; ++d)
        for (int a = 0; a < 3; ++a) d_Gh[a][d] = st_d1(F(GHX + a), sg->off[d], sg->inv12h[d]);

    double Rt[6] = {0}, Rchi[6] = {0};
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            int ij = SY[i][j];
            double R = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) R += -0.5 * gtu[SY[l][m]] * dd_gt[ij][l][m];
            for (int k = 0; k < 3; ++k) {
                R += 0.5 * (gt[SY[k][i]] * d_Gh[k][j] + gt[SY[k][j]] * d_Gh[k][i]);
                double G = 0.0;
                for (int m = 0; m < 3; ++m) G += gt[SY[k][m]] * chris[m][ij];
                R += Gh[k] * G;
            }
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) {
                    double g_lm = gtu[SY[l][m]];
                    for (int k = 0; k < 3; ++k) {
                        double Gjkm = 0.0, Gikm = 0.0, Gkij = 0.0;
                        for (int n = 0; n < 3; ++n) {
                            Gjkm += gt[SY[k][n]] * chris[n][SY[j][m]];
                            Gikm += gt[SY[k][n]] * chris[n][SY[i][m]];
                            Gkij += gt[SY[k][n]] * chris[n][ij];
                        }
                        R += g_lm * (chris[k][SY[l][i]] * Gjkm + chris[k][SY[l][j]] * Gikm);
                        R -= g_lm * chris[k][SY[l][m]] * Gkij;
                    }
                }
            Rt[ij] = R;
            double DDchi = dd_chi[i][j];
            for (int k = 0; k < 3; ++k) DDchi -= chris[k][ij] * d_chi[k];
            double lap_chi = 0.0, dchi2 = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) {
                    double g_lm = gtu[SY[l][m]];
                    double Dlm = dd_chi[l][m];
                    for (int k = 0; k < 3; ++k) Dlm -= chris[k][SY[l][m]] * d_chi[k];
                    lap_chi += g_lm * Dlm;
                    dchi2 += g_lm * d_chi[l] * d_chi[m];
                }
            Rchi[ij] = (0.5 / (chi + 1e-30)) * (DDchi + gt[ij] * lap_chi) -
                (0.25 / ((chi * chi) + 1e-30)) * (d_chi[i] * d_chi[j] - 3.0 * gt[ij] * dchi2);
        }

    double Rs = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rs += gtu[SY[i][j]] * (Rt[SY[i][j]] + Rchi[SY[i][j]]);
    Rs *= chi;
    const double rho = 0.0;
    *H = Rs + (2.0 / 3.0) * K * K - AtAt - 16.0 * PI_ * rho; /* :1127 */

    double d_At[6][3], d_K[3];
    for (int a = 0; a < 6; ++a)
        for (int d = 0; d < 3; ++d) d_At[a][d] = st_d1(F(AXX + a), sg->off[d], sg->inv12h[d]);
    for (int d = 0; d < 3; ++d) d_K[d] = st_d1(F(KTR), sg->off[d], sg->inv12h[d]);

    for (int i = 0; i < 3; ++i) { /* :1138-1155 */
        double Mi = 0.0;
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                double g_jk = gtu[SY[j][k]];
                double DA = d_At[SY[k][i]][j];
                for (int m = 0; m < 3; ++m)
                    DA -= chris[m][SY[j][k]] * At[SY[m][i]] + chris[m][SY[j][i]] * At[SY[k][m]];
                Mi += g_jk * DA;
                Mi -= (3.0 / (2.0 * chi + 1e-30)) * At[SY[i][j]] * g_jk * d_chi[k];
            }
        Mi -= (2.0 / 3.0) * d_K[i];
        M[i] = Mi;
    }
#undef F
}

void orc_constraints(const orc_geom* g, const double* u, double* ham, double* mom) {
    stencil_geom sg;
    make_sg(g, &sg);
    const long stride = orc_stride(g);
    memset(ham, 0, sizeof(double) * stride);
    memset(mom, 0, sizeof(double) * 3 * stride);
    const int ng = g->ng, tx = tx_(g), ty = ty_(g);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ng; k < ng + g->n[2]; ++k)
        for (int j = ng; j < ng + g->n[1]; ++j)
            for (int i = ng; i < ng + g->n[0]; ++i) {
                long c = i + (long)tx * (j + (long)ty * k);
                constraint_point(&sg, u, stride, c, ham + c, mom + 3 * c);
            }
}

void orc_constraint_sums(const orc_geom* g, const double* u, double* h2, double* m2,
                         long* npts) {
    const long stride = orc_stride(g);
    double* ham = (double*)malloc(sizeof(double) * stride);
    double* mom = (double*)malloc(sizeof(double) * 3 * stride);
    orc_constraints(g, u, ham, mom);
    const int ng = g->ng, tx = tx_(g), ty = ty_(g);
    double sh = 0.0, sm = 0.0;
    long n = 0;
    for (int k = ng; k < ng + g->n[2]; ++k)
        for (int j = ng; j < ng + g->n[1]; ++j)
            for (int i = ng; i < ng + g->n[0]; ++i) {
                long c = i + (long)tx * (j + (long)ty * k);
                sh += ham[c] * ham[c];
                sm += mom[3 * c] * mom[3 * c] + mom[3 * c + 1] * mom[3 * c + 1] +
                    mom[3 * c + 2] * mom[3 * c + 2];
                ++n;
            }
    *h2 = sh;
    *m2 = sm;
    *npts = n;
    free(ham);
    free(mom);
}

/* ---------------------------------------------------------------------------
 * Ghost fills
 * ------------------------------------------------------------------------- */

/* zero-gradient copy on every face, x then y then z, amr.cpp:447-480 */
void orc_fill_zero_gradient(const orc_geom* g, double* u) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const long stride = orc_stride(g);
    const int ie[3] = {ng + g->n[0], ng + g->n[1], ng + g->n[2]};
    for (int v = 0; v < ORC_NV; ++v) {
        double* f = u + (long)v * stride;
#define A(i, j, k) f[(i) + (long)tx * ((j) + (long)ty * (k))]
        for (int k = 0; k < tz; ++k)
            for (int j = 0; j < ty; ++j)
                for (int q = 0; q < ng; ++q) {
                    A(q, j, k) = A(ng, j, k);
                    A(ie[0] + q, j, k) = A(ie[0] - 1, j, k);
                }
        for (int k = 0; k < tz; ++k)
            for (int i = 0; i < tx; ++i)
                for (int q = 0; q < ng; ++q) {
                    A(i, q, k) = A(i, ng, k);
                    A(i, ie[1] + q, k) = A(i, ie[1] - 1, k);
                }
        for (int j = 0; j < ty; ++j)
            for (int i = 0; i < tx; ++i)
                for (int q = 0; q < ng; ++q) {
                    A(i, j, q) = A(i, j, ng);
                    A(i, j, ie[2] + q) = A(i, j, ie[2] - 1);
                }
#undef A
    }
}

/* periodic wrap on every face (no reference counterpart: the gauge-wave
 * configuration needs it, the reference has no periodic boundary) */
void orc_fill_periodic(const orc_geom* g, double* u) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const long stride = orc_stride(g);
    for (int v = 0; v < ORC_NV; ++v) {
        double* f = u + (long)v * stride;
        for (int k = 0; k < tz; ++k)
            for (int j = 0; j < ty; ++j)
                for (int i = 0; i < tx; ++i) {
                    int ii = i, jj = j, kk = k;
                    if (ii < ng) ii += g->n[0];
                    else if (ii >= ng + g->n[0]) ii -= g->n[0];
                    if (jj < ng) jj += g->n[1];
                    else if (jj >= ng + g->n[1]) jj -= g->n[1];
                    if (kk < ng) kk += g->n[2];
                    else if (kk >= ng + g->n[2]) kk -= g->n[2];
                    if (ii != i || jj != j || kk != k)
                        f[i + (long)tx * (j + (long)ty * k)] =
                            f[ii + (long)tx * (jj + (long)ty * kk)];
                }
    }
}

/* asymptotic values of the 1/r falloff, main.cpp:382-394 */
static inline double f_inf(int v) {
    return (v == CHI || v == GXX || v == GYY || v == GZZ || v == ALPHA) ? 1.0 : 0.0;
}

/* 1/r "Sommerfeld" falloff from the outermost interior layer: x faces over all
 * (j,k), then y faces over all (i,k), then z faces over all (i,j), main.cpp:351-463 */
void orc_fill_sommerfeld(const orc_geom* g, double* u) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const long stride = orc_stride(g);
    const int is = ng;
    const int ie[3] = {tx - ng - 1, ty - ng - 1, tz - ng - 1};
    for (int v = 0; v < ORC_NV; ++v) {
        const double fi = f_inf(v);
        double* f = u + (long)v * stride;
#define A(i, j, k) f[(i) + (long)tx * ((j) + (long)ty * (k))]
        for (int k = 0; k < tz; ++k)
            for (int j = 0; j < ty; ++j) {
                double y = xc(g, 1, j), z = xc(g, 2, k);
                for (int q = 0; q < ng; ++q) {
                    double xi = xc(g, 0, is), xg = xc(g, 0, is - 1 - q);
                    double ri = sqrt(xi * xi + y * y + z * z) + 1e-30;
                    double rg = sqrt(xg * xg + y * y + z * z) + 1e-30;
                    A(is - 1 - q, j, k) = fi + (A(is, j, k) - fi) * ri / rg;
                    xi = xc(g, 0, ie[0]);
                    xg = xc(g, 0, ie[0] + 1 + q);
                    ri = sqrt(xi * xi + y * y + z * z) + 1e-30;
                    rg = sqrt(xg * xg + y * y + z * z) + 1e-30;
                    A(ie[0] + 1 + q, j, k) = fi + (A(ie[0], j, k) - fi) * ri / rg;
                }
            }
        for (int k = 0; k < tz; ++k)
            for (int i = 0; i < tx; ++i) {
                double x = xc(g, 0, i), z = xc(g, 2, k);
                for (int q = 0; q < ng; ++q) {
                    double yi = xc(g, 1, is), yg = xc(g, 1, is - 1 - q);
                    double ri = sqrt(x * x + yi * yi + z * z) + 1e-30;
                    double rg = sqrt(x * x + yg * yg + z * z) + 1e-30;
                    A(i, is - 1 - q, k) = fi + (A(i, is, k) - fi) * ri / rg;
                    yi = xc(g, 1, ie[1]);
                    yg = xc(g, 1, ie[1] + 1 + q);
                    ri = sqrt(x * x + yi * yi + z * z) + 1e-30;
                    rg = sqrt(x * x + yg * yg + z * z) + 1e-30;
                    A(i, ie[1] + 1 + q, k) = fi + (A(i, ie[1], k) - fi) * ri / rg;
                }
            }
        for (int j = 0; j < ty; ++j)
            for (int i = 0; i < tx; ++i) {
                double x = xc(g, 0, i), y = xc(g, 1, j);
                for (int q = 0; q < ng; ++q) {
                    double zi = xc(g, 2, is), zg = xc(g, 2, is - 1 - q);
                    double ri = sqrt(x * x + y * y + zi * zi) + 1e-30;
                    double rg = sqrt(x * x + y * y + zg * zg) + 1e-30;
                    A(i, j, is - 1 - q) = fi + (A(i, j, is) - fi) * ri / rg;
                    zi = xc(g, 2, ie[2]);
                    zg = xc(g, 2, ie[2] + 1 + q);
                    ri = sqrt(x * x + y * y + zi * zi) + 1e-30;
                    rg = sqrt(x * x + y * y + zg * zg) + 1e-30;
                    A(i, j, ie[2] + 1 + q) = fi + (A(i, j, ie[2]) - fi) * ri / rg;
                }
            }
#undef A
    }
}

/* chi in [1e-4, 1.5] (non-finite -> 1e-4), alpha >= 1e-6 (non-finite -> 1e-6)
 * over all cells, main.cpp:588-608 */
void orc_floors(const orc_geom* g, double* u) {
    const long stride = orc_stride(g);
    double* chi = u + (long)CHI * stride;
    double* alpha = u + (long)ALPHA * stride;
    for (long c = 0; c < stride; ++c) {
        if (!isfinite(chi[c]) || chi[c] < 1.0e-4) chi[c] = 1.0e-4;
        if (chi[c] > 1.5) chi[c] = 1.5;
        if (!isfinite(alpha[c]) || alpha[c] < 1.0e-6) alpha[c] = 1.0e-6;
    }
}

/* det(gt) = 1 by cbrt rescale (reset to identity when det <= 1e-10 or
 * non-finite), then remove the trace of At, all cells, main.cpp:612-671 */
void orc_algebraic(const orc_geom* g, double* u) {
    const long stride = orc_stride(g);
    for (long c = 0; c < stride; ++c) {
        double* G[6];
        double* Ap[6];
        for (int a = 0; a < 6; ++a) {
            G[a] = u + (long)(GXX + a) * stride + c;
            Ap[a] = u + (long)(AXX + a) * stride + c;
        }
        double gxx = *G[0], gxy = *G[1], gxz = *G[2], gyy = *G[3], gyz = *G[4], gzz = *G[5];
        double det = gxx * (gyy * gzz - gyz * gyz) - gxy * (gxy * gzz - gyz * gxz) +
            gxz * (gxy * gyz - gyy * gxz);
        if (isfinite(det) && det > 1.0e-10) {
            double s = cbrt(1.0 / det);
            gxx *= s; gxy *= s; gxz *= s; gyy *= s; gyz *= s; gzz *= s;
        } else {
            gxx = 1.0; gxy = 0.0; gxz = 0.0; gyy = 1.0; gyz = 0.0; gzz = 1.0;
        }
        *G[0] = gxx; *G[1] = gxy; *G[2] = gxz; *G[3] = gyy; *G[4] = gyz; *G[5] = gzz;
        const double ixx = gyy * gzz - gyz * gyz;
        const double ixy = gxz * gyz - gxy * gzz;
        const double ixz = gxy * gyz - gxz * gyy;
        const double iyy = gxx * gzz - gxz * gxz;
        const double iyz = gxz * gxy - gxx * gyz;
        const double izz = gxx * gyy - gxy * gxy;
        double axx = *Ap[0], axy = *Ap[1], axz = *Ap[2], ayy = *Ap[3], ayz = *Ap[4], azz = *Ap[5];
        const double trA = ixx * axx + iyy * ayy + izz * azz + 2.0 * (ixy * axy + ixz * axz + iyz * ayz);
        const double t3 = trA / 3.0;
        *Ap[0] = axx - t3 * gxx;
        *Ap[1] = axy - t3 * gxy;
        *Ap[2] = axz - t3 * gxz;
        *Ap[3] = ayy - t3 * gyy;
        *Ap[4] = ayz - t3 * gyz;
        *Ap[5] = azz - t3 * gzz;
    }
}

/* d = a1 s1 + a2 s2 + a3 dt r at interior points, main.cpp:306-335 */
static void combine(const orc_geom* g, double* d, const double* s1, double a1, const double* s2,
                    double a2, const double* r, double a3, double dt) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g);
    const long stride = orc_stride(g);
    for (int v = 0; v < ORC_NV; ++v)
        for (int k = ng; k < ng + g->n[2]; ++k)
            for (int j = ng; j < ng + g->n[1]; ++j)
                for (int i = ng; i < ng + g->n[0]; ++i) {
                    long c = (long)v * stride + i + (long)tx * (j + (long)ty * k);
                    d[c] = a1 * s1[c] + a2 * s2[c] + a3 * dt * r[c];
                }
}

static void outer_bc(const orc_geom* g, double* u, int bc) {
    if (bc == ORC_BC_PERIODIC) orc_fill_periodic(g, u);
    else orc_fill_sommerfeld(g, u);
}
static void level_fill(const orc_geom* g, double* u, int bc) {
    if (bc == ORC_BC_PERIODIC) orc_fill_periodic(g, u);
    else orc_fill_zero_gradient(g, u);
}

/* One level-0 step of AMRHierarchy::subcycle (amr.cpp:303-330) around
 * TimeIntegrator::sspRK3Step's spacetime part (main.cpp:673-689). */
void orc_rk3_step(const orc_params* p, const orc_geom* g, double* u, double* stage,
                  double* rhs, double dt, int bc) {
    orc_rk3_step_matter(p, g, u, stage, rhs, dt, bc, NULL, NULL, NULL, NULL);
}

/* The same step with matter sources held fixed over its three RHS evaluations
 * (main.cpp:296-302 with the primitives unchanged between stages). */
void orc_rk3_step_matter(const orc_params* p, const orc_geom* g, double* u, double* stage, double* rhs,
                         double dt, int bc, const double* rho, const double* Si, const double* Sij,
                         const double* S) {
    level_fill(g, u, bc);
    orc_rhs(p, g, u, rhs, rho, Si, Sij, S);
    combine(g, stage, u, 1.0, u, 0.0, rhs, 1.0, dt);
    orc_floors(g, stage);
    outer_bc(g, stage, bc);

    orc_rhs(p, g, stage, rhs, rho, Si, Sij, S);
    combine(g, stage, u, 0.75, stage, 0.25, rhs, 0.25, dt);
    orc_floors(g, stage);
    outer_bc(g, stage, bc);

    orc_rhs(p, g, stage, rhs, rho, Si, Sij, S);
    combine(g, u, u, 1.0 / 3.0, stage, 2.0 / 3.0, rhs, 2.0 / 3.0, dt);
    orc_floors(g, u);
    orc_algebraic(g, u);
    outer_bc(g, u, bc);
    level_fill(g, u, bc);
}

/* ---------------------------------------------------------------------------
 * Initial data
 * ------------------------------------------------------------------------- */

/* ccz4.cpp:1165-1188 (other fields left as they are, zero in a fresh block) */
void orc_init_flat(const orc_geom* g, double* u) {
    const long stride = orc_stride(g);
    for (long c = 0; c < stride; ++c) {
        u[(long)CHI * stride + c] = 1.0;
        u[(long)GXX * stride + c] = 1.0;
        u[(long)GXY * stride + c] = 0.0;
        u[(long)GXZ * stride + c] = 0.0;
        u[(long)GYY * stride + c] = 1.0;
        u[(long)GYZ * stride + c] = 0.0;
        u[(long)GZZ * stride + c] = 1.0;
        u[(long)ALPHA * stride + c] = 1.0;
    }
}

/* ccz4.cpp:1190-1221; amplitude < 0 gives the g_xx = 1 - |A| sin variant */
void orc_init_gauge_wave(const orc_geom* g, double* u, double amplitude, double wavelength) {
    const int tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const long stride = orc_stride(g);
    for (int k = 0; k < tz; ++k)
        for (int j = 0; j < ty; ++j)
            for (int i = 0; i < tx; ++i) {
                long c = i + (long)tx * (j + (long)ty * k);
                double x = xc(g, 0, i);
                double H = amplitude * sin(2.0 * PI_ * x / wavelength);
                double detg = (1.0 + H);
                double chi = pow(detg, -1.0 / 3.0);
                u[(long)CHI * stride + c] = chi;
                u[(long)GXX * stride + c] = (1.0 + H) * chi;
                u[(long)GXY * stride + c] = 0.0;
                u[(long)GXZ * stride + c] = 0.0;
                u[(long)GYY * stride + c] = chi;
                u[(long)GYZ * stride + c] = 0.0;
                u[(long)GZZ * stride + c] = chi;
                u[(long)ALPHA * stride + c] = sqrt(1.0 + H);
            }
}

/* initial_data.cpp:79-89, with an optional floor on r (0 = none) */
double orc_bl_conformal_factor(int nbh, const double* mass, const double* pos, double x,
                               double y, double z, double r_floor) {
    double psi = 1.0;
    for (int b = 0; b < nbh; ++b) {
        double dx = x - pos[3 * b], dy = y - pos[3 * b + 1], dz = z - pos[3 * b + 2];
        double r = sqrt(dx * dx + dy * dy + dz * dz + 1.0e-30);
        if (r < r_floor) r = r_floor;
        psi += mass[b] / (2.0 * r);
    }
    return psi;
}

/* initial_data.cpp:97-158 */
void orc_init_brill_lindquist(const orc_geom* g, double* u, int nbh, const double* mass,
                              const double* pos, double r_floor) {
    const long stride = orc_stride(g);
    memset(u, 0, sizeof(double) * ORC_NV * stride);
    orc_init_flat(g, u);
    const int tx = tx_(g), ty = ty_(g), tz = tz_(g);
    for (int k = 0; k < tz; ++k)
        for (int j = 0; j < ty; ++j)
            for (int i = 0; i < tx; ++i) {
                long c = i + (long)tx * (j + (long)ty * k);
                const double x = xc(g, 0, i), y = xc(g, 1, j), z = xc(g, 2, k);
                const double psi = orc_bl_conformal_factor(nbh, mass, pos, x, y, z, r_floor);
                const double psi2 = psi * psi;
                const double chi = 1.0 / (psi2 * psi2);
                u[(long)CHI * stride + c] = chi;
                u[(long)ALPHA * stride + c] = sqrt(chi);
                double dpx = 0.0, dpy = 0.0, dpz = 0.0;
                for (int b = 0; b < nbh; ++b) {
                    const double rx = x - pos[3 * b], ry = y - pos[3 * b + 1], rz = z - pos[3 * b + 2];
                    double r2 = rx * rx + ry * ry + rz * rz + 1.0e-20;
                    if (r2 < r_floor * r_floor) r2 = r_floor * r_floor;
                    const double r3 = r2 * sqrt(r2);
                    const double cc = -mass[b] / (2.0 * r3);
                    dpx += cc * rx;
                    dpy += cc * ry;
                    dpz += cc * rz;
                }
                const double gf = 8.0 / (3.0 * psi);
                u[(long)GHX * stride + c] = gf * dpx;
                u[(long)GHY * stride + c] = gf * dpy;
                u[(long)GHZ * stride + c] = gf * dpz;
            }
}

/* ---------------------------------------------------------------------------
 * AMR inter-level operators
 * ------------------------------------------------------------------------- */

/* trilinear prolongation, nearest coarse centre + one-sided neighbour chosen
 * by the sign of the fractional offset, indices clamped to the coarse block,
 * amr.cpp:484-564. ghosts_only != 0 restricts the writes to fine ghost cells. */
void orc_prolongate(const orc_geom* cg, const double* uc, const orc_geom* fg, double* uf,
                    int ghosts_only) {
    const int ftx = tx_(fg), fty = ty_(fg), ftz = tz_(fg);
    const int ctx = tx_(cg), cty = ty_(cg), ctz = tz_(cg);
    const long fs = orc_stride(fg), cs = orc_stride(cg);
    const int cis = cg->ng;
    const int ct[3] = {ctx, cty, ctz};
    for (int v = 0; v < ORC_NV; ++v) {
        const double* C = uc + (long)v * cs;
        double* Fo = uf + (long)v * fs;
        for (int k = 0; k < ftz; ++k)
            for (int j = 0; j < fty; ++j)
                for (int i = 0; i < ftx; ++i) {
                    if (ghosts_only && i >= fg->ng && i < fg->ng + fg->n[0] && j >= fg->ng &&
                        j < fg->ng + fg->n[1] && k >= fg->ng && k < fg->ng + fg->n[2])
                        continue;
                    const double X[3] = {xc(fg, 0, i), xc(fg, 1, j), xc(fg, 2, k)};
                    double fr[3];
                    int ci[3], cn[3];
                    for (int d = 0; d < 3; ++d) {
                        double f = (X[d] - xc(cg, d, cis)) / cg->dx[d] + cis;
                        int c0 = (int)round(f);
                        if (c0 > ct[d] - 1) c0 = ct[d] - 1;
                        if (c0 < 0) c0 = 0;
                        fr[d] = f - (double)c0;
                        int c1 = c0 + (fr[d] >= 0.0 ? 1 : -1);
                        if (c1 > ct[d] - 1) c1 = ct[d] - 1;
                        if (c1 < 0) c1 = 0;
                        ci[d] = c0;
                        cn[d] = c1;
                    }
                    const double ax = fabs(fr[0]), ay = fabs(fr[1]), az = fabs(fr[2]);
                    const double w000 = (1 - ax) * (1 - ay) * (1 - az);
                    const double w100 = ax * (1 - ay) * (1 - az);
                    const double w010 = (1 - ax) * ay * (1 - az);
                    const double w001 = (1 - ax) * (1 - ay) * az;
                    const double w110 = ax * ay * (1 - az);
                    const double w101 = ax * (1 - ay) * az;
                    const double w011 = (1 - ax) * ay * az;
                    const double w111 = ax * ay * az;
#define CV(a, b, c) C[(a) + (long)ctx * ((b) + (long)cty * (c))]
                    Fo[i + (long)ftx * (j + (long)fty * k)] = w000 * CV(ci[0], ci[1], ci[2]) +
                        w100 * CV(cn[0], ci[1], ci[2]) + w010 * CV(ci[0], cn[1], ci[2]) +
                        w001 * CV(ci[0], ci[1], cn[2]) + w110 * CV(cn[0], cn[1], ci[2]) +
                        w101 * CV(cn[0], ci[1], cn[2]) + w011 * CV(ci[0], cn[1], cn[2]) +
                        w111 * CV(cn[0], cn[1], cn[2]);
#undef CV
                }
    }
}

/* 2x2x2 mean of fine cells around each coarse centre whose stencil lies in
 * [istart, iend + ng) of the fine block, amr.cpp:566-626 (ratio 2) */
void orc_restrict(const orc_geom* fg, const double* uf, const orc_geom* cg, double* uc) {
    const int ratio = 2;
    const int ftx = tx_(fg), fty = ty_(fg);
    const int ctx = tx_(cg), cty = ty_(cg);
    const long fs = orc_stride(fg), cs = orc_stride(cg);
    const int fis = fg->ng;
    const int fie[3] = {fg->ng + fg->n[0], fg->ng + fg->n[1], fg->ng + fg->n[2]};
    for (int v = 0; v < ORC_NV; ++v) {
        const double* Fv = uf + (long)v * fs;
        double* Cv = uc + (long)v * cs;
        for (int ck = cg->ng; ck < cg->ng + cg->n[2]; ++ck)
            for (int cj = cg->ng; cj < cg->ng + cg->n[1]; ++cj)
                for (int ci = cg->ng; ci < cg->ng + cg->n[0]; ++ci) {
                    const double x = xc(cg, 0, ci), y = xc(cg, 1, cj), z = xc(cg, 2, ck);
                    const double fx = (x - xc(fg, 0, 0)) / fg->dx[0];
                    const double fy = (y - xc(fg, 1, 0)) / fg->dx[1];
                    const double fz = (z - xc(fg, 2, 0)) / fg->dx[2];
                    const int fi = (int)round(fx) - ratio / 2;
                    const int fj = (int)round(fy) - ratio / 2;
                    const int fk = (int)round(fz) - ratio / 2;
                    if (fi >= fis && fi + ratio <= fie[0] + fg->ng && fj >= fis &&
                        fj + ratio <= fie[1] + fg->ng && fk >= fis && fk + ratio <= fie[2] + fg->ng) {
                        double sum = 0.0;
                        for (int rk = 0; rk < ratio; ++rk)
                            for (int rj = 0; rj < ratio; ++rj)
                                for (int ri = 0; ri < ratio; ++ri)
                                    sum += Fv[(fi + ri) + (long)ftx * ((fj + rj) + (long)fty * (fk + rk))];
                        Cv[ci + (long)ctx * (cj + (long)cty * ck)] = sum / (ratio * ratio * ratio);
                    }
                }
    }
}

/* ---------------------------------------------------------------------------
 * Pieces for hierarchy drivers (oracle/hierarchy.py)
 * ------------------------------------------------------------------------- */

/* One RK stage of one block: rhs = L(u_in); u_out = a1 u_n + a2 u_in + a3 dt rhs
 * on interior cells; floors on all cells; det/trace constraints when final
 * (main.cpp:673-687). u_out may alias u_n. */
void orc_stage(const orc_params* p, const orc_geom* g, const double* u_n, const double* u_in,
               double* u_out, double* rhs, double a1, double a2, double a3, double dt, int final) {
    orc_rhs(p, g, u_in, rhs, NULL, NULL, NULL, NULL);
    combine(g, u_out, u_n, a1, u_in, a2, rhs, a3, dt);
    orc_floors(g, u_out);
    if (final) orc_algebraic(g, u_out);
}

/* Zero-gradient copy on the faces flagged in mask (bit 2d: low face of axis
 * d, bit 2d+1: high face), x then y then z passes, amr.cpp:447-480. */
void orc_fill_zero_gradient_masked(const orc_geom* g, double* u, int mask) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const long stride = orc_stride(g);
    const int ie[3] = {ng + g->n[0], ng + g->n[1], ng + g->n[2]};
    for (int v = 0; v < ORC_NV; ++v) {
        double* f = u + (long)v * stride;
#define A(i, j, k) f[(i) + (long)tx * ((j) + (long)ty * (k))]
        if (mask & 1)
            for (int k = 0; k < tz; ++k)
                for (int j = 0; j < ty; ++j)
                    for (int q = 0; q < ng; ++q) A(q, j, k) = A(ng, j, k);
        if (mask & 2)
            for (int k = 0; k < tz; ++k)
                for (int j = 0; j < ty; ++j)
                    for (int q = 0; q < ng; ++q) A(ie[0] + q, j, k) = A(ie[0] - 1, j, k);
        if (mask & 4)
            for (int k = 0; k < tz; ++k)
                for (int i = 0; i < tx; ++i)
                    for (int q = 0; q < ng; ++q) A(i, q, k) = A(i, ng, k);
        if (mask & 8)
            for (int k = 0; k < tz; ++k)
                for (int i = 0; i < tx; ++i)
                    for (int q = 0; q < ng; ++q) A(i, ie[1] + q, k) = A(i, ie[1] - 1, k);
        if (mask & 16)
            for (int j = 0; j < ty; ++j)
                for (int i = 0; i < tx; ++i)
                    for (int q = 0; q < ng; ++q) A(i, j, q) = A(i, j, ng);
        if (mask & 32)
            for (int j = 0; j < ty; ++j)
                for (int i = 0; i < tx; ++i)
                    for (int q = 0; q < ng; ++q) A(i, j, ie[2] + q) = A(i, j, ie[2] - 1);
#undef A
    }
}

/* Trilinear prolongation (amr.cpp:484-564) into the fine cells whose mask
 * byte is non-zero. */
void orc_prolongate_masked(const orc_geom* cg, const double* uc, const orc_geom* fg, double* uf,
                           const unsigned char* mask) {
    const int ftx = tx_(fg), fty = ty_(fg), ftz = tz_(fg);
    const int ctx = tx_(cg), cty = ty_(cg), ctz = tz_(cg);
    const long fs = orc_stride(fg), cs = orc_stride(cg);
    const int cis = cg->ng;
    const int ct[3] = {ctx, cty, ctz};
    for (int k = 0; k < ftz; ++k)
        for (int j = 0; j < fty; ++j)
            for (int i = 0; i < ftx; ++i) {
                const long fc = i + (long)ftx * (j + (long)fty * k);
                if (!mask[fc]) continue;
                const double X[3] = {xc(fg, 0, i), xc(fg, 1, j), xc(fg, 2, k)};
                double fr[3];
                int ci[3], cn[3];
                for (int d = 0; d < 3; ++d) {
                    double f = (X[d] - xc(cg, d, cis)) / cg->dx[d] + cis;
                    int c0 = (int)round(f);
                    if (c0 > ct[d] - 1) c0 = ct[d] - 1;
                    if (c0 < 0) c0 = 0;
                    fr[d] = f - (double)c0;
                    int c1 = c0 + (fr[d] >= 0.0 ? 1 : -1);
                    if (c1 > ct[d] - 1) c1 = ct[d] - 1;
                    if (c1 < 0) c1 = 0;
                    ci[d] = c0;
                    cn[d] = c1;
                }
                const double ax = fabs(fr[0]), ay = fabs(fr[1]), az = fabs(fr[2]);
                const double w000 = (1 - ax) * (1 - ay) * (1 - az);
                const double w100 = ax * (1 - ay) * (1 - az);
                const double w010 = (1 - ax) * ay * (1 - az);
                const double w001 = (1 - ax) * (1 - ay) * az;
                const double w110 = ax * ay * (1 - az);
                const double w101 = ax * (1 - ay) * az;
                const double w011 = (1 - ax) * ay * az;
                const double w111 = ax * ay * az;
                for (int v = 0; v < ORC_NV; ++v) {
                    const double* C = uc + (long)v * cs;
#define CV(a, b, c) C[(a) + (long)ctx * ((b) + (long)cty * (c))]
                    uf[(long)v * fs + fc] = w000 * CV(ci[0], ci[1], ci[2]) + w100 * CV(cn[0], ci[1], ci[2]) +
                        w010 * CV(ci[0], cn[1], ci[2]) + w001 * CV(ci[0], ci[1], cn[2]) +
                        w110 * CV(cn[0], cn[1], ci[2]) + w101 * CV(cn[0], ci[1], cn[2]) +
                        w011 * CV(ci[0], cn[1], cn[2]) + w111 * CV(cn[0], cn[1], cn[2]);
#undef CV
                }
            }
}

/* GRMHDEvolution::computeMatterSources, grmhd.cpp:1034-1103, at interior
 * cells: the ADM matter sources of a magnetised perfect fluid from the
 * primitives (PrimitiveVar order: rho, v^x, v^y, v^z, p, B^x, B^y, B^z, eps,
 * T, Ye; types.hpp:149-162). h = 1 + eps + p / (rho + 1e-30) (grmhd.hpp:55);
 * W = 1 / sqrt(max(1 - v^2, 1e-10)) with std::max's NaN behaviour;
 * b^2 = B^2 / W^2 + (B.v)^2; b_i = B_i / W^2 + (B.v) v_i;
 * rho_ADM = rho h W^2 - p + b^2 / 2; S_i = (rho h W^2 + b^2) v_i - (B.v) b_i;
 * S_ij = (rho h W^2 + b^2) v_i v_j + (p + b^2/2) delta_ij - b_i b_j - B_i B_j / W^2;
 * S = S_xx + S_yy + S_zz. Cells outside the interior keep their values. */
void orc_matter_sources(const orc_geom* g, const double* prim, double* rho, double* Si, double* Sij,
                        double* S) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g);
    const long stride = orc_stride(g);
    for (int k = ng; k < ng + g->n[2]; ++k)
        for (int j = ng; j < ng + g->n[1]; ++j)
            for (int i = ng; i < ng + g->n[0]; ++i) {
                const long c = i + (long)tx * (j + (long)ty * k);
                const double rho_p = prim[c], vx = prim[stride + c], vy = prim[2 * stride + c],
                             vz = prim[3 * stride + c], press = prim[4 * stride + c];
                const double Bx = prim[5 * stride + c], By = prim[6 * stride + c], Bz = prim[7 * stride + c];
                const double eps = prim[8 * stride + c];
                const double h = 1.0 + eps + press / (rho_p + 1e-30);
                const double v2 = vx * vx + vy * vy + vz * vz;
                const double one_m = 1.0 - v2;
                const double W = 1.0 / sqrt(one_m < 1.0e-10 ? 1.0e-10 : one_m);
                const double W2 = W * W;
                const double Bv = Bx * vx + By * vy + Bz * vz;
                const double B2 = Bx * Bx + By * By + Bz * Bz;
                const double b2 = B2 / W2 + Bv * Bv;
                const double rhoHW2 = rho_p * h * W2;
                rho[c] = rhoHW2 - press + 0.5 * b2;
                const double vel[3] = {vx, vy, vz};
                const double bco[3] = {Bx / W2 + Bv * vx, By / W2 + Bv * vy, Bz / W2 + Bv * vz};
                const double Bco[3] = {Bx, By, Bz};
                for (int a = 0; a < 3; ++a) Si[3 * c + a] = (rhoHW2 + b2) * vel[a] - Bv * bco[a];
                double tr = 0.0;
                for (int a = 0; a < 3; ++a)
                    for (int b = a; b < 3; ++b) {
                        const double delta = a == b ? 1.0 : 0.0;
                        const int s = a == 0 ? b : (a == 1 ? 2 + b : 5);  /* symIdx, types.hpp:52-54 */
                        const double v = (rhoHW2 + b2) * vel[a] * vel[b] + (press + 0.5 * b2) * delta -
                            bco[a] * bco[b] - Bco[a] * Bco[b] / W2;
                        Sij[6 * c + s] = v;
                        if (a == b) tr += v;
                    }
                S[c] = tr;
            }
}

/* ---------------------------------------------------------------------------
 * Psi4 extraction, postprocess.cpp:61-99 (interp), :106-162 (spin-weight -2
 * harmonics), :167-235 (Psi4 at a point), :245-314 (Psi4Extractor::extract).
 * std::complex arithmetic is written out as GCC evaluates it for finite
 * values: complex x complex = (ac - bd, ad + bc), complex x real and
 * complex / real component-wise.
 * ------------------------------------------------------------------------- */
typedef struct { double re, im; } orc_cplx;

static orc_cplx cmul(orc_cplx a, orc_cplx b) {
    orc_cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static orc_cplx cscale(orc_cplx a, double s) {
    orc_cplx r = {a.re * s, a.im * s};
    return r;
}
static orc_cplx cadd(orc_cplx a, orc_cplx b) {
    orc_cplx r = {a.re + b.re, a.im + b.im};
    return r;
}

static double pp_interp(const orc_geom* g, const double* u, int var, double px, double py, double pz) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const long stride = orc_stride(g);
    const double ix = (px - g->lo[0]) / g->dx[0] + ng - 0.5;
    const double iy = (py - g->lo[1]) / g->dx[1] + ng - 0.5;
    const double iz = (pz - g->lo[2]) / g->dx[2] + ng - 0.5;
    const int nx = tx - 1, ny = ty - 1, nz = tz - 1;
#define CLAMP(v, lo, hi) ((v) < (lo) ? (lo) : ((v) > (hi) ? (hi) : (v)))
    const int i0 = CLAMP((int)floor(ix), 0, nx - 1), j0 = CLAMP((int)floor(iy), 0, ny - 1),
              k0 = CLAMP((int)floor(iz), 0, nz - 1);
#undef CLAMP
    const int i1 = i0 + 1 < nx ? i0 + 1 : nx, j1 = j0 + 1 < ny ? j0 + 1 : ny, k1 = k0 + 1 < nz ? k0 + 1 : nz;
    const double wx = ix - floor(ix), wy = iy - floor(iy), wz = iz - floor(iz);
    const double* f = u + (long)var * stride;
#define D(i, j, k) f[((i) < nx ? (i) : nx) + (long)tx * (((j) < ny ? (j) : ny) + (long)ty * ((k) < nz ? (k) : nz))]
    return (1 - wz) * ((1 - wy) * ((1 - wx) * D(i0, j0, k0) + wx * D(i1, j0, k0)) +
                       wy * ((1 - wx) * D(i0, j1, k0) + wx * D(i1, j1, k0))) +
        wz * ((1 - wy) * ((1 - wx) * D(i0, j0, k1) + wx * D(i1, j0, k1)) +
              wy * ((1 - wx) * D(i0, j1, k1) + wx * D(i1, j1, k1)));
#undef D
}

#define ORC_PI 3.14159265358979323846

/* -2 Y_lm: l = 2 all m, l = 3 m = +-3; zero otherwise (postprocess.cpp:106-162) */
static orc_cplx sw_ylm(int l, int m, double theta, double phi) {
    const double c2th = cos(theta / 2.0), s2th = sin(theta / 2.0);
    orc_cplx e = {cos(m * phi), sin(m * phi)}, z = {0.0, 0.0};
    if (l == 2) {
        if (m == 2) return cscale(e, sqrt(5.0 / (4.0 * ORC_PI)) * pow(c2th, 4));
        if (m == 1) return cscale(e, sqrt(5.0 / ORC_PI) * pow(c2th, 3) * s2th);
        if (m == 0) {
            orc_cplx r = {sqrt(15.0 / (2.0 * ORC_PI)) * pow(c2th, 2) * pow(s2th, 2), 0.0};
            return r;
        }
        if (m == -1) return cscale(e, sqrt(5.0 / ORC_PI) * c2th * pow(s2th, 3));
        if (m == -2) return cscale(e, sqrt(5.0 / (4.0 * ORC_PI)) * pow(s2th, 4));
    }
    if (l == 3) {
        const double N33 = sqrt(21.0 / (2.0 * ORC_PI));
        if (m == 3) return cscale(e, -N33 / 4.0 * pow(c2th, 5) * s2th / 2.0);
        if (m == -3) return cscale(e, N33 / 4.0 * c2th * pow(s2th, 5) / 2.0);
    }
    return z;
}

static orc_cplx psi4_at(const orc_geom* g, const double* u, double px, double py, double pz, double nx, double ny,
                        double nz) {
    orc_cplx zero = {0.0, 0.0};
    const double chi = pp_interp(g, u, CHI, px, py, pz);
    if (chi < 1.0e-12) return zero;
    const double rho = sqrt(nx * nx + ny * ny);
    double tx, ty, tz, phx, phy, phz;
    if (rho > 1.0e-10) {
        tx = nx * nz / rho;
        ty = ny * nz / rho;
        tz = -rho;
        phx = -ny / rho;
        phy = nx / rho;
        phz = 0.0;
    } else {
        tx = 1.0, ty = 0.0, tz = 0.0, phx = 0.0, phy = 1.0, phz = 0.0;
    }
    const double sqrt2 = sqrt(2.0);
    const orc_cplx mx = {tx / sqrt2, -phx / sqrt2}, my = {ty / sqrt2, -phy / sqrt2}, mz = {tz / sqrt2, -phz / sqrt2};
    const double fac = 1.0 / chi;
    const double Bxx = pp_interp(g, u, AXX, px, py, pz) * fac, Bxy = pp_interp(g, u, AXY, px, py, pz) * fac,
                 Bxz = pp_interp(g, u, AXZ, px, py, pz) * fac, Byy = pp_interp(g, u, AYY, px, py, pz) * fac,
                 Byz = pp_interp(g, u, AYZ, px, py, pz) * fac, Bzz = pp_interp(g, u, AZZ, px, py, pz) * fac;
    orc_cplx p = cmul(cscale(mx, Bxx), mx);
    p = cadd(p, cmul(cscale(my, Byy), my));
    p = cadd(p, cmul(cscale(mz, Bzz), mz));
    p = cadd(p, cmul(cscale(mx, 2.0 * Bxy), my));
    p = cadd(p, cmul(cscale(mx, 2.0 * Bxz), mz));
    p = cadd(p, cmul(cscale(my, 2.0 * Byz), mz));
    p.re = -p.re;
    p.im = -p.im;
    return p;
}

void orc_psi4_modes(const orc_geom* g, const double* hi, const double* u, const double* radii, int nr, int n_theta,
                    int n_phi, int l_max, double* modes, int* npoints) {
    const int nm = (l_max + 1) * (l_max + 1) - 4;
    const double dth = ORC_PI / n_theta, dph = 2.0 * ORC_PI / n_phi;
    for (int r = 0; r < nr; ++r) {
        const double r_ext = radii[r];
        double* out = modes + (long)r * nm * 2;
        int* seen = (int*)calloc((size_t)nm, sizeof(int));
        int inside = 0;
        for (int q = 0; q < 2 * nm; ++q) out[q] = 0.0;
        for (int it = 0; it < n_theta; ++it) {
            const double theta = (it + 0.5) * dth, sth = sin(theta), cth = cos(theta);
            for (int jp = 0; jp < n_phi; ++jp) {
                const double phi = jp * dph, sph = sin(phi), cph = cos(phi);
                const double px = r_ext * sth * cph, py = r_ext * sth * sph, pz = r_ext * cth;
                const double nx = sth * cph, ny = sth * sph, nz = cth;
                /* lowerCorner() + dx <= p <= upperCorner() - dx (postprocess.cpp:273-278) */
                if (!(px >= g->lo[0] + g->dx[0] && px <= hi[0] - g->dx[0] && py >= g->lo[1] + g->dx[1] &&
                      py <= hi[1] - g->dx[1] && pz >= g->lo[2] + g->dx[2] && pz <= hi[2] - g->dx[2]))
                    continue;
                ++inside;
                const orc_cplx psi4 = psi4_at(g, u, px, py, pz, nx, ny, nz);
                int q = 0;
                for (int l = 2; l <= l_max; ++l)
                    for (int m = -l; m <= l; ++m, ++q) {
                        orc_cplx y = sw_ylm(l, m, theta, phi);
                        y.im = -y.im;
                        const orc_cplx c = cscale(cscale(cscale(cscale(cmul(psi4, y), sth), dth), dph), r_ext);
                        if (seen[q]) {
                            out[2 * q] += c.re;
                            out[2 * q + 1] += c.im;
                        } else {
                            out[2 * q] = c.re;
                            out[2 * q + 1] = c.im;
                            seen[q] = 1;
                        }
                    }
            }
        }
        if (npoints) npoints[r] = inside;
        free(seen);
    }
}

/* ---------------------------------------------------------------------------
 * Apparent-horizon flow, horizon_finder.cpp:55-98 (interpolate, indices
 * clamped per access), :114-281 (computeExpansion), :292-300 (angular grid),
 * :310-449 (findHorizon), :452-507 (findAllHorizons scan).
 * ------------------------------------------------------------------------- */
static double hz_interp(const orc_geom* g, const double* u, int var, double px, double py, double pz) {
    const int ng = g->ng, tx = tx_(g), ty = ty_(g), tz = tz_(g);
    const double ix = (px - g->lo[0]) / g->dx[0] + ng - 0.5;
    const double iy = (py - g->lo[1]) / g->dx[1] + ng - 0.5;
    const double iz = (pz - g->lo[2]) / g->dx[2] + ng - 0.5;
    const int i0 = (int)floor(ix), j0 = (int)floor(iy), k0 = (int)floor(iz);
    const int nx = tx - 1, ny = ty - 1, nz = tz - 1;
    const int i1 = i0 + 1 < nx ? i0 + 1 : nx, j1 = j0 + 1 < ny ? j0 + 1 : ny, k1 = k0 + 1 < nz ? k0 + 1 : nz;
    const double wx = ix - floor(ix), wy = iy - floor(iy), wz = iz - floor(iz);
    const double* f = u + (long)var * orc_stride(g);
#define CL(v, n) ((v) < (n) ? ((v) > 0 ? (v) : 0) : ((n) > 0 ? (n) : 0))
#define D(i, j, k) f[CL(i, nx) + (long)tx * (CL(j, ny) + (long)ty * CL(k, nz))]
    return (1 - wz) * ((1 - wy) * ((1 - wx) * D(i0, j0, k0) + wx * D(i1, j0, k0)) +
                       wy * ((1 - wx) * D(i0, j1, k0) + wx * D(i1, j1, k0))) +
        wz * ((1 - wy) * ((1 - wx) * D(i0, j0, k1) + wx * D(i1, j0, k1)) +
              wy * ((1 - wx) * D(i0, j1, k1) + wx * D(i1, j1, k1)));
#undef D
#undef CL
}

/* component dir of the unit normal s^i at a displaced point (the scomp lambda) */
static double hz_scomp(const orc_geom* g, const double* u, double px, double py, double pz, double snx, double sny,
                       double snz, int dir, double delta) {
    const double ppx = px + (dir == 0 ? delta : 0.0), ppy = py + (dir == 1 ? delta : 0.0),
                 ppz = pz + (dir == 2 ? delta : 0.0);
    const double chi = hz_interp(g, u, CHI, ppx, ppy, ppz);
    if (chi < 1.0e-12) return 0.0;
    const double gxx = hz_interp(g, u, GXX, ppx, ppy, ppz), gxy = hz_interp(g, u, GXY, ppx, ppy, ppz),
                 gxz = hz_interp(g, u, GXZ, ppx, ppy, ppz), gyy = hz_interp(g, u, GYY, ppx, ppy, ppz),
                 gyz = hz_interp(g, u, GYZ, ppx, ppy, ppz), gzz = hz_interp(g, u, GZZ, ppx, ppy, ppz);
    const double det = gxx * (gyy * gzz - gyz * gyz) - gxy * (gxy * gzz - gyz * gxz) + gxz * (gxy * gyz - gyy * gxz);
    if (fabs(det) < 1.0e-14) return 0.0;
    const double idet = 1.0 / det;
    const double igxx = (gyy * gzz - gyz * gyz) * idet, igxy = (gxz * gyz - gxy * gzz) * idet,
                 igxz = (gxy * gyz - gxz * gyy) * idet, igyy = (gxx * gzz - gxz * gxz) * idet,
                 igyz = (gxy * gxz - gxx * gyz) * idet, igzz = (gxx * gyy - gxy * gxy) * idet;
    const double hxx = gxx / chi, hxy = gxy / chi, hxz = gxz / chi, hyy = gyy / chi, hyz = gyz / chi, hzz = gzz / chi;
    const double sx = hxx * snx + hxy * sny + hxz * snz, sy = hxy * snx + hyy * sny + hyz * snz,
                 sz = hxz * snx + hyz * sny + hzz * snz;
    const double n2 = snx * sx + sny * sy + snz * sz;
    if (n2 < 1.0e-14) return 0.0;
    const double nm = sqrt(n2);
    const double ixx = chi * igxx, ixy = chi * igxy, ixz = chi * igxz, iyy = chi * igyy, iyz = chi * igyz,
                 izz = chi * igzz;
    if (dir == 0) return (ixx * sx + ixy * sy + ixz * sz) / nm;
    if (dir == 1) return (ixy * sx + iyy * sy + iyz * sz) / nm;
    return (ixz * sx + iyz * sy + izz * sz) / nm;
}

double orc_horizon_expansion(const orc_geom* g, const double* u, double px, double py, double pz, double snx,
                             double sny, double snz) {
    const double chi = hz_interp(g, u, CHI, px, py, pz);
    const double gxx = hz_interp(g, u, GXX, px, py, pz), gxy = hz_interp(g, u, GXY, px, py, pz),
                 gxz = hz_interp(g, u, GXZ, px, py, pz), gyy = hz_interp(g, u, GYY, px, py, pz),
                 gyz = hz_interp(g, u, GYZ, px, py, pz), gzz = hz_interp(g, u, GZZ, px, py, pz);
    const double Axx = hz_interp(g, u, AXX, px, py, pz), Axy = hz_interp(g, u, AXY, px, py, pz),
                 Axz = hz_interp(g, u, AXZ, px, py, pz), Ayy = hz_interp(g, u, AYY, px, py, pz),
                 Ayz = hz_interp(g, u, AYZ, px, py, pz), Azz = hz_interp(g, u, AZZ, px, py, pz);
    const double K = hz_interp(g, u, KTR, px, py, pz);
    if (chi < 1.0e-12) return 0.0;
    const double hxx = gxx / chi, hxy = gxy / chi, hxz = gxz / chi, hyy = gyy / chi, hyz = gyz / chi, hzz = gzz / chi;
    const double det = gxx * (gyy * gzz - gyz * gyz) - gxy * (gxy * gzz - gyz * gxz) + gxz * (gxy * gyz - gyy * gxz);
    if (fabs(det) < 1.0e-14) return 0.0;
    const double sx = hxx * snx + hxy * sny + hxz * snz, sy = hxy * snx + hyy * sny + hyz * snz,
                 sz = hxz * snx + hyz * sny + hzz * snz;
    const double norm2 = snx * sx + sny * sy + snz * sz;
    if (norm2 < 1.0e-14) return 0.0;
    const double norm = sqrt(norm2);
    const double ux = snx / norm, uy = sny / norm, uz = snz / norm;
    const double Kxx = (Axx + gxx * K / 3.0) / chi, Kxy = (Axy + gxy * K / 3.0) / chi, Kxz = (Axz + gxz * K / 3.0) / chi,
                 Kyy = (Ayy + gyy * K / 3.0) / chi, Kyz = (Ayz + gyz * K / 3.0) / chi, Kzz = (Azz + gzz * K / 3.0) / chi;
    const double Kss = Kxx * ux * ux + Kyy * uy * uy + Kzz * uz * uz +
        2.0 * (Kxy * ux * uy + Kxz * ux * uz + Kyz * uy * uz);
    const double eps = g->dx[0];
#define SC(d, e) hz_scomp(g, u, px, py, pz, snx, sny, snz, d, e)
    const double div_s = (SC(0, eps) - SC(0, -eps)) / (2.0 * eps) + (SC(1, eps) - SC(1, -eps)) / (2.0 * eps) +
        (SC(2, eps) - SC(2, -eps)) / (2.0 * eps);
#undef SC
    return div_s + K - Kss;
}

/* findHorizon's flow and surface integrals. h[Nth * 2 Nth] in/out (start:
 * the initial radius everywhere); returns the number of iterations run when
 * converged (max |Theta| < tol at that iteration), -1 otherwise. res[0..4] =
 * area, irreducible mass, spin (clamped), equatorial and polar circumference. */
int orc_find_horizon(const orc_geom* g, const double* u, const double* center, int max_iterations, double tol,
                     int ang_res, double* h, double* res) {
    const int Nth = ang_res, Nph = 2 * ang_res;
    const double h_grid = g->dx[0], flow_step = 0.05 * h_grid;
    int converged = -1;
    for (int iter = 0; iter < max_iterations; ++iter) {
        double max_theta = 0.0;
        for (int i = 0; i < Nth; ++i) {
            const double th = ORC_PI * (i + 0.5) / Nth, sth = sin(th), cth = cos(th);
            for (int j = 0; j < Nph; ++j) {
                const double ph = 2.0 * ORC_PI * j / Nph, sph = sin(ph), cph = cos(ph);
                const double r = h[i * Nph + j];
                const double px = center[0] + r * sth * cph, py = center[1] + r * sth * sph, pz = center[2] + r * cth;
                const double Theta = orc_horizon_expansion(g, u, px, py, pz, sth * cph, sth * sph, cth);
                h[i * Nph + j] -= flow_step * Theta;
                const double lo = 1.0e-6 * h_grid;
                h[i * Nph + j] = h[i * Nph + j] < lo ? lo : h[i * Nph + j];
                const double a = fabs(Theta);
                max_theta = max_theta < a ? a : max_theta;
            }
        }
        if (max_theta < tol) {
            converged = iter + 1;
            break;
        }
    }
    if (converged < 0) return -1;
    const double dth = ORC_PI / Nth, dph = 2.0 * ORC_PI / Nph;
    double area = 0.0, jz = 0.0;
    for (int i = 0; i < Nth; ++i) {
        const double th = ORC_PI * (i + 0.5) / Nth, sth = sin(th), cth = cos(th);
        for (int j = 0; j < Nph; ++j) {
            const double ph = 2.0 * ORC_PI * j / Nph, sph = sin(ph), cph = cos(ph);
            const double r = h[i * Nph + j];
            const double px = center[0] + r * sth * cph, py = center[1] + r * sth * sph, pz = center[2] + r * cth;
            const double chi = hz_interp(g, u, CHI, px, py, pz);
            if (chi < 1.0e-12) continue;
            const double gxx = hz_interp(g, u, GXX, px, py, pz), gyy = hz_interp(g, u, GYY, px, py, pz),
                         gzz = hz_interp(g, u, GZZ, px, py, pz);
            const double sqrt_g = sqrt(fabs(gxx * gyy * gzz)) / (chi * sqrt(chi));
            area += sqrt_g * r * r * sth * dth * dph;
            jz += (-sph * px + cph * py) * sqrt_g * r * sth * dth * dph;
        }
    }
    const double mirr = sqrt(area / (16.0 * ORC_PI));
    double ceq = 0.0, cpol = 0.0;
    for (int j = 0; j < Nph; ++j) ceq += h[(Nth / 2) * Nph + j] * dph;
    for (int i = 0; i < Nth; ++i) cpol += h[i * Nph] * dth;
    double a = mirr > 1.0e-12 ? jz / (mirr * mirr) : 0.0;
    a = a < -1.0 ? -1.0 : (a > 1.0 ? 1.0 : a);
    res[0] = area;
    res[1] = mirr;
    res[2] = a;
    res[3] = ceq;
    res[4] = 2.0 * cpol;
    return converged;
}
