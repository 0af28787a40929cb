/*
 * ccz4_oracle.h -- CPU oracle for the CCZ4 RHS + SSP-RK3 hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA path is
 * compared against; it is never linked into, called by, or shipped with the
 * product library (granite_b200/libgranite_ccz4.so). Only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py use it.
 *
 * Parity pin: every function below restates a reference routine of GRANITE
 * v0.6.7 (file:line cited per function) in the same floating-point evaluation
 * order, so that, built with -O2 -ffp-contract=off, it reproduces the compiled
 * reference (oracle/_ref, built from the reference sources by oracle/Makefile)
 * bit for bit. tests/test_oracle_pin.py checks that on seeded inputs.
 *
 * Data layout is the reference GridBlock layout (grid.hpp:109-116):
 *   u[v * stride + i + tx * (j + ty * k)],  tx = n0 + 2 ng, ty = n1 + 2 ng,
 *   stride = tx * ty * (n2 + 2 ng),  v in SpacetimeVar order (types.hpp:104-130).
 * Matter sources mirror the reference std::vector<std::array<>> layouts:
 *   rho[N], Si[N][3], Sij[N][6], S[N] (N = stride). NULL means vacuum.
 */
#ifndef GRANITE_CCZ4_ORACLE_H
#define GRANITE_CCZ4_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NV 22

typedef struct {
    int n[3];        /* interior cells per axis */
    int ng;          /* ghost width */
    double lo[3];    /* lower corner of the interior */
    double dx[3];    /* cell spacing (hi - lo) / n, grid.cpp:20-22 */
} orc_geom;

typedef struct {
    double kappa1, kappa2, eta, ko_sigma, chi_blend_center, chi_blend_width;
} orc_params;

/* ghost-fill modes used by the RK3 driver */
enum { ORC_BC_SOMMERFELD = 0, ORC_BC_PERIODIC = 1 };

long orc_stride(const orc_geom* g);

/* RHS (+ KO when ko_sigma > 0) at interior points; ghosts of rhs untouched. */
void orc_rhs(const orc_params* p, const orc_geom* g, const double* u, double* rhs,
             const double* rho, const double* Si, const double* Sij, const double* S);
/* KO dissipation added to rhs at interior points. */
void orc_dissipation(const orc_params* p, const orc_geom* g, const double* u, double* rhs);
/* Hamiltonian and momentum constraints; ham[N], mom[N][3]; ghosts set to 0. */
void orc_constraints(const orc_geom* g, const double* u, double* ham, double* mom);

/* ghost fills over all 22 fields */
void orc_fill_zero_gradient(const orc_geom* g, double* u);
void orc_fill_sommerfeld(const orc_geom* g, double* u);
void orc_fill_periodic(const orc_geom* g, double* u);
/* floors on chi and alpha (all cells), algebraic det/trace constraints (all cells) */
void orc_floors(const orc_geom* g, double* u);
void orc_algebraic(const orc_geom* g, double* u);

/* One coarse step of a single-level grid: level ghost fill, 3 RK stages with
 * per-stage floors and outer-BC, final algebraic constraints, level ghost fill.
 * u: state (in/out); stage, rhs: scratch of the same size. bc: ORC_BC_*. */
void orc_rk3_step(const orc_params* p, const orc_geom* g, double* u, double* stage,
                  double* rhs, double dt, int bc);
/* orc_rk3_step with matter sources (layout as orc_rhs) in all three stages. */
void orc_rk3_step_matter(const orc_params* p, const orc_geom* g, double* u, double* stage, double* rhs,
                         double dt, int bc, const double* rho, const double* Si, const double* Sij,
                         const double* S);

/* initial data over all cells */
void orc_init_flat(const orc_geom* g, double* u);
void orc_init_gauge_wave(const orc_geom* g, double* u, double amplitude, double wavelength);
void orc_init_brill_lindquist(const orc_geom* g, double* u, int nbh, const double* mass,
                              const double* pos /* [nbh][3] */, double r_floor);
double orc_bl_conformal_factor(int nbh, const double* mass, const double* pos, double x,
                               double y, double z, double r_floor);

/* AMR inter-level operators over all fields */
void orc_prolongate(const orc_geom* coarse, const double* uc, const orc_geom* fine, double* uf,
                    int ghosts_only);
void orc_restrict(const orc_geom* fine, const double* uf, const orc_geom* coarse, double* uc);

/* hierarchy-driver pieces (oracle/hierarchy.py) */
void orc_stage(const orc_params* p, const orc_geom* g, const double* u_n, const double* u_in,
               double* u_out, double* rhs, double a1, double a2, double a3, double dt, int final);
void orc_fill_zero_gradient_masked(const orc_geom* g, double* u, int mask);
void orc_prolongate_masked(const orc_geom* cg, const double* uc, const orc_geom* fg, double* uf,
                           const unsigned char* mask);

/* sum over interior points of H^2 and |M|^2 of one block (for RMS norms) */
void orc_constraint_sums(const orc_geom* g, const double* u, double* h2, double* m2,
                         long* npts);

/* GRMHD matter sources of the CCZ4 RHS (grmhd.cpp:1034-1103): prim[11][N] in
 * PrimitiveVar order; rho[N], Si[N][3], Sij[N][6], S[N] written at interior
 * cells only. */
#define ORC_NPRIM 11
void orc_matter_sources(const orc_geom* g, const double* prim, double* rho, double* Si, double* Sij,
                        double* S);

/* Psi4Extractor::extract (postprocess.cpp:245-314) on one block at one time:
 * modes[r][q][re, im] for extraction radius r and q over l = 2..l_max,
 * m = -l..l; hi = the block's upper corner; npoints[r] (nullable) = the sphere
 * points of radius r inside the block. */
void orc_psi4_modes(const orc_geom* g, const double* hi, const double* u, const double* radii, int nr, int n_theta,
                    int n_phi, int l_max, double* modes, int* npoints);

/* Apparent-horizon flow (horizon_finder.cpp): the null expansion at a point
 * for the coordinate normal sn (computeExpansion, :114-281), and findHorizon
 * (:310-449): h[ang_res * 2 ang_res] in (initial radius) / out; returns the
 * iterations run when converged, else -1; res = area, irreducible mass, spin,
 * equatorial and polar circumference. */
double orc_horizon_expansion(const orc_geom* g, const double* u, double px, double py, double pz, double snx,
                             double sny, double snz);
int orc_find_horizon(const orc_geom* g, const double* u, const double* center, int max_iterations, double tol,
                     int ang_res, double* h, double* res);

/* OpenMP thread count used by the parallel loops (0 = leave default) */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
