// ref_shim.cpp -- C ABI over the compiled GRANITE reference (test infrastructure).
//
// oracle/Makefile compiles this file together with the unmodified reference
// sources src/spacetime/ccz4.cpp, src/core/grid.cpp, src/amr/amr.cpp,
// src/initial_data/initial_data.cpp, src/grmhd/{grmhd,hlld,tabulated_eos}.cpp,
// src/postprocess/postprocess.cpp and src/horizon/horizon_finder.cpp into
// oracle/_ref/libgranite_ref_*.so.
// The shim only copies flat buffers in and out of reference GridBlocks and
// calls the reference's own operators; it adds no arithmetic of its own except
// in ref_rk3_steps, whose main.cpp lambdas (combine, floors, algebraic
// constraints, 1/r outer boundary; main.cpp:306-521,588-689) are not linkable
// (main.cpp needs yaml-cpp, HDF5 and the GRMHD module), so that driver uses the
// oracle's restatement of those lambdas (ccz4_oracle.c) around the reference
// computeRHSVacuum and AMRHierarchy::fillGhostZones.
#include "granite/amr/amr.hpp"
#include "granite/core/grid.hpp"
#include "granite/grmhd/grmhd.hpp"
#include "granite/horizon/horizon_finder.hpp"
#include "granite/postprocess/postprocess.hpp"
#include "granite/initial_data/initial_data.hpp"
#include "granite/spacetime/ccz4.hpp"

#include "ccz4_oracle.h"

#include <chrono>
#include <cstring>
#include <iostream>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace granite;

namespace {

struct Geo {
    std::array<int, DIM> n;
    int ng;
    std::array<Real, DIM> lo, hi;
};

Geo geo(const int* n, int ng, const double* lo, const double* hi) {
    Geo g;
    for (int d = 0; d < 3; ++d) {
        g.n[d] = n[d];
        g.lo[d] = lo[d];
        g.hi[d] = hi[d];
    }
    g.ng = ng;
    return g;
}

std::unique_ptr<GridBlock> block(const Geo& g, int level = 0, int id = 0) {
    return std::make_unique<GridBlock>(id, level, g.n, g.lo, g.hi, g.ng, NUM_SPACETIME_VARS);
}

size_t nbytes(const GridBlock& b) {
    return sizeof(Real) * b.totalSize() * NUM_SPACETIME_VARS;
}

spacetime::CCZ4Params params(const double* p6) {
    spacetime::CCZ4Params p;
    p.kappa1 = p6[0];
    p.kappa2 = p6[1];
    p.eta = p6[2];
    p.ko_sigma = p6[3];
    p.chi_blend_center = p6[4];
    p.chi_blend_width = p6[5];
    return p;
}

orc_geom ogeom(const GridBlock& b) {
    orc_geom o;
    for (int d = 0; d < 3; ++d) {
        o.n[d] = b.numCells()[d];
        o.lo[d] = b.lowerCorner()[d];
        o.dx[d] = b.dx(d);
    }
    o.ng = b.getNumGhost();
    return o;
}

} // namespace

extern "C" {

void ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// CCZ4Evolution::computeRHS / computeRHSVacuum (ccz4.cpp:229-865). p6 = {kappa1,
// kappa2, eta, ko_sigma, chi_blend_center, chi_blend_width}. Matter arrays may
// all be NULL (vacuum overload). rhs receives the full block (ghosts zero).
void ref_rhs(const double* p6, const int* n, int ng, const double* lo, const double* hi,
             const double* u, double* rhs, const double* rho, const double* Si,
             const double* Sij, const double* S) {
    Geo g = geo(n, ng, lo, hi);
    auto in = block(g);
    auto out = block(g, 0, 1);
    std::memcpy(in->flatBuffer(), u, nbytes(*in));
    spacetime::CCZ4Evolution ev(params(p6));
    if (!rho) {
        ev.computeRHSVacuum(*in, *out);
    } else {
        size_t N = in->totalSize();
        std::vector<Real> r(rho, rho + N), s(S, S + N);
        std::vector<std::array<Real, DIM>> si(N);
        std::vector<std::array<Real, SYM_TENSOR_COMPS>> sij(N);
        for (size_t c = 0; c < N; ++c) {
            for (int a = 0; a < 3; ++a) si[c][a] = Si[3 * c + a];
            for (int a = 0; a < 6; ++a) sij[c][a] = Sij[6 * c + a];
        }
        ev.computeRHS(*in, *out, r, si, sij, s);
    }
    std::memcpy(rhs, out->flatBuffer(), nbytes(*out));
}

// CCZ4Evolution::applyDissipation (ccz4.cpp:871-935): rhs (full block) in/out.
void ref_dissipation(const double* p6, const int* n, int ng, const double* lo, const double* hi,
                     const double* u, double* rhs) {
    Geo g = geo(n, ng, lo, hi);
    auto in = block(g);
    auto out = block(g, 0, 1);
    std::memcpy(in->flatBuffer(), u, nbytes(*in));
    std::memcpy(out->flatBuffer(), rhs, nbytes(*out));
    spacetime::CCZ4Evolution ev(params(p6));
    ev.applyDissipation(*in, *out);
    std::memcpy(rhs, out->flatBuffer(), nbytes(*out));
}

// CCZ4Evolution::computeConstraints (ccz4.cpp:941-1159): ham[N], mom[N][3].
void ref_constraints(const int* n, int ng, const double* lo, const double* hi, const double* u,
                     double* ham, double* mom) {
    Geo g = geo(n, ng, lo, hi);
    auto in = block(g);
    std::memcpy(in->flatBuffer(), u, nbytes(*in));
    spacetime::CCZ4Params p;
    spacetime::CCZ4Evolution ev(p);
    std::vector<Real> h;
    std::vector<std::array<Real, DIM>> m;
    ev.computeConstraints(*in, h, m);
    for (size_t c = 0; c < h.size(); ++c) {
        ham[c] = h[c];
        for (int a = 0; a < 3; ++a) mom[3 * c + a] = m[c][a];
    }
}

// GRMHDEvolution::computeMatterSources (grmhd.cpp:1034-1103): prim[11][N]
// (PrimitiveVar order, types.hpp:149-162) in; rho[N], Si[N][3], Sij[N][6],
// S[N] in/out (interior written, the rest keeps the caller's values). The
// ideal-gas EOS is a placeholder: the routine only calls the non-virtual
// EquationOfState::enthalpy (grmhd.hpp:55).
void ref_matter_sources(const int* n, int ng, const double* lo, const double* hi, const double* prim,
                        double* rho, double* Si, double* Sij, double* S) {
    Geo g = geo(n, ng, lo, hi);
    auto st = block(g);
    auto pr = std::make_unique<GridBlock>(1, 0, g.n, g.lo, g.hi, g.ng, NUM_PRIMITIVE_VARS);
    std::memcpy(pr->flatBuffer(), prim, sizeof(Real) * pr->totalSize() * NUM_PRIMITIVE_VARS);
    const size_t N = st->totalSize();
    std::vector<Real> r(rho, rho + N), s(S, S + N);
    std::vector<std::array<Real, DIM>> si(N);
    std::vector<std::array<Real, SYM_TENSOR_COMPS>> sij(N);
    for (size_t c = 0; c < N; ++c) {
        for (int a = 0; a < 3; ++a) si[c][a] = Si[3 * c + a];
        for (int a = 0; a < 6; ++a) sij[c][a] = Sij[6 * c + a];
    }
    grmhd::GRMHDParams gp;
    grmhd::GRMHDEvolution ev(gp, std::make_shared<grmhd::IdealGasEOS>());
    ev.computeMatterSources(*st, *pr, r, si, sij, s);
    for (size_t c = 0; c < N; ++c) {
        rho[c] = r[c];
        S[c] = s[c];
        for (int a = 0; a < 3; ++a) Si[3 * c + a] = si[c][a];
        for (int a = 0; a < 6; ++a) Sij[6 * c + a] = sij[c][a];
    }
}

// Psi4Extractor::extract at time 0 then getMode (postprocess.cpp:245-326):
// modes[r][q][re, im], q over l = 2..l_max, m = -l..l.
void ref_psi4_modes(const int* n, int ng, const double* lo, const double* hi, const double* u, const double* radii,
                    int nr, int n_theta, int n_phi, int l_max, double* modes) {
    auto b = block(geo(n, ng, lo, hi));
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    postprocess::GWExtractionParams gp;
    gp.extraction_radii.assign(radii, radii + nr);
    gp.l_max = l_max;
    gp.n_theta = n_theta;
    gp.n_phi = n_phi;
    postprocess::Psi4Extractor ex(gp);
    ex.extract(*b, 0.0);
    int q = 0;
    for (int r = 0; r < nr; ++r)
        for (int l = 2; l <= l_max; ++l)
            for (int m = -l; m <= l; ++m, ++q) {
                const std::complex<Real> v = ex.getMode(l, m, radii[r]);
                modes[2 * q] = v.real();
                modes[2 * q + 1] = v.imag();
            }
}

// A Psi4 time series and its analysis (postprocess.cpp:245-475): extract at
// times[t] from the block states u + t * block size, t < nt, then per radius r
// and mode q (l = 2..l_max, m = -l..l):
//   count[r][q]            the recorded entries,
//   series[r][q][t][3]     their (time, re, im),
//   strain[r][q][2]        computeStrain,
//   energy[r]              computeRadiatedEnergy,
//   extrap[q][2]           extrapolateToInfinity,
// and computeEnergySpectrum(sl, sm, radii[sr]) into spec[k][2], k < the return value.
int ref_psi4_series(const int* n, int ng, const double* lo, const double* hi, const double* u, const double* times,
                    int nt, const double* radii, int nr, int n_theta, int n_phi, int l_max, int* count,
                    double* series, double* strain, double* energy, double* extrap, int sl, int sm, int sr,
                    double* spec, int spec_cap) {
    auto b = block(geo(n, ng, lo, hi));
    const size_t per = b->totalSize() * NUM_SPACETIME_VARS;
    postprocess::GWExtractionParams gp;
    gp.extraction_radii.assign(radii, radii + nr);
    gp.l_max = l_max;
    gp.n_theta = n_theta;
    gp.n_phi = n_phi;
    postprocess::Psi4Extractor ex(gp);
    for (int t = 0; t < nt; ++t) {
        std::memcpy(b->flatBuffer(), u + t * per, nbytes(*b));
        ex.extract(*b, times[t]);
    }
    const int nm = (l_max + 1) * (l_max + 1) - 4;
    for (int r = 0; r < nr; ++r) {
        int q = 0;
        for (int l = 2; l <= l_max; ++l)
            for (int m = -l; m <= l; ++m, ++q) {
                const auto& s = ex.getTimeSeries(l, m, radii[r]);
                const int rq = r * nm + q;
                count[rq] = (int)s.size();
                for (size_t t = 0; t < s.size() && (int)t < nt; ++t) {
                    series[3 * ((size_t)rq * nt + t)] = s[t].first;
                    series[3 * ((size_t)rq * nt + t) + 1] = s[t].second.real();
                    series[3 * ((size_t)rq * nt + t) + 2] = s[t].second.imag();
                }
                const std::complex<Real> h = ex.computeStrain(l, m, radii[r]);
                strain[2 * rq] = h.real();
                strain[2 * rq + 1] = h.imag();
                if (r == 0) {
                    const std::complex<Real> e = ex.extrapolateToInfinity(l, m);
                    extrap[2 * q] = e.real();
                    extrap[2 * q + 1] = e.imag();
                }
            }
        energy[r] = ex.computeRadiatedEnergy(radii[r]);
    }
    const auto sp = ex.computeEnergySpectrum(sl, sm, radii[sr]);
    for (size_t k = 0; k < sp.size() && (int)k < spec_cap; ++k) {
        spec[2 * k] = sp[k].first;
        spec[2 * k + 1] = sp[k].second;
    }
    return (int)sp.size();
}

// ApparentHorizonFinder::findHorizon (horizon_finder.cpp:310-449). Returns 1 and
// res = area, irreducible mass, spin, equatorial / polar circumference and
// surface[N][3] when found, 0 otherwise.
int ref_find_horizon(const int* n, int ng, const double* lo, const double* hi, const double* u,
                     const double* center, int max_iterations, double tol, int ang_res, double init_r, double* res,
                     double* surface) {
    auto b = block(geo(n, ng, lo, hi));
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    horizon::HorizonParams hp;
    hp.max_iterations = max_iterations;
    hp.tolerance = tol;
    hp.angular_resolution = ang_res;
    hp.initial_guess_radius = init_r;
    horizon::ApparentHorizonFinder f(hp);
    auto r = f.findHorizon(*b, {center[0], center[1], center[2]});
    if (!r) return 0;
    res[0] = r->area;
    res[1] = r->irreducible_mass;
    res[2] = r->spin;
    res[3] = r->circumference_equatorial;
    res[4] = r->circumference_polar;
    for (size_t q = 0; q < r->surface_points.size(); ++q)
        for (int d = 0; d < 3; ++d) surface[3 * q + d] = r->surface_points[q][d];
    return 1;
}

// findAllHorizons (horizon_finder.cpp:452-507): up to cap horizons; per horizon
// out[6 h ..] = centroid x, y, z, area, irreducible mass, spin. Returns the count.
int ref_find_all_horizons(const int* n, int ng, const double* lo, const double* hi, const double* u,
                          int max_iterations, double tol, int ang_res, double init_r, double* out, int cap) {
    auto b = block(geo(n, ng, lo, hi));
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    horizon::HorizonParams hp;
    hp.max_iterations = max_iterations;
    hp.tolerance = tol;
    hp.angular_resolution = ang_res;
    hp.initial_guess_radius = init_r;
    horizon::ApparentHorizonFinder f(hp);
    const auto all = f.findAllHorizons(*b);
    for (size_t q = 0; q < all.size() && (int)q < cap; ++q) {
        for (int d = 0; d < 3; ++d) out[6 * q + d] = all[q].centroid[d];
        out[6 * q + 3] = all[q].area;
        out[6 * q + 4] = all[q].irreducible_mass;
        out[6 * q + 5] = all[q].spin;
    }
    return (int)all.size();
}

// findCommonHorizon (horizon_finder.cpp:510-551) over nh given horizons, each
// hz[3 h ..] = centroid x, y, z and mass_circ[2 h ..] = irreducible mass,
// equatorial circumference (the fields it reads). Same outputs as
// ref_find_horizon, plus the result's centroid and id in cen_id[0..3].
int ref_find_common_horizon(const int* n, int ng, const double* lo, const double* hi, const double* u,
                            const double* hz, const double* mass_circ, int nh, int max_iterations, double tol,
                            int ang_res, double init_r, double* res, double* surface, double* cen_id) {
    auto b = block(geo(n, ng, lo, hi));
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    horizon::HorizonParams hp;
    hp.max_iterations = max_iterations;
    hp.tolerance = tol;
    hp.angular_resolution = ang_res;
    hp.initial_guess_radius = init_r;
    std::vector<horizon::HorizonData> in(nh);
    for (int h = 0; h < nh; ++h) {
        in[h].centroid = {hz[3 * h], hz[3 * h + 1], hz[3 * h + 2]};
        in[h].irreducible_mass = mass_circ[2 * h];
        in[h].circumference_equatorial = mass_circ[2 * h + 1];
    }
    horizon::ApparentHorizonFinder f(hp);
    auto r = f.findCommonHorizon(*b, in);
    if (!r) return 0;
    res[0] = r->area;
    res[1] = r->irreducible_mass;
    res[2] = r->spin;
    res[3] = r->circumference_equatorial;
    res[4] = r->circumference_polar;
    for (size_t q = 0; q < r->surface_points.size(); ++q)
        for (int d = 0; d < 3; ++d) surface[3 * q + d] = r->surface_points[q][d];
    for (int d = 0; d < 3; ++d) cen_id[d] = r->centroid[d];
    cen_id[3] = r->id;
    return 1;
}

// ApparentHorizonFinder::computeSpin (horizon_finder.cpp:553-582) of a horizon
// with the given circumferences (the only fields it reads; the block is unused).
double ref_compute_spin(double c_eq, double c_pol) {
    const int n[3] = {4, 4, 4};
    const double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {1.0, 1.0, 1.0};
    auto b = block(geo(n, 4, lo, hi));
    horizon::HorizonData h;
    h.circumference_equatorial = c_eq;
    h.circumference_polar = c_pol;
    return horizon::ApparentHorizonFinder(horizon::HorizonParams{}).computeSpin(*b, h);
}

// setFlatSpacetime / setGaugeWaveData (ccz4.cpp:1165-1221) on a zeroed block.
void ref_init_flat(const int* n, int ng, const double* lo, const double* hi, double* u) {
    auto b = block(geo(n, ng, lo, hi));
    spacetime::setFlatSpacetime(*b);
    std::memcpy(u, b->flatBuffer(), nbytes(*b));
}

void ref_init_gauge_wave(const int* n, int ng, const double* lo, const double* hi, double* u,
                         double amplitude, double wavelength) {
    auto b = block(geo(n, ng, lo, hi));
    spacetime::setGaugeWaveData(*b, amplitude, wavelength);
    std::memcpy(u, b->flatBuffer(), nbytes(*b));
}

// BrillLindquist::apply / conformalFactor (initial_data.cpp:79-158).
void ref_init_brill_lindquist(const int* n, int ng, const double* lo, const double* hi,
                              double* u, int nbh, const double* mass, const double* pos) {
    auto b = block(geo(n, ng, lo, hi));
    std::vector<initial_data::BlackHoleParams> bhs(nbh);
    for (int i = 0; i < nbh; ++i) {
        bhs[i].mass = mass[i];
        bhs[i].position = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        bhs[i].momentum = {0, 0, 0};
        bhs[i].spin = {0, 0, 0};
    }
    initial_data::BrillLindquist bl(bhs);
    bl.apply(*b);
    std::memcpy(u, b->flatBuffer(), nbytes(*b));
}

double ref_bl_conformal_factor(int nbh, const double* mass, const double* pos, double x,
                               double y, double z) {
    std::vector<initial_data::BlackHoleParams> bhs(nbh);
    for (int i = 0; i < nbh; ++i) {
        bhs[i].mass = mass[i];
        bhs[i].position = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        bhs[i].momentum = {0, 0, 0};
        bhs[i].spin = {0, 0, 0};
    }
    return initial_data::BrillLindquist(bhs).conformalFactor(x, y, z);
}

// AMRHierarchy::prolongate / restrict_data (amr.cpp:484-626). Levels are
// passed explicitly because both operators check coarse.level < fine.level.
void ref_prolongate(const int* cn, const double* clo, const double* chi_, int clevel,
                    const double* uc, const int* fn, const double* flo, const double* fhi,
                    int flevel, double* uf, int ng) {
    auto cb = block(geo(cn, ng, clo, chi_), clevel);
    auto fb = block(geo(fn, ng, flo, fhi), flevel, 1);
    std::memcpy(cb->flatBuffer(), uc, nbytes(*cb));
    std::memcpy(fb->flatBuffer(), uf, nbytes(*fb));
    amr::AMRParams ap;
    SimulationParams sp;
    amr::AMRHierarchy h(ap, sp);
    h.prolongate(*cb, *fb);
    std::memcpy(uf, fb->flatBuffer(), nbytes(*fb));
}

void ref_restrict(const int* fn, const double* flo, const double* fhi, int flevel,
                  const double* uf, const int* cn, const double* clo, const double* chi_,
                  int clevel, double* uc, int ng) {
    auto cb = block(geo(cn, ng, clo, chi_), clevel);
    auto fb = block(geo(fn, ng, flo, fhi), flevel, 1);
    std::memcpy(cb->flatBuffer(), uc, nbytes(*cb));
    std::memcpy(fb->flatBuffer(), uf, nbytes(*fb));
    amr::AMRParams ap;
    SimulationParams sp;
    amr::AMRHierarchy h(ap, sp);
    h.restrict_data(*fb, *cb);
    std::memcpy(uc, cb->flatBuffer(), nbytes(*cb));
}

// AMRHierarchy::fillGhostZones(0) on a one-block level 0 (amr.cpp:400-482).
void ref_fill_level0(const int* n, int ng, const double* lo, const double* hi, double* u) {
    amr::AMRParams ap;
    ap.max_levels = 1;
    SimulationParams sp;
    for (int d = 0; d < 3; ++d) {
        sp.ncells[d] = n[d];
        sp.domain_lo[d] = lo[d];
        sp.domain_hi[d] = hi[d];
    }
    sp.ghost_cells = ng;
    amr::AMRHierarchy h(ap, sp);
    // initialize() prints a level summary to std::cout (amr.cpp:55-57); keep
    // the caller's stdout clean
    std::cout.setstate(std::ios_base::failbit);
    h.initialize([](const GridBlock&, int, int, int) { return false; });
    std::cout.clear();
    GridBlock* b = h.getLevel(0)[0];
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    h.fillGhostZones(0);
    std::memcpy(u, b->flatBuffer(), nbytes(*b));
}

void ref_rk3_steps_matter(const double* p6, const int* n, int ng, const double* lo, const double* hi,
                          double* u, double dt, int nsteps, int bc, const double* rho, const double* Si,
                          const double* Sij, const double* S);

// Wall seconds of the step loop alone of the last ref_rk3_steps(_matter) call
// on this thread: the hierarchy, block allocation and the copies in and out
// are set-up, not the reference's step (the CPU baseline times only this).
static thread_local double g_last_loop_seconds = 0.0;
double ref_last_loop_seconds() { return g_last_loop_seconds; }

// nsteps single-level coarse steps: AMRHierarchy::subcycle(0) (fillGhostZones,
// evolve, fillGhostZones; amr.cpp:303-330) around the spacetime part of
// TimeIntegrator::sspRK3Step (main.cpp:673-689) with the reference
// computeRHSVacuum. bc: 0 = reference zero-gradient + 1/r falloff, 1 = periodic.
void ref_rk3_steps(const double* p6, const int* n, int ng, const double* lo, const double* hi,
                   double* u, double dt, int nsteps, int bc) {
    ref_rk3_steps_matter(p6, n, ng, lo, hi, u, dt, nsteps, bc, nullptr, nullptr, nullptr, nullptr);
}

// The same with matter sources held fixed over the steps (rho[N], Si[N][3],
// Sij[N][6], S[N], N = totalSize()), every stage calling the reference
// computeRHS with them as applyRHS does (main.cpp:300-301); all NULL = vacuum
// (computeRHSVacuum).
void ref_rk3_steps_matter(const double* p6, const int* n, int ng, const double* lo, const double* hi,
                          double* u, double dt, int nsteps, int bc, const double* rho, const double* Si,
                          const double* Sij, const double* S) {
    amr::AMRParams ap;
    ap.max_levels = 1;
    SimulationParams sp;
    for (int d = 0; d < 3; ++d) {
        sp.ncells[d] = n[d];
        sp.domain_lo[d] = lo[d];
        sp.domain_hi[d] = hi[d];
    }
    sp.ghost_cells = ng;
    amr::AMRHierarchy h(ap, sp);
    // initialize() prints a level summary to std::cout (amr.cpp:55-57); keep
    // the caller's stdout clean
    std::cout.setstate(std::ios_base::failbit);
    h.initialize([](const GridBlock&, int, int, int) { return false; });
    std::cout.clear();
    GridBlock& st = *h.getLevel(0)[0];
    std::memcpy(st.flatBuffer(), u, nbytes(st));
    Geo g = geo(n, ng, lo, hi);
    auto stage = block(g, 0, 1);
    auto rhs = block(g, 0, 2);
    spacetime::CCZ4Evolution ev(params(p6));
    const orc_geom og = ogeom(st);
    const long N = static_cast<long>(st.totalSize()) * NUM_SPACETIME_VARS;
    const size_t cells = st.totalSize();
    std::vector<Real> m_rho, m_S;
    std::vector<std::array<Real, DIM>> m_si;
    std::vector<std::array<Real, SYM_TENSOR_COMPS>> m_sij;
    if (rho) {
        m_rho.assign(rho, rho + cells);
        m_S.assign(S, S + cells);
        m_si.resize(cells);
        m_sij.resize(cells);
        for (size_t c = 0; c < cells; ++c) {
            for (int a = 0; a < 3; ++a) m_si[c][a] = Si[3 * c + a];
            for (int a = 0; a < 6; ++a) m_sij[c][a] = Sij[6 * c + a];
        }
    }
    auto rhs_of = [&](const GridBlock& in) {
        if (rho) ev.computeRHS(in, *rhs, m_rho, m_si, m_sij, m_S);
        else ev.computeRHSVacuum(in, *rhs);
    };
    auto level_fill = [&]() {
        if (bc == ORC_BC_PERIODIC) orc_fill_periodic(&og, st.flatBuffer());
        else h.fillGhostZones(0);
    };
    auto outer = [&](GridBlock& b) {
        if (bc == ORC_BC_PERIODIC) orc_fill_periodic(&og, b.flatBuffer());
        else orc_fill_sommerfeld(&og, b.flatBuffer());
    };
    auto combine = [&](GridBlock& d, const GridBlock& s1, Real a1, const GridBlock& s2, Real a2,
                       Real a3) {
        const int is = d.istart();
        for (int v = 0; v < NUM_SPACETIME_VARS; ++v)
            for (int k = is; k < d.iend(2); ++k)
                for (int j = is; j < d.iend(1); ++j)
                    for (int i = is; i < d.iend(0); ++i)
                        d.data(v, i, j, k) = a1 * s1.data(v, i, j, k) + a2 * s2.data(v, i, j, k) +
                            a3 * dt * rhs->data(v, i, j, k);
    };
    (void)N;
    const auto t_loop = std::chrono::steady_clock::now();
    for (int s = 0; s < nsteps; ++s) {
        level_fill();
        rhs_of(st);
        combine(*stage, st, 1.0, st, 0.0, 1.0);
        orc_floors(&og, stage->flatBuffer());
        outer(*stage);
        rhs_of(*stage);
        combine(*stage, st, 0.75, *stage, 0.25, 0.25);
        orc_floors(&og, stage->flatBuffer());
        outer(*stage);
        rhs_of(*stage);
        combine(st, st, 1.0 / 3.0, *stage, 2.0 / 3.0, 2.0 / 3.0);
        orc_floors(&og, st.flatBuffer());
        orc_algebraic(&og, st.flatBuffer());
        outer(st);
        level_fill();
    }
    g_last_loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop).count();
    std::memcpy(u, st.flatBuffer(), nbytes(st));
}

// ---------------------------------------------------------------------------
// The reference Berger-Oliger hierarchy: AMRHierarchy built from tracking
// spheres (amr.cpp:34-301), stepped by AMRHierarchy::subcycle (amr.cpp:303-350)
// with the spacetime part of TimeIntegrator::sspRK3Step as evolve_func
// (main.cpp:86-690, the restated lambdas of ccz4_oracle.c around the reference
// computeRHSVacuum). Regridding inside subcycle follows the regrid_interval
// given at creation (0 = off); ref_hier_regrid runs AMRHierarchy::regrid on
// demand.
// ---------------------------------------------------------------------------
struct RefHier {
    std::unique_ptr<amr::AMRHierarchy> h;
    std::vector<GridBlock*> blocks;  // level order, then creation order
    int tag_var = -1;                // tagger of the in-step regrid (see tagger_of)
    double tag_threshold = 0.0;
};

namespace {
void relist(RefHier* r) {
    r->blocks.clear();
    for (int L = 0; L < r->h->numLevels(); ++L)
        for (GridBlock* b : r->h->getLevel(L)) r->blocks.push_back(b);
}
} // namespace

// regrid_interval > 0 turns on the regrid inside subcycle (amr.cpp:343-349),
// with the tagger of ref_hier_set_tagger (none by default).
void* ref_hier_create(const int* n, const double* lo, const double* hi, int max_levels, int nspheres,
                      const double* centers, const double* radii, const int* min_levels, int regrid_interval) {
    amr::AMRParams ap;
    ap.max_levels = max_levels;
    ap.regrid_interval = regrid_interval;
    SimulationParams sp;
    for (int d = 0; d < 3; ++d) {
        sp.ncells[d] = n[d];
        sp.domain_lo[d] = lo[d];
        sp.domain_hi[d] = hi[d];
    }
    sp.ghost_cells = 4;
    auto* r = new RefHier();
    r->h = std::make_unique<amr::AMRHierarchy>(ap, sp);
    for (int s = 0; s < nspheres; ++s)
        r->h->addTrackingSphere({centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]}, radii[s], min_levels[s]);
    std::cout.setstate(std::ios_base::failbit);
    r->h->initialize([](const GridBlock&, int, int, int) { return false; });
    std::cout.clear();
    relist(r);
    return r;
}

int ref_hier_num_blocks(void* hp) { return (int)static_cast<RefHier*>(hp)->blocks.size(); }

void ref_hier_block_info(void* hp, int i, int* level, int* n, double* lo, double* hi) {
    GridBlock* b = static_cast<RefHier*>(hp)->blocks[i];
    *level = b->getLevel();
    for (int d = 0; d < 3; ++d) {
        n[d] = b->numCells()[d];
        lo[d] = b->lowerCorner()[d];
        hi[d] = b->upperCorner()[d];
    }
}

void ref_hier_get(void* hp, int i, double* u) {
    GridBlock* b = static_cast<RefHier*>(hp)->blocks[i];
    std::memcpy(u, b->flatBuffer(), nbytes(*b));
}

void ref_hier_set(void* hp, int i, const double* u) {
    GridBlock* b = static_cast<RefHier*>(hp)->blocks[i];
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
}

namespace {
amr::TaggingFunction tagger_of(int var, double threshold);
} // namespace

void ref_hier_set_tagger(void* hp, int var, double threshold) {
    RefHier* r = static_cast<RefHier*>(hp);
    r->tag_var = var;
    r->tag_threshold = threshold;
}

// nsteps coarse steps of AMRHierarchy::subcycle(0) (regrids included when the
// interval is set); the block list is re-read afterwards.
void ref_hier_step(void* hp, const double* p6, double dt_coarse, int nsteps) {
    RefHier* r = static_cast<RefHier*>(hp);
    spacetime::CCZ4Evolution ev(params(p6));
    auto evolve = [&](std::vector<GridBlock*>& blocks, Real dt) {
        // stage by stage over all blocks of the level, as sspRK3Step does
        std::vector<std::unique_ptr<GridBlock>> stage, rhs;
        for (GridBlock* b : blocks) {
            stage.push_back(std::make_unique<GridBlock>(b->getId(), b->getLevel(), b->numCells(),
                                                        b->lowerCorner(), b->upperCorner(),
                                                        b->getNumGhost(), NUM_SPACETIME_VARS));
            rhs.push_back(std::make_unique<GridBlock>(b->getId(), b->getLevel(), b->numCells(),
                                                      b->lowerCorner(), b->upperCorner(),
                                                      b->getNumGhost(), NUM_SPACETIME_VARS));
        }
        const double a1[3] = {1.0, 0.75, 1.0 / 3.0}, a2[3] = {0.0, 0.25, 2.0 / 3.0},
                     a3[3] = {1.0, 0.25, 2.0 / 3.0};
        for (int s = 0; s < 3; ++s) {
            for (size_t q = 0; q < blocks.size(); ++q) {
                GridBlock& st = *blocks[q];
                GridBlock& in = s == 0 ? st : *stage[q];
                GridBlock& out = s == 2 ? st : *stage[q];
                const orc_geom og = ogeom(st);
                ev.computeRHSVacuum(in, *rhs[q]);
                const int is = st.istart();
                for (int v = 0; v < NUM_SPACETIME_VARS; ++v)
                    for (int k = is; k < st.iend(2); ++k)
                        for (int j = is; j < st.iend(1); ++j)
                            for (int i = is; i < st.iend(0); ++i)
                                out.data(v, i, j, k) = a1[s] * st.data(v, i, j, k) + a2[s] * in.data(v, i, j, k) +
                                    a3[s] * dt * rhs[q]->data(v, i, j, k);
                orc_floors(&og, out.flatBuffer());
                if (s == 2) orc_algebraic(&og, out.flatBuffer());
                orc_fill_sommerfeld(&og, out.flatBuffer());
            }
        }
    };
    r->h->setLevelDt(0, dt_coarse);
    const amr::TaggingFunction tagger = tagger_of(r->tag_var, r->tag_threshold);
    std::cout.setstate(std::ios_base::failbit);
    for (int s = 0; s < nsteps; ++s) r->h->subcycle(0, evolve, tagger);
    std::cout.clear();
    relist(r);
}

// AMRHierarchy::updateTrackingSpheres (amr.cpp:632-636): new centres of the
// first n tracking spheres.
void ref_hier_update_spheres(void* hp, int n, const double* centers) {
    std::vector<std::array<Real, DIM>> c(n);
    for (int s = 0; s < n; ++s) c[s] = {centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]};
    static_cast<RefHier*>(hp)->h->updateTrackingSpheres(c);
}

namespace {
amr::TaggingFunction tagger_of(int var, double threshold) {
    if (var == static_cast<int>(SpacetimeVar::CHI)) return amr::gradientChiTagger(threshold);
    if (var == static_cast<int>(SpacetimeVar::LAPSE)) return amr::gradientLapseTagger(threshold);
    return [](const GridBlock&, int, int, int) { return false; };
}
} // namespace

// AMRHierarchy::regrid(level, tagger) (amr.cpp:80-301) with gradientChiTagger
// (var 0), gradientLapseTagger (var 18) or a tagger that never tags (any other
// var). The block list is rebuilt (level order, then creation order); returns
// its length.
int ref_hier_regrid(void* hp, int level, int var, double threshold) {
    RefHier* r = static_cast<RefHier*>(hp);
    std::cout.setstate(std::ios_base::failbit);  // regrid prints one line per new block
    r->h->regrid(level, tagger_of(var, threshold));
    std::cout.clear();
    relist(r);
    return (int)r->blocks.size();
}

// gradientChiTagger / gradientLapseTagger (amr.cpp:653-731) over the interior
// cells of one block: the number of tagged cells.
long long ref_tag_count(const int* n, int ng, const double* lo, const double* hi, const double* u, int var,
                        double threshold) {
    auto b = block(geo(n, ng, lo, hi));
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    const amr::TaggingFunction t = tagger_of(var, threshold);
    long long count = 0;
    for (int k = b->istart(2); k < b->iend(2); ++k)
        for (int j = b->istart(1); j < b->iend(1); ++j)
            for (int i = b->istart(0); i < b->iend(0); ++i) count += t(*b, i, j, k) ? 1 : 0;
    return count;
}

// compositeTagger (amr.cpp:723-731) of nt gradient taggers (vars[q], thresholds[q])
// over the interior: the cells it tags.
long long ref_composite_tag_count(const int* n, int ng, const double* lo, const double* hi, const double* u,
                                  int nt, const int* vars, const double* thresholds) {
    auto b = block(geo(n, ng, lo, hi));
    std::memcpy(b->flatBuffer(), u, nbytes(*b));
    std::vector<amr::TaggingFunction> ts;
    for (int q = 0; q < nt; ++q) ts.push_back(tagger_of(vars[q], thresholds[q]));
    const amr::TaggingFunction t = amr::compositeTagger(std::move(ts));
    long long count = 0;
    for (int k = b->istart(2); k < b->iend(2); ++k)
        for (int j = b->istart(1); j < b->iend(1); ++j)
            for (int i = b->istart(0); i < b->iend(0); ++i) count += t(*b, i, j, k) ? 1 : 0;
    return count;
}

void ref_hier_destroy(void* hp) { delete static_cast<RefHier*>(hp); }

} // extern "C"
