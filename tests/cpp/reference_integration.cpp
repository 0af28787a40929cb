// The integration code a GRANITE maintainer adds, compiled against the
// reference's own headers and linked with its own grid.cpp / amr.cpp and
// libgranite_ccz4.so (recipe: the `integration` target of oracle/Makefile; run
// by tests/test_reference_integration_cpu.py):
//   - granite_b200::CCZ4Evolution, RK3Step and the diagnostics classes
//     instantiated on granite::GridBlock (ccz4.hpp:49-115, amr.hpp:43,
//     postprocess.hpp:34-69, horizon_finder.hpp:43-87);
//   - the block-list mirror of a reference AMRHierarchy (amr.hpp:64) and the
//     regrid callback of granite_ccz4_hierarchy_step_regrid driving the
//     reference's AMRHierarchy::regrid (amr.cpp:80-301) for the geometry.
// main() builds a reference hierarchy from a tracking sphere on the host and
// checks that detail::desc_of reproduces every block's geometry; the device
// calls are compiled and linked, and run only where a GPU is present (without
// one, granite_ccz4_create must answer GRANITE_ERR_NO_DEVICE).
#include <cstdio>
#include <vector>

#include "granite/amr/amr.hpp"
#include "granite/core/grid.hpp"
#include "granite/core/types.hpp"
#include "granite_b200_diagnostics.hpp"
#include "granite_ccz4_evolution.hpp"

using granite::GridBlock;
namespace amr = granite::amr;

// The operator drop-in: the reference call sites with the wrapper's classes.
void operator_call_sites(GridBlock& st, GridBlock& rhs, GridBlock& prim) {
    using CCZ4Evolution = granite_b200::CCZ4Evolution;
    CCZ4Evolution ccz4(granite_b200::CCZ4Params{});
    const size_t N = st.totalSize();
    std::vector<granite::Real> rho(N), S(N), ham;
    std::vector<std::array<granite::Real, 3>> Si(N), mom;
    std::vector<std::array<granite::Real, 6>> Sij(N);
    granite_b200::MatterSources().computeMatterSources(st, prim, rho, Si, Sij, S);  // grmhd.cpp:1034
    ccz4.computeRHS(st, rhs, rho, Si, Sij, S);                                      // main.cpp:301
    ccz4.computeRHSVacuum(st, rhs);
    ccz4.applyDissipation(st, rhs);
    ccz4.computeConstraints(st, ham, mom);  // main.cpp:1225

    granite_b200::Psi4Extractor gw(granite_b200::GWExtractionParams{});
    gw.extract(st, 0.0);
    (void)gw.computeStrain(2, 2, 100.0);
    granite_b200::ApparentHorizonFinder finder(granite_b200::HorizonParams{});
    auto all = finder.findAllHorizons(st);
    (void)finder.findCommonHorizon(st, all);
    if (auto h = finder.findHorizon(st, {0.0, 0.0, 0.0})) (void)finder.computeSpin(*h);
}

// The evolution-step drop-in (amr.hpp:43) handed to the reference's subcycle.
void evolve_with_reference_subcycle(amr::AMRHierarchy& hierarchy, const amr::TaggingFunction& tagger) {
    granite_b200::RK3Step<GridBlock> gpu_step(granite_b200::CCZ4Params{});
    amr::EvolutionStepFunc evolve_func = [&](std::vector<GridBlock*>& blocks, granite::Real dt) {
        gpu_step(blocks, dt);
    };
    hierarchy.subcycle(0, evolve_func, tagger);
}

// The regrid callback: the reference's AMRHierarchy keeps the geometry, the
// device keeps the state; new blocks are appended to the context.
struct Regrid {
    void* ctx;
    amr::AMRHierarchy* amr;
    double threshold;
};

int on_regrid(void* user, int level, long long /*step_num*/) {
    auto* r = static_cast<Regrid*>(user);
    long long tagged = 0;  // the tagger only decides when no sphere requires level + 1
    if (int e = granite_ccz4_tag_count(r->ctx, level, 0, r->threshold, &tagged)) return e;
    const size_t known = r->amr->getLevel(level + 1).size();
    r->amr->regrid(level, [tagged](const GridBlock&, int, int, int) { return tagged > 0; });
    std::vector<granite_block_desc> add;  // new blocks are appended to their level
    auto lv = r->amr->getLevel(level + 1);
    for (size_t i = known; i < lv.size(); ++i) add.push_back(granite_b200::detail::desc_of(*lv[i]));
    return add.empty() ? 0 : granite_ccz4_regrid_add(r->ctx, add.data(), (int)add.size());
}

int mirror_and_step(void* ctx, amr::AMRHierarchy& hierarchy, double dt, int regrid_interval) {
    for (int lev = 0; lev < hierarchy.numLevels(); ++lev)
        for (GridBlock* b : hierarchy.getLevel(lev)) {
            const granite_block_desc d = granite_b200::detail::desc_of(*b);
            if (int e = granite_ccz4_add_block(ctx, &d, nullptr)) return e;
        }
    if (int e = granite_ccz4_commit(ctx)) return e;
    Regrid regrid{ctx, &hierarchy, 0.1};
    return granite_ccz4_hierarchy_step_regrid(ctx, dt, GRANITE_PRECISION_FP64, GRANITE_AMR_REFERENCE,
                                              regrid_interval, on_regrid, &regrid);
}

int main() {
    amr::AMRParams ap;
    ap.max_levels = 3;
    granite::SimulationParams sp;
    sp.ncells = {16, 16, 16};
    sp.domain_lo = {-8.0, -8.0, -8.0};
    sp.domain_hi = {8.0, 8.0, 8.0};
    amr::AMRHierarchy hierarchy(ap, sp);
    hierarchy.addTrackingSphere({1.0, -0.5, 0.25}, 2.0, 2);
    hierarchy.initialize([](const GridBlock&, int, int, int) { return false; });

    int failures = 0, blocks = 0;
    for (int lev = 0; lev < hierarchy.numLevels(); ++lev)
        for (GridBlock* b : hierarchy.getLevel(lev)) {
            const granite_block_desc d = granite_b200::detail::desc_of(*b);
            bool same = d.nghost == b->getNumGhost() && d.level == b->getLevel() && d.id == b->getId();
            for (int a = 0; a < 3; ++a)
                same = same && d.ncells[a] == b->numCells()[a] && d.lo[a] == b->lowerCorner()[a] &&
                       d.hi[a] == b->upperCorner()[a];
            if (!same) {
                std::printf("FAIL: block %d of level %d: descriptor differs from the GridBlock\n", b->getId(), lev);
                ++failures;
            }
            ++blocks;
        }
    if (hierarchy.numLevels() != 3 || blocks < 3) {
        std::printf("FAIL: expected 3 levels from the tracking sphere, got %d levels, %d blocks\n",
                    hierarchy.numLevels(), blocks);
        ++failures;
    }

    granite_ccz4_params p;
    granite_ccz4_default_params(&p);
    void* ctx = nullptr;
    const int rc = granite_ccz4_create(&p, &ctx);
    if (rc == GRANITE_OK) {
        granite_ccz4_destroy(ctx);
        std::printf("device present: context created and destroyed\n");
    } else if (rc != GRANITE_ERR_NO_DEVICE) {
        std::printf("FAIL: granite_ccz4_create returned %d\n", rc);
        ++failures;
    }
    std::printf("%d blocks on %d levels mirrored\n", blocks, hierarchy.numLevels());
    std::printf(failures ? "FAILED (%d failures)\n" : "OK (%d failures)\n", failures);
    return failures ? 1 : 0;
}
