// C++ drop-ins of include/granite_b200_diagnostics.hpp on a block type with the
// reference GridBlock interface: the matter sources of fluids whose ADM
// sources are known in closed form, Psi4 modes of flat space, and the horizon
// finder's answers on flat space. Built and run by
// tests/test_cpp_diagnostics_gpu.py.
#include <cmath>
#include <cstdio>
#include <vector>

#include "granite_b200_diagnostics.hpp"

namespace {

class Block {  // reference GridBlock interface and layout (grid.hpp)
public:
    Block(int id, int level, std::array<int, 3> n, std::array<double, 3> lo, std::array<double, 3> hi, int ng, int nv)
        : id_(id), level_(level), ng_(ng), n_(n), lo_(lo), hi_(hi) {
        data_.assign((size_t)nv * totalSize(), 0.0);
    }
    int getId() const { return id_; }
    int getLevel() const { return level_; }
    int getNumGhost() const { return ng_; }
    int totalCells(int d) const { return n_[d] + 2 * ng_; }
    size_t totalSize() const { return (size_t)totalCells(0) * totalCells(1) * totalCells(2); }
    size_t cell(int i, int j, int k) const { return i + (size_t)totalCells(0) * (j + (size_t)totalCells(1) * k); }
    double& data(int v, int i, int j, int k) { return data_[(size_t)v * totalSize() + cell(i, j, k)]; }
    const std::array<int, 3>& numCells() const { return n_; }
    const std::array<double, 3>& lowerCorner() const { return lo_; }
    const std::array<double, 3>& upperCorner() const { return hi_; }
    double* flatBuffer() { return data_.data(); }
    const double* flatBuffer() const { return data_.data(); }

private:
    int id_, level_, ng_;
    std::array<int, 3> n_;
    std::array<double, 3> lo_, hi_;
    std::vector<double> data_;
};

int failures = 0;
void check(bool ok, const char* what) {
    if (!ok) {
        ++failures;
        std::printf("FAIL: %s\n", what);
    }
}
bool close(double a, double b, double tol = 1e-14) { return std::abs(a - b) <= tol * std::max(1.0, std::abs(b)); }

void set_flat(Block& g) {  // setFlatSpacetime (ccz4.cpp:1165-1188)
    for (int k = 0; k < g.totalCells(2); ++k)
        for (int j = 0; j < g.totalCells(1); ++j)
            for (int i = 0; i < g.totalCells(0); ++i)
                for (int v : {0, 1, 4, 6, 18}) g.data(v, i, j, k) = 1.0;
}

}  // namespace

int main() {
    using namespace granite_b200;
    const std::array<int, 3> n{12, 10, 8};
    const std::array<double, 3> lo{-1, -1, -1}, hi{1, 1, 1};

    // matter sources of a static fluid and of a boosted one, B = 0
    {
        Block st(0, 0, n, lo, hi, 4, 22), prim(1, 0, n, lo, hi, 4, 11);
        const size_t N = st.totalSize();
        std::vector<double> rho(N, -7.0), S(N, -7.0);
        std::vector<std::array<double, 3>> Si(N, {-7.0, -7.0, -7.0});
        std::vector<std::array<double, 6>> Sij(N);
        for (auto& a : Sij) a.fill(-7.0);
        const double r0 = 0.5, p0 = 0.2, e0 = 0.3, vx = 0.6;
        for (int k = 4; k < 12; ++k)
            for (int j = 4; j < 14; ++j)
                for (int i = 4; i < 16; ++i) {
                    prim.data(0, i, j, k) = r0;
                    prim.data(1, i, j, k) = i < 10 ? 0.0 : vx;
                    prim.data(4, i, j, k) = p0;
                    prim.data(8, i, j, k) = e0;
                }
        MatterSources().computeMatterSources(st, prim, rho, Si, Sij, S);
        const double h = 1.0 + e0 + p0 / r0, W2 = 1.0 / (1.0 - vx * vx);
        const size_t c0 = st.cell(5, 6, 7), c1 = st.cell(12, 6, 7);
        check(close(rho[c0], r0 * h - p0) && close(S[c0], 3 * p0) && Si[c0][0] == 0.0 && close(Sij[c0][0], p0) &&
                  Sij[c0][1] == 0.0 && close(Sij[c0][3], p0),
              "static fluid: rho = rho0 (1 + eps), S_ij = p delta_ij");
        check(close(rho[c1], r0 * h * W2 - p0) && close(Si[c1][0], r0 * h * W2 * vx) &&
                  close(Sij[c1][0], r0 * h * W2 * vx * vx + p0) && close(Sij[c1][3], p0) &&
                  close(S[c1], r0 * h * W2 * vx * vx + 3 * p0),
              "boosted fluid: rho h W^2 - p, rho h W^2 v, rho h W^2 v v + p delta");
        check(rho[st.cell(0, 0, 0)] == -7.0 && S[st.cell(3, 5, 5)] == -7.0 && Si[st.cell(16, 5, 5)][2] == -7.0,
              "cells outside the interior keep their values");
    }

    // Psi4 of flat space: every mode of every radius inside the block is zero
    {
        Block g(0, 0, {24, 24, 24}, {-6, -6, -6}, {6, 6, 6}, 4, 22);
        set_flat(g);
        GWExtractionParams gp;
        gp.extraction_radii = {2.0, 4.0, 20.0};
        gp.l_max = 3;
        gp.n_theta = 12;
        gp.n_phi = 24;
        Psi4Extractor ex(gp);
        ex.extract(g, 0.0);
        ex.extract(g, 0.5);
        check(ex.getTimeSeries(2, 2, 2.0).size() == 2 && ex.getMode(3, -3, 4.0) == std::complex<double>(0.0, 0.0),
              "flat space: zero modes, one entry per time");
        check(ex.getTimeSeries(2, 0, 20.0).empty(), "a sphere outside the block records nothing");
        check(ex.computeRadiatedEnergy(2.0) == 0.0 && ex.extrapolateToInfinity(2, 1) == std::complex<double>(0, 0),
              "analysis of zero modes");
    }

    // horizons in flat space. The reference's expansion differentiates the unit
    // normal along the fixed coordinate direction of each surface point, which is
    // constant in flat space: Theta = 0 and the flow stops at its first iteration
    // with the initial sphere (area 4 pi r^2 to the midpoint rule, both
    // circumferences 2 pi r); no lapse minimum is below 0.5, so findAll finds none.
    {
        Block g(0, 0, {20, 20, 20}, {-2, -2, -2}, {2, 2, 2}, 4, 22);
        set_flat(g);
        HorizonParams hp;
        hp.max_iterations = 50;
        hp.angular_resolution = 6;
        ApparentHorizonFinder f(hp);
        const auto hz = f.findHorizon(g, {0.0, 0.0, 0.0});
        check(hz.has_value() && std::abs(hz->area - 4.0 * DIAG_PI) < 0.02 * 4.0 * DIAG_PI &&
                  close(hz->circumference_equatorial, 2.0 * DIAG_PI, 1e-12) &&
                  close(hz->circumference_polar, 2.0 * DIAG_PI, 1e-12) && std::abs(hz->spin) < 1e-12 &&
                  hz->surface_points.size() == 72,
              "flat space: the initial unit sphere");
        check(f.findAllHorizons(g).empty(), "no lapse minimum below 0.5 in flat space");
        HorizonData h;
        h.circumference_equatorial = 2.0;
        h.circumference_polar = 2.5;
        check(close(f.computeSpin(h), 0.25 / (DIAG_PI / 2.0 - 1.0)), "spin from the circumference ratio");
        check(!f.findCommonHorizon(g, std::vector<HorizonData>{h}).has_value(), "a common horizon needs two");
    }

    std::printf("OK (%d failures)\n", failures);
    return failures ? 1 : 0;
}
