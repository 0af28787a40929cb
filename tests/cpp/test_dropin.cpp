// C++ drop-in check: the assertions of the reference's own unit tests
// (tests/spacetime/test_ccz4_flat.cpp, tests/spacetime/test_gauge_wave.cpp of
// GRANITE), run against granite_b200::CCZ4Evolution from
// include/granite_ccz4_evolution.hpp on a block type with the reference
// GridBlock interface. Built and run by tests/test_cpp_dropin_gpu.py.
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

#include "granite_ccz4_evolution.hpp"

namespace {

// Minimal block with the reference GridBlock interface and layout (grid.hpp).
class Block {
public:
    Block(int id, int level, std::array<int, 3> n, std::array<double, 3> lo, std::array<double, 3> hi,
          int ng, int nv)
        : id_(id), level_(level), ng_(ng), nv_(nv), n_(n), lo_(lo), hi_(hi) {
        for (int d = 0; d < 3; ++d) dx_[d] = (hi_[d] - lo_[d]) / n_[d];
        data_.assign((size_t)nv_ * totalSize(), 0.0);
    }
    int getId() const { return id_; }
    int getLevel() const { return level_; }
    int getNumGhost() const { return ng_; }
    int totalCells(int d) const { return n_[d] + 2 * ng_; }
    size_t totalSize() const { return (size_t)totalCells(0) * totalCells(1) * totalCells(2); }
    double dx(int d) const { return dx_[d]; }
    double x(int d, int i) const { return lo_[d] + ((double)i - ng_ + 0.5) * dx_[d]; }
    int istart() const { return ng_; }
    int iend(int d) const { return ng_ + n_[d]; }
    double& data(int v, int i, int j, int k) {
        return data_[(size_t)v * totalSize() + i + (size_t)totalCells(0) * (j + (size_t)totalCells(1) * k)];
    }
    double data(int v, int i, int j, int k) const {
        return data_[(size_t)v * totalSize() + i + (size_t)totalCells(0) * (j + (size_t)totalCells(1) * k)];
    }
    const std::array<int, 3>& numCells() const { return n_; }
    const std::array<double, 3>& lowerCorner() const { return lo_; }
    const std::array<double, 3>& upperCorner() const { return hi_; }
    double* flatBuffer() { return data_.data(); }
    const double* flatBuffer() const { return data_.data(); }

private:
    int id_, level_, ng_, nv_;
    std::array<int, 3> n_;
    std::array<double, 3> lo_, hi_, dx_;
    std::vector<double> data_;
};

enum { CHI = 0, GXX = 1, GXY = 2, GXZ = 3, GYY = 4, GYZ = 5, GZZ = 6, KTR = 13, THETA = 17, LAPSE = 18,
       SHIFTX = 19 };

void set_flat(Block& g) {  // setFlatSpacetime, ccz4.cpp:1165-1188
    for (int k = 0; k < g.totalCells(2); ++k)
        for (int j = 0; j < g.totalCells(1); ++j)
            for (int i = 0; i < g.totalCells(0); ++i) {
                g.data(CHI, i, j, k) = 1.0;
                g.data(GXX, i, j, k) = 1.0;
                g.data(GYY, i, j, k) = 1.0;
                g.data(GZZ, i, j, k) = 1.0;
                g.data(LAPSE, i, j, k) = 1.0;
            }
}

void set_gauge_wave(Block& g, double A, double L) {  // setGaugeWaveData, ccz4.cpp:1190-1221
    for (int k = 0; k < g.totalCells(2); ++k)
        for (int j = 0; j < g.totalCells(1); ++j)
            for (int i = 0; i < g.totalCells(0); ++i) {
                const double H = A * std::sin(2.0 * 3.14159265358979323846 * g.x(0, i) / L);
                const double chi = std::pow(1.0 + H, -1.0 / 3.0);
                g.data(CHI, i, j, k) = chi;
                g.data(GXX, i, j, k) = (1.0 + H) * chi;
                g.data(GYY, i, j, k) = chi;
                g.data(GZZ, i, j, k) = chi;
                g.data(LAPSE, i, j, k) = std::sqrt(1.0 + H);
            }
}

int failures = 0;
#define EXPECT(cond, msg)                                      \
    do {                                                       \
        if (!(cond)) {                                         \
            std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, msg); \
            ++failures;                                        \
        }                                                      \
    } while (0)

double max_abs(const Block& b, int lo_off, int hi_off) {
    double m = 0.0;
    for (int v = 0; v < 22; ++v)
        for (int k = b.istart() + lo_off; k < b.iend(2) - hi_off; ++k)
            for (int j = b.istart() + lo_off; j < b.iend(1) - hi_off; ++j)
                for (int i = b.istart() + lo_off; i < b.iend(0) - hi_off; ++i) m = std::fmax(m, std::fabs(b.data(v, i, j, k)));
    return m;
}

}  // namespace

int main() {
    using granite_b200::CCZ4Evolution;
    using granite_b200::CCZ4Params;
    const std::array<int, 3> n{32, 32, 32};
    const std::array<double, 3> lo{-10, -10, -10}, hi{10, 10, 10};

    // test_ccz4_flat.cpp:44-63 RHSIsZeroForFlatSpacetime
    Block grid(0, 0, n, lo, hi, 4, 22), rhs(1, 0, n, lo, hi, 4, 22);
    set_flat(grid);
    CCZ4Params p0;
    p0.ko_sigma = 0.0;
    CCZ4Evolution ccz4(p0);
    ccz4.computeRHSVacuum(grid, rhs);
    EXPECT(max_abs(rhs, 1, 1) < 1e-10, "flat RHS not zero");

    // :65-104 RHSMatchesVacuumOverload (bit-exact)
    {
        Block r1(2, 0, n, lo, hi, 4, 22), r2(3, 0, n, lo, hi, 4, 22);
        const size_t N = grid.totalSize();
        std::vector<double> rho(N, 0.0), S(N, 0.0);
        std::vector<std::array<double, 3>> Si(N, {0, 0, 0});
        std::vector<std::array<double, 6>> Sij(N, {0, 0, 0, 0, 0, 0});
        ccz4.computeRHS(grid, r1, rho, Si, Sij, S);
        ccz4.computeRHSVacuum(grid, r2);
        bool same = true;
        for (size_t q = 0; q < 22 * N; ++q) same = same && r1.flatBuffer()[q] == r2.flatBuffer()[q];
        EXPECT(same, "computeRHS with zero sources differs from computeRHSVacuum");
    }

    // :106-150 constraints vanish for flat
    {
        std::vector<double> ham;
        std::vector<std::array<double, 3>> mom;
        ccz4.computeConstraints(grid, ham, mom);
        double mh = 0, mm = 0;
        for (size_t q = 0; q < ham.size(); ++q) {
            mh = std::fmax(mh, std::fabs(ham[q]));
            for (int a = 0; a < 3; ++a) mm = std::fmax(mm, std::fabs(mom[q][a]));
        }
        EXPECT(mh < 1e-10 && mm < 1e-10, "flat constraints not zero");
    }

    // :192-230 KO on constant data < 1e-12
    {
        CCZ4Params pk;
        pk.ko_sigma = 0.35;
        CCZ4Evolution ko(pk);
        Block r(4, 0, n, lo, hi, 4, 22);
        ko.computeRHSVacuum(grid, r);
        EXPECT(max_abs(r, 3, 3) < 1e-12, "KO on a constant field not zero");
    }

    // :240-286 KO bounded on a gauge wave; test_gauge_wave.cpp:91-127
    {
        const std::array<int, 3> ng{64, 8, 8};
        const std::array<double, 3> glo{0, 0, 0}, ghi{1.0, 0.125, 0.125};
        Block gw(10, 0, ng, glo, ghi, 4, 22), gr(11, 0, ng, glo, ghi, 4, 22);
        set_gauge_wave(gw, 0.01, 1.0);
        CCZ4Params pk;
        pk.ko_sigma = 0.35;
        CCZ4Evolution(pk).computeRHSVacuum(gw, gr);
        const double m = max_abs(gr, 3, 3);
        EXPECT(std::isfinite(m) && m > 0.0 && m < 50.0, "KO on the gauge wave not finite/bounded");
        // applyDissipation alone on zero RHS equals the KO part
        Block gk(12, 0, ng, glo, ghi, 4, 22);
        CCZ4Evolution(pk).applyDissipation(gw, gk);
        EXPECT(max_abs(gk, 3, 3) > 0.0 && max_abs(gk, 3, 3) < 50.0, "applyDissipation out of bounds");
    }

    // :298-331 selective advection finite in a flat region with a shift
    {
        Block g2(0, 0, n, lo, hi, 4, 22), r2(1, 0, n, lo, hi, 4, 22);
        set_flat(g2);
        for (int k = 0; k < g2.totalCells(2); ++k)
            for (int j = 0; j < g2.totalCells(1); ++j)
                for (int i = 0; i < g2.totalCells(0); ++i) {
                    g2.data(LAPSE, i, j, k) = 1.0 + 0.01 * g2.x(0, i);
                    g2.data(SHIFTX, i, j, k) = 0.5;
                }
        ccz4.computeRHSVacuum(g2, r2);
        EXPECT(std::isfinite(max_abs(r2, 2, 2)), "advection with chi = 1 not finite");
    }

    // one RK3 step through the EvolutionStepFunc-shaped functor
    {
        Block g3(0, 0, {24, 24, 24}, {-3, -3, -3}, {3, 3, 3}, 4, 22);
        set_flat(g3);
        std::vector<Block*> blocks{&g3};
        granite_b200::RK3Step<Block> step(CCZ4Params{});
        step(blocks, 0.05);
        step(blocks, 0.05);
        EXPECT(std::fabs(g3.data(CHI, 10, 10, 10) - 1.0) < 1e-12, "flat state drifted under RK3");
    }

    std::printf("%s (%d failures)\n", failures ? "FAILED" : "OK", failures);
    return failures ? 1 : 0;
}
