// granite_b200_diagnostics.hpp -- C++17 drop-ins for the reference's matter
// coupling and diagnostics over the C ABI of granite_ccz4.h.
//
//   MatterSources::computeMatterSources   GRMHDEvolution::computeMatterSources
//                                         (grmhd.hpp:333-338, grmhd.cpp:1034-1103)
//   Psi4Extractor                         postprocess.hpp:34-69 (extract on the
//                                         GPU; the time-series analysis on the host,
//                                         postprocess.cpp:316-475)
//   ApparentHorizonFinder                 horizon_finder.hpp:43-87 (the flow and the
//                                         lapse-minimum scan on the GPU)
//
// Header only; link libgranite_ccz4.so. The block type is a template parameter
// with the reference GridBlock interface (see granite_ccz4_evolution.hpp); the
// primitive block of computeMatterSources has 11 fields. Every failed ABI call
// throws std::runtime_error with the library's message.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <map>
#include <optional>
#include <utility>
#include <vector>

#include "granite_ccz4_evolution.hpp"

namespace granite_b200 {

constexpr double DIAG_PI = 3.14159265358979323846;  // constants::PI

// GRMHDEvolution::computeMatterSources: interior cells of rho, Si, Sij, S from the
// primitives (bit for bit the reference's); the arrays are sized totalSize().
class MatterSources {
public:
    explicit MatterSources(int device = 0) : ctx_(CCZ4Params(), device) {}

    template <class Block, class PBlock, class V1, class V3, class V6>
    void computeMatterSources(const Block& spacetime_grid, const PBlock& prim_grid, V1& rho_src, V3& Si, V6& Sij,
                              V1& S_trace) const {
        const granite_block_desc d = detail::desc_of(spacetime_grid);
        ctx_.check(granite_ccz4_matter_sources_host(ctx_.get(), &d, prim_grid.flatBuffer(), rho_src.data(),
                                                    Si.data()->data(), Sij.data()->data(), S_trace.data()),
                   "computeMatterSources");
    }

private:
    detail::Context ctx_;
};

// postprocess.hpp:23-28
struct GWExtractionParams {
    std::vector<double> extraction_radii = {100.0, 200.0, 300.0, 500.0};
    int l_max = 4;
    int n_theta = 100;
    int n_phi = 200;
};

class Psi4Extractor {
public:
    using Series = std::vector<std::pair<double, std::complex<double>>>;

    explicit Psi4Extractor(const GWExtractionParams& params, int device = 0)
        : params_(params), ctx_(CCZ4Params(), device) {}

    // Psi4Extractor::extract: modes of every radius with a sphere point inside the block
    template <class Block>
    void extract(const Block& spacetime, double time) {
        const granite_block_desc d = detail::desc_of(spacetime);
        const int nr = (int)params_.extraction_radii.size();
        const int nm = (params_.l_max + 1) * (params_.l_max + 1) - 4;
        std::vector<double> modes((size_t)nr * nm * 2);
        std::vector<int> npts(nr);
        ctx_.check(granite_ccz4_psi4_modes_host(ctx_.get(), &d, spacetime.flatBuffer(),
                                                params_.extraction_radii.data(), nr, params_.n_theta,
                                                params_.n_phi, params_.l_max, modes.data(), npts.data()),
                   "Psi4Extractor::extract");
        for (int r = 0; r < nr; ++r) {
            if (npts[r] == 0) continue;  // no sphere point inside the block: nothing recorded
            int q = 0;
            for (int l = 2; l <= params_.l_max; ++l)
                for (int m = -l; m <= l; ++m, ++q) {
                    const std::complex<double> v(modes[2 * ((size_t)r * nm + q)], modes[2 * ((size_t)r * nm + q) + 1]);
                    Series& s = data_[params_.extraction_radii[r]][{l, m}];
                    if (!s.empty() && s.back().first == time)
                        s.back().second += v;
                    else
                        s.push_back({time, v});
                }
        }
    }

    std::complex<double> getMode(int l, int m, double r_ext) const {
        const Series& s = getTimeSeries(l, m, r_ext);
        return s.empty() ? std::complex<double>(0.0, 0.0) : s.back().second;
    }

    // trapezoid double integration (postprocess.cpp:328-353)
    std::complex<double> computeStrain(int l, int m, double r_ext) const {
        const Series& s = getTimeSeries(l, m, r_ext);
        if (s.size() < 3) return {0.0, 0.0};
        std::complex<double> h_dot{0.0, 0.0}, h{0.0, 0.0};
        for (size_t i = 1; i < s.size(); ++i) {
            const double dt = s[i].first - s[i - 1].first;
            h_dot += 0.5 * (s[i].second + s[i - 1].second) * dt;
            h += h_dot * dt;
        }
        return h;
    }

    // postprocess.cpp:355-377
    double computeRadiatedEnergy(double r_ext) const {
        auto it = data_.find(r_ext);
        if (it == data_.end()) return 0.0;
        double E = 0.0;
        for (const auto& kv : it->second) {
            const Series& s = kv.second;
            if (s.size() < 2) continue;
            std::complex<double> hdot{0.0, 0.0};
            for (size_t i = 1; i < s.size(); ++i) {
                const double dt = s[i].first - s[i - 1].first;
                hdot += 0.5 * (s[i].second + s[i - 1].second) * dt;
                E += std::norm(hdot) * dt;
            }
        }
        return r_ext * r_ext / (16.0 * DIAG_PI) * E;
    }

    // the reference returns zero (postprocess.cpp:379-385)
    std::array<double, 3> computeRadiatedMomentum(double) const { return {0.0, 0.0, 0.0}; }

    // postprocess.cpp:387-433
    std::vector<std::pair<double, double>> computeEnergySpectrum(int l, int m, double r_ext) const {
        const Series& s = getTimeSeries(l, m, r_ext);
        const size_t N = s.size();
        if (N < 2) return {};
        const double T = s.back().first - s.front().first;
        const double dt = T / (double)(N > 1 ? N - 1 : 1);
        std::vector<std::complex<double>> h(N, {0.0, 0.0});
        std::complex<double> h_dot{0.0, 0.0}, h_val{0.0, 0.0};
        for (size_t i = 1; i < N; ++i) {
            const double dti = s[i].first - s[i - 1].first;
            h_dot += 0.5 * (s[i].second + s[i - 1].second) * dti;
            h_val += h_dot * dti;
            h[i] = h_val;
        }
        std::vector<std::pair<double, double>> out;
        const int nf = std::min((int)N / 2, 500);
        const double df = 1.0 / T;
        for (int k = 0; k < nf; ++k) {
            const double f = k * df;
            std::complex<double> ht{0.0, 0.0};
            for (size_t i = 0; i < N; ++i) {
                const double phase = -2.0 * DIAG_PI * f * s[i].first;
                ht += h[i] * std::complex<double>(std::cos(phase), std::sin(phase)) * dt;
            }
            out.push_back({f, (DIAG_PI * r_ext * r_ext / 2.0) * f * f * std::norm(ht)});
        }
        return out;
    }

    // Richardson extrapolation over the two outermost radii (postprocess.cpp:435-456)
    std::complex<double> extrapolateToInfinity(int l, int m) const {
        const auto& radii = params_.extraction_radii;
        if (radii.size() < 2) return getMode(l, m, radii.empty() ? 0.0 : radii.back());
        const double r1 = radii[radii.size() - 2], r2 = radii.back();
        const auto p1 = getMode(l, m, r1), p2 = getMode(l, m, r2);
        const double denom = r1 * r1 - r2 * r2;
        if (std::abs(denom) < 1.0e-12) return p2;
        return (r1 * r1 * p2 - r2 * r2 * p1) / denom;
    }

    const Series& getTimeSeries(int l, int m, double r_ext) const {
        static const Series empty;
        auto it = data_.find(r_ext);
        if (it == data_.end()) return empty;
        auto jt = it->second.find({l, m});
        return jt == it->second.end() ? empty : jt->second;
    }

private:
    GWExtractionParams params_;
    detail::Context ctx_;
    std::map<double, std::map<std::pair<int, int>, Series>> data_;
};

// horizon_finder.hpp:17-41
struct HorizonParams {
    int max_iterations = 200;
    double tolerance = 1.0e-10;
    int angular_resolution = 50;
    double initial_guess_radius = 1.0;
    int find_every = 10;
};

struct HorizonData {
    int id = 0;
    std::array<double, 3> centroid{};
    double area = 0.0, irreducible_mass = 0.0, spin = 0.0;
    std::array<double, 3> spin_axis{0.0, 0.0, 1.0};
    double circumference_equatorial = 0.0, circumference_polar = 0.0;
    std::vector<std::array<double, 3>> surface_points;
};

class ApparentHorizonFinder {
public:
    explicit ApparentHorizonFinder(const HorizonParams& params, int device = 0)
        : params_(params), device_(device), ctx_(CCZ4Params(), device) {}

    template <class Block>
    std::optional<HorizonData> findHorizon(const Block& spacetime, std::array<double, 3> center) const {
        const granite_block_desc d = detail::desc_of(spacetime);
        const granite_horizon_params p = cparams(params_);
        const int n = params_.angular_resolution;
        std::vector<double> radii((size_t)n * 2 * n);
        granite_horizon hz;
        ctx_.check(granite_ccz4_find_horizon_host(ctx_.get(), &d, spacetime.flatBuffer(), &p, center.data(), &hz,
                                                  radii.data()),
                   "findHorizon");
        if (!hz.found) return std::nullopt;
        return data_of(hz, &radii);
    }

    // horizon_finder.cpp:452-507 (the block is made resident for the scan)
    template <class Block>
    std::vector<HorizonData> findAllHorizons(const Block& spacetime) const {
        detail::Context c(CCZ4Params(), device_);
        granite_block_desc d = detail::desc_of(spacetime);
        c.check(granite_ccz4_add_block(c.get(), &d, nullptr), "add_block");
        c.check(granite_ccz4_commit(c.get()), "commit");
        c.check(granite_ccz4_upload_block(c.get(), 0, spacetime.flatBuffer()), "upload");
        const granite_horizon_params p = cparams(params_);
        std::vector<granite_horizon> hz(64);
        int n = 0;
        c.check(granite_ccz4_find_all_horizons(c.get(), 0, &p, hz.data(), (int)hz.size(), &n), "findAllHorizons");
        std::vector<HorizonData> out;
        for (int i = 0; i < std::min(n, (int)hz.size()); ++i) out.push_back(data_of(hz[i], nullptr));
        return out;
    }

    // horizon_finder.cpp:510-551
    template <class Block>
    std::optional<HorizonData> findCommonHorizon(const Block& spacetime, const std::vector<HorizonData>& hs) const {
        if (hs.size() < 2) return std::nullopt;
        double total = 0.0;
        std::array<double, 3> cc{0.0, 0.0, 0.0};
        for (const auto& h : hs) {
            for (int d = 0; d < 3; ++d) cc[d] += h.irreducible_mass * h.centroid[d];
            total += h.irreducible_mass;
        }
        if (total < 1.0e-14) return std::nullopt;
        for (int d = 0; d < 3; ++d) cc[d] /= total;
        double max_r = 0.0;
        for (const auto& h : hs) {
            double dist = 0.0;
            for (int d = 0; d < 3; ++d) dist += (h.centroid[d] - cc[d]) * (h.centroid[d] - cc[d]);
            max_r = std::max(max_r, std::sqrt(dist) + h.circumference_equatorial / (2.0 * DIAG_PI));
        }
        HorizonParams cp = params_;
        cp.initial_guess_radius = 1.2 * max_r;
        auto r = ApparentHorizonFinder(cp, device_).findHorizon(spacetime, cc);
        if (r) r->id = (int)hs.size();
        return r;
    }

    // horizon_finder.cpp:553-582: spin from the circumference ratio
    double computeSpin(const HorizonData& h) const {
        if (h.circumference_equatorial < 1.0e-12) return 0.0;
        const double ratio = h.circumference_polar / h.circumference_equatorial;
        if (ratio <= 1.0) return 0.0;
        if (ratio >= DIAG_PI / 2.0) return 1.0;
        return (ratio - 1.0) / (DIAG_PI / 2.0 - 1.0);
    }

private:
    static granite_horizon_params cparams(const HorizonParams& h) {
        granite_horizon_params p;
        p.max_iterations = h.max_iterations;
        p.tolerance = h.tolerance;
        p.angular_resolution = h.angular_resolution;
        p.initial_guess_radius = h.initial_guess_radius;
        return p;
    }

    HorizonData data_of(const granite_horizon& hz, const std::vector<double>* radii) const {
        HorizonData h;
        h.id = hz.id;
        for (int d = 0; d < 3; ++d) h.centroid[d] = hz.centroid[d];
        h.area = hz.area;
        h.irreducible_mass = hz.irreducible_mass;
        h.spin = hz.spin;
        h.circumference_equatorial = hz.circumference_equatorial;
        h.circumference_polar = hz.circumference_polar;
        if (radii) {  // surface points on the finder's angular grid (horizon_finder.cpp:292-300, 384-395)
            const int nth = params_.angular_resolution, nph = 2 * nth;
            for (int i = 0; i < nth; ++i) {
                const double th = DIAG_PI * (i + 0.5) / nth, sth = std::sin(th), cth = std::cos(th);
                for (int j = 0; j < nph; ++j) {
                    const double ph = 2.0 * DIAG_PI * j / nph;
                    const double r = (*radii)[(size_t)i * nph + j];
                    h.surface_points.push_back({h.centroid[0] + r * sth * std::cos(ph),
                                                h.centroid[1] + r * sth * std::sin(ph), h.centroid[2] + r * cth});
                }
            }
        }
        return h;
    }

    HorizonParams params_;
    int device_;
    detail::Context ctx_;
};

}  // namespace granite_b200
