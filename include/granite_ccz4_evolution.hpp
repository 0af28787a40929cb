// granite_ccz4_evolution.hpp -- C++17 drop-in over the C ABI of granite_ccz4.h.
//
// Mirrors granite::spacetime::CCZ4Evolution (include/granite/spacetime/ccz4.hpp:49-115
// of GRANITE) method for method, and provides an RK3 step functor with the
// signature of amr::EvolutionStepFunc (include/granite/amr/amr.hpp:43). Header
// only; link libgranite_ccz4.so. The block type is a template parameter so the
// reference's own granite::GridBlock (grid.hpp:44-162) works unchanged: it needs
// numCells(), lowerCorner(), upperCorner(), getNumGhost(), getLevel(), getId(),
// totalSize() and flatBuffer().
//
// Errors: the reference signals none (NaNs propagate, ccz4.cpp); here every
// failed ABI call throws std::runtime_error with the library's message, and a
// context that cannot find an sm_100 device throws at construction.
#pragma once

#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "granite_ccz4.h"

namespace granite_b200 {

// CCZ4Params, ccz4.hpp:25-34
struct CCZ4Params {
    double kappa1 = 0.02;
    double kappa2 = 0.0;
    double eta = 2.0;
    double ko_sigma = 0.1;
    int fd_order = 4;
    bool use_moving_puncture = true;
    double chi_blend_center = 0.05;
    double chi_blend_width = 0.02;
};

namespace detail {
inline granite_ccz4_params to_c(const CCZ4Params& p, int device) {
    granite_ccz4_params c;
    granite_ccz4_default_params(&c);
    c.kappa1 = p.kappa1;
    c.kappa2 = p.kappa2;
    c.eta = p.eta;
    c.ko_sigma = p.ko_sigma;
    c.chi_blend_center = p.chi_blend_center;
    c.chi_blend_width = p.chi_blend_width;
    c.fd_order = p.fd_order;
    c.device = device;
    return c;
}

template <class Block>
granite_block_desc desc_of(const Block& b) {
    granite_block_desc d;
    for (int a = 0; a < 3; ++a) {
        d.ncells[a] = b.numCells()[a];
        d.lo[a] = b.lowerCorner()[a];
        d.hi[a] = b.upperCorner()[a];
    }
    d.nghost = b.getNumGhost();
    d.level = b.getLevel();
    d.id = b.getId();
    return d;
}

class Context {
public:
    Context(const CCZ4Params& p, int device) {
        granite_ccz4_params c = to_c(p, device);
        const int rc = granite_ccz4_create(&c, &h_);
        if (rc != GRANITE_OK)
            throw std::runtime_error("granite_ccz4_create failed (" + std::to_string(rc) +
                                     "): no usable sm_100 GPU or bad parameters");
    }
    ~Context() { granite_ccz4_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    void* get() const { return h_; }
    void check(int rc, const char* what) const {
        if (rc == GRANITE_OK) return;
        char buf[512];
        granite_ccz4_last_error(h_, buf, sizeof(buf));
        throw std::runtime_error(std::string(what) + ": " + buf);
    }

private:
    void* h_ = nullptr;
};
}  // namespace detail

// Same public methods as the reference CCZ4Evolution. The methods are const
// as in the reference, but one object must not be used from two host threads
// at once (one CUDA stream per object).
class CCZ4Evolution {
public:
    explicit CCZ4Evolution(const CCZ4Params& params, int device = 0,
                           int precision = GRANITE_PRECISION_FP64)
        : params_(params), precision_(precision), ctx_(params, device) {}

    // ccz4.hpp:69-74; matter arrays are std::vector<Real>, std::vector<std::array<Real,3>>,
    // std::vector<std::array<Real,6>>, std::vector<Real> sized totalSize()
    template <class Block, class V1, class V3, class V6>
    void computeRHS(const Block& grid, Block& rhs, const V1& rho, const V3& Si, const V6& Sij,
                    const V1& S) const {
        const granite_block_desc d = detail::desc_of(grid);
        ctx_.check(granite_ccz4_compute_rhs_host(ctx_.get(), &d, grid.flatBuffer(), rhs.flatBuffer(),
                                                 rho.data(), Si.data()->data(), Sij.data()->data(),
                                                 S.data(), precision_),
                   "computeRHS");
    }

    // ccz4.hpp:81
    template <class Block>
    void computeRHSVacuum(const Block& grid, Block& rhs) const {
        const granite_block_desc d = detail::desc_of(grid);
        ctx_.check(granite_ccz4_compute_rhs_host(ctx_.get(), &d, grid.flatBuffer(), rhs.flatBuffer(), nullptr,
                                                 nullptr, nullptr, nullptr, precision_),
                   "computeRHSVacuum");
    }

    // ccz4.hpp:90-92; ham and mom are resized to totalSize() like the reference
    template <class Block>
    void computeConstraints(const Block& grid, std::vector<double>& ham,
                            std::vector<std::array<double, 3>>& mom) const {
        const granite_block_desc d = detail::desc_of(grid);
        ham.assign(grid.totalSize(), 0.0);
        mom.assign(grid.totalSize(), {0.0, 0.0, 0.0});
        ctx_.check(granite_ccz4_compute_constraints_host(ctx_.get(), &d, grid.flatBuffer(), ham.data(),
                                                         mom.data()->data()),
                   "computeConstraints");
    }

    // ccz4.hpp:99
    template <class Block>
    void applyDissipation(const Block& grid, Block& rhs) const {
        const granite_block_desc d = detail::desc_of(grid);
        ctx_.check(granite_ccz4_apply_dissipation_host(ctx_.get(), &d, grid.flatBuffer(), rhs.flatBuffer()),
                   "applyDissipation");
    }

    const CCZ4Params& params() const { return params_; }

private:
    CCZ4Params params_;
    int precision_;
    detail::Context ctx_;
};

// Drop-in for the evolve_func the reference passes to AMRHierarchy::subcycle
// (main.cpp:1142-1177): one SSP-RK3 step of all blocks of a level
// (TimeIntegrator::sspRK3Step, main.cpp:86-690, vacuum spacetime part) with the
// reference boundaries. The blocks are kept resident on the device between
// calls as long as the same set of blocks is passed; host data is uploaded
// before and downloaded after every call so the caller's GridBlocks always hold
// the current state (as the reference's do).
template <class Block>
class RK3Step {
public:
    explicit RK3Step(const CCZ4Params& params, int device = 0, int precision = GRANITE_PRECISION_FP64,
                     int bc = GRANITE_BC_REFERENCE)
        : params_(params), device_(device), precision_(precision), bc_(bc) {}

    void operator()(std::vector<Block*>& blocks, double dt) {
        if (!ctx_ || blocks != bound_) bind(blocks);
        if (blocks.empty()) return;
        std::vector<double*> bufs(blocks.size());
        for (size_t i = 0; i < blocks.size(); ++i) bufs[i] = blocks[i]->flatBuffer();
        // the whole level in, one step, the whole level out (one synchronisation)
        ctx_->check(granite_ccz4_upload_all(ctx_->get(), bufs.data()), "upload");
        ctx_->check(granite_ccz4_rk3_step(ctx_->get(), level_, dt, precision_, bc_), "rk3_step");
        ctx_->check(granite_ccz4_download_all(ctx_->get(), bufs.data()), "download");
    }

private:
    void bind(std::vector<Block*>& blocks) {
        ctx_.reset();
        ctx_.reset(new detail::Context(params_, device_));
        level_ = blocks.empty() ? 0 : blocks[0]->getLevel();
        for (Block* b : blocks) {
            granite_block_desc d = detail::desc_of(*b);
            d.level = level_;
            ctx_->check(granite_ccz4_add_block(ctx_->get(), &d, nullptr), "add_block");
        }
        ctx_->check(granite_ccz4_commit(ctx_->get()), "commit");
        bound_ = blocks;
    }

    CCZ4Params params_;
    int device_, precision_, bc_;
    int level_ = 0;
    std::vector<Block*> bound_;
    std::unique_ptr<detail::Context> ctx_;
};

}  // namespace granite_b200
