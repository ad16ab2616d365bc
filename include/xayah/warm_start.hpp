// xayah::smoke::WarmStartNetwork -- RAII owner of the learned pressure warm
// start (no reference counterpart) for C++ callers.
//
// The network lives on the device (libdiffsmoke.so, xs_warm_start_*); this
// class only owns the handle, moves parameters between host and device and
// forwards training and inference calls on the caller's stream.  Hand it to
// ExecutionContext::set_learned_warm_start to warm-start a model's forward
// pressure solves.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <utility>
#include <vector>

#include "diff_smoke.h"
#include "xayah/smoke.hpp"

namespace xayah::smoke {

class WarmStartNetwork {
public:
    // Network grid nx x ny x nz (multiples of 8; the coarsest level must still
    // tile into 128-voxel planes); `factor` = fluid grid / network grid.
    WarmStartNetwork(std::uint32_t nx, std::uint32_t ny, std::uint32_t nz, std::uint32_t max_batch = 1, std::uint32_t factor = 1,
                     std::uint64_t seed = 0, cudaStream_t stream = nullptr)
        : stream_(stream) {
        check(xs_warm_start_create(&net_, max_batch, nx, ny, nz, factor), "xs_warm_start_create");
        check(xs_warm_start_initialize(net_, stream_, seed), "xs_warm_start_initialize");
    }
    WarmStartNetwork(const WarmStartNetwork&) = delete;
    WarmStartNetwork& operator=(const WarmStartNetwork&) = delete;
    WarmStartNetwork(WarmStartNetwork&& o) noexcept : net_(std::exchange(o.net_, nullptr)), stream_(o.stream_) {}
    WarmStartNetwork& operator=(WarmStartNetwork&& o) noexcept {
        if (this != &o) {
            reset();
            net_ = std::exchange(o.net_, nullptr);
            stream_ = o.stream_;
        }
        return *this;
    }
    ~WarmStartNetwork() { reset(); }

    [[nodiscard]] XsWarmStartNet* native() const noexcept { return net_; }
    [[nodiscard]] static std::size_t parameter_count() noexcept { return xs_warm_start_parameter_count(); }

    [[nodiscard]] std::vector<float> parameters() const {
        std::vector<float> p(parameter_count());
        check(xs_warm_start_get_parameters(net_, stream_, p.data()), "xs_warm_start_get_parameters");
        return p;
    }
    void set_parameters(const std::vector<float>& p) {
        if (p.size() != parameter_count()) throw std::invalid_argument("warm-start parameter count mismatch");
        check(xs_warm_start_set_parameters(net_, stream_, p.data()), "xs_warm_start_set_parameters");
    }

    // One Adam step on a batch of (rhs, pressure) pairs on the network grid
    // (device arrays [batch][cells]); the loss lands in *loss (device, may be null).
    void train_step(std::uint32_t batch, const float* rhs, const float* pressure, float learning_rate, double* loss = nullptr) {
        check(xs_warm_start_train_step(net_, stream_, batch, rhs, pressure, learning_rate, loss), "xs_warm_start_train_step");
    }
    void predict(std::uint32_t batch, const float* rhs, float* guess) {
        check(xs_warm_start_predict(net_, stream_, batch, rhs, guess), "xs_warm_start_predict");
    }
    // Synchronises; throws if a bounded device wait expired.
    void check_status() { check(xs_warm_start_status(net_, stream_), "xs_warm_start_status"); }

private:
    void reset() noexcept {
        if (net_) xs_warm_start_destroy(net_);
        net_ = nullptr;
    }
    XsWarmStartNet* net_{nullptr};
    cudaStream_t stream_{nullptr};
};

}  // namespace xayah::smoke
