// Host-side launch helpers shared by the kernel translation units.
#pragma once

#include <mutex>

#include <cuda_runtime.h>

#include "diff_smoke.h"

namespace xs {

// Counts one launch and converts the launch error into a status.
XsStatus check_launch();
// Converts a CUDA runtime status into an XsStatus (without counting).
XsStatus check_cuda(cudaError_t e);

inline bool valid_grid(const XsGrid& g) {
    return g.nx > 0 && g.ny > 0 && g.nz > 0 && g.cell_size > 0.0f && g.time_step > 0.0f &&
           static_cast<unsigned long long>(g.nx + 1) * (g.ny + 1) * (g.nz + 1) < (1ull << 32);
}
inline bool valid(const XsVector& v) { return v.x && v.y && v.z; }
inline bool valid(const XsAdjointVector& v) { return v.x && v.y && v.z; }

// A set-up call that must run once per device (a kernel attribute applies to
// the device and context it was set on), thread-safe.
class DeviceOnce {
public:
    template <class F>
    bool run(F&& f) {
        int device = 0;
        if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) return false;
        std::lock_guard<std::mutex> lock(mu_);
        if (done_[device]) return true;
        if (f() != cudaSuccess) return false;
        done_[device] = true;
        return true;
    }

private:
    static constexpr int kMaxDevices = 64;
    std::mutex mu_;
    bool done_[kMaxDevices] = {};
};

}  // namespace xs
