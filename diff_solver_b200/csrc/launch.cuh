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

// Kernels index cells and faces with 32-bit integers: (nx + 1)(ny + 1)(nz + 1)
// must stay below 2^32.  Each factor is widened before the + 1, and the
// product is formed one factor at a time so that it cannot wrap.
inline bool valid_grid(const XsGrid& g) {
    if (!(g.nx > 0 && g.ny > 0 && g.nz > 0 && g.cell_size > 0.0f && g.time_step > 0.0f)) return false;
    constexpr unsigned long long kLimit = 1ull << 32;
    const unsigned long long a = g.nx + 1ull, b = g.ny + 1ull, c = g.nz + 1ull;
    if (a >= kLimit || b >= kLimit || c >= kLimit) return false;
    const unsigned long long ab = a * b;  // < 2^64: both factors < 2^32
    return ab < kLimit && ab * c < kLimit;
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
