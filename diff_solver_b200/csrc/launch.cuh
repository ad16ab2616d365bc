// Host-side launch helpers shared by the kernel translation units.
#pragma once

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

}  // namespace xs
