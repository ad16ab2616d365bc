// Launch accounting and error conversion for the C ABI.
#include <atomic>

#include "launch.cuh"

namespace xs {

namespace {
std::atomic<unsigned long long> g_launches{0};
thread_local int g_last_error = 0;
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

XsStatus check_cuda(cudaError_t e) {
    if (e == cudaSuccess) return XS_OK;
    g_last_error = static_cast<int>(e);
    return XS_CUDA_ERROR;
}

XsStatus check_launch() {
    count_launch();
    return check_cuda(cudaGetLastError());
}

}  // namespace xs

extern "C" {
uint64_t xs_launch_count(void) { return xs::g_launches.load(std::memory_order_relaxed); }
int xs_last_cuda_error(void) { return xs::g_last_error; }
const char* xs_status_string(int status) {
    switch (status) {
        case XS_OK: return "ok";
        case XS_CUDA_ERROR: return "cuda error";
        case XS_NOT_CONVERGED: return "pressure solve did not converge";
        case XS_NUMERICAL_ERROR: return "numerical error (NaN/Inf or breakdown)";
        case XS_INVALID_ARGUMENT: return "invalid argument";
        case XS_TIMEOUT: return "device-side wait timed out";
        case XS_CAPACITY_EXCEEDED: return "grid larger than the entry point's fixed capacity";
        default: return "unknown status";
    }
}
}
