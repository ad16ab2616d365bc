// A pressure solve for callers that cannot allocate device memory.
//
// Some hosts of this solver never call cudaMalloc themselves: code that runs
// under a caller-owned memory budget (an engine with its own pooled
// allocator that forbids stray allocations), code inside a plugin that only
// receives input and output buffers, or host code on a path where an
// allocation could fail or stall at an inconvenient time.  The regular
// xs_pressure_solve needs a caller-provided workspace; this variant instead
// keeps its scratch (solver control block, reduction slots, the FP64
// iterate and the seven FP32 vectors of the CG and smoothing recurrences) in
// one statically sized array in device memory that belongs to the library.
//
// Limits and sharing:
//  * At most XS_STATIC_SOLVE_MAX_CELLS cells; larger grids are rejected with
//    XS_CAPACITY_EXCEEDED before anything is launched.
//  * The array is part of this file's device module: each GPU on which the
//    entry point is used holds it (about 9.1 MiB at the 64^3 limit) until the
//    process exits.
//  * All calls on a device share the one array and it keeps whatever the
//    last call left in it; the solver zeroes its control block at the start
//    of every call and writes every other scratch value before reading it.
//    Calls whose executions overlap on the GPU (different streams, or
//    different host threads without ordering) race on the array: order
//    them on one stream.
//  * The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress, with that device current, and remembers it; make
//    that first call before any stream capture begins.
//  * Failures inside the solve (a barrier timeout, no convergence within the
//    iteration cap) are only reported through host_stats: with host_stats
//    NULL the call does not synchronise, and its status covers the argument
//    checks and the launches alone.
#include <mutex>

#include "common.cuh"
#include "launch.cuh"
#include "pressure.cuh"

namespace xs {
namespace {

constexpr size_t round256(size_t v) { return (v + 255) / 256 * 256; }

constexpr uint64_t kStaticMaxCells = XS_STATIC_SOLVE_MAX_CELLS;
// Same carving as carve_pressure_workspace for the largest admitted grid.
constexpr size_t kStaticBytes = round256(sizeof(SolverState)) + round256(sizeof(double) * kPartialSlots * kMaxPersistentBlocks) +
                                round256(sizeof(double) * kStaticMaxCells) + 7 * round256(sizeof(float) * kStaticMaxCells);

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;

// Device address of g_static_scratch on the current device (set up once
// per device, with that device current).
XsStatus static_scratch(void** out) {
    static std::mutex mu;
    static void* addresses[kMaxDevices] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return XS_CUDA_ERROR;
    if (device < 0 || device >= kMaxDevices) return XS_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(mu);
    if (addresses[device] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return check_cuda(e);
        addresses[device] = p;
    }
    *out = addresses[device];
    return XS_OK;
}

}  // namespace
}  // namespace xs

using namespace xs;

extern "C" XsStatus xs_pressure_solve_static(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                                             const uint32_t* cell_mask, XsScalarBoundary pressure_boundary, const float* rhs,
                                             float* pressure, XsSolveStats* host_stats) {
    if (!valid_grid(grid) || !solve || !rhs || !pressure) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    if (cell_count(g) > kStaticMaxCells || pressure_workspace_bytes(g) > kStaticBytes) return XS_CAPACITY_EXCEEDED;
    void* scratch = nullptr;
    XsStatus s = static_scratch(&scratch);
    if (s != XS_OK) return s;
    s = solve_pressure(stream, g, *solve, pressure_anchor, cell_mask, pressure_boundary, rhs, nullptr, pressure, nullptr, scratch, nullptr);
    if (s != XS_OK || host_stats == nullptr) return s;
    return read_solve_stats(stream, scratch, g, host_stats);
}
