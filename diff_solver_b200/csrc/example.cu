// Kernels of the reference's forward example driver
// (examples/smoke/forward/simulation.cu): the pulsed double-jet controls the
// driver writes before every step.  The per-step metrics reduction lives with
// the step composition (step.cu, xs_smoke_reduce_metrics).
#include "common.cuh"
#include "launch.cuh"

namespace xs {

struct Jets {
    float pulse_period, radius, density_rate, temperature_rate;
    XsVec3 left_center, right_center, left_acceleration, right_acceleration;
};

__device__ __forceinline__ float jet_weight(float x, float y, float z, const XsVec3& c, float radius) {
    const float dx = x - c.x, dy = y - c.y, dz = z - c.z;
    return expf(-0.5f * (dx * dx + dy * dy + dz * dz) / (radius * radius));
}

// simulation.cu:35-57: two Gaussian jets whose strengths pulse in antiphase
// with the given period; each cell's sources are the rates times the summed
// weight, its external acceleration the weighted jet accelerations.
__global__ void write_control_kernel(Grid g, uint64_t step, Jets j, float* __restrict__ density_source, float* __restrict__ temperature_source,
                                     XsVector acceleration) {
    const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nx = static_cast<uint32_t>(g.nx), ny = static_cast<uint32_t>(g.ny);
    if (cell >= nx * ny * static_cast<uint32_t>(g.nz)) return;
    const float x = (static_cast<float>(cell % nx) + 0.5f) * g.h;
    const float y = (static_cast<float>(cell / nx % ny) + 0.5f) * g.h;
    const float z = (static_cast<float>(cell / (nx * ny)) + 0.5f) * g.h;
    constexpr float kTwoPi = 6.28318530717958647692f;
    const float phase = kTwoPi * (static_cast<float>(step) * g.dt) / j.pulse_period;
    const float left = (0.75f + 0.25f * sinf(phase)) * jet_weight(x, y, z, j.left_center, j.radius);
    const float right = (0.75f + 0.25f * sinf(phase + 0.5f * kTwoPi)) * jet_weight(x, y, z, j.right_center, j.radius);
    const float both = left + right;
    density_source[cell] = j.density_rate * both;
    temperature_source[cell] = j.temperature_rate * both;
    acceleration.x[cell] = left * j.left_acceleration.x + right * j.right_acceleration.x;
    acceleration.y[cell] = left * j.left_acceleration.y + right * j.right_acceleration.y;
    acceleration.z[cell] = left * j.left_acceleration.z + right * j.right_acceleration.z;
}

}  // namespace xs

using namespace xs;

extern "C" XsStatus xs_smoke_write_control(cudaStream_t stream, XsGrid grid, uint64_t step, float pulse_period, XsVec3 left_center,
                                           XsVec3 right_center, float source_radius, float density_source_rate,
                                           float temperature_source_rate, XsVec3 left_acceleration, XsVec3 right_acceleration,
                                           float* density_source, float* temperature_source, XsVector external_acceleration) {
    if (!valid_grid(grid) || !density_source || !temperature_source || !valid(external_acceleration) || !(pulse_period != 0.0f) ||
        !(source_radius != 0.0f))
        return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    const Jets j{pulse_period, source_radius, density_source_rate, temperature_source_rate, left_center, right_center, left_acceleration,
                 right_acceleration};
    write_control_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(g, step, j, density_source, temperature_source,
                                                                            external_acceleration);
    return check_launch();
}
