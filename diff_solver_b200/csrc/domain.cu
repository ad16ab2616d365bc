// Device-side domain construction: collider rasterisation, collider face
// velocities and the pressure anchor (solvers/smoke/model.cpp:32-183).  The
// reference loops over every cell on the host; here one thread per cell or
// face tests the (few) colliders, so large grids build in milliseconds.
#include <cstring>
#include <vector>

#include "common.cuh"
#include "launch.cuh"

namespace xs {

constexpr int kMaxColliders = 32;

struct ColliderSet {
    uint32_t count;
    XsCollider items[kMaxColliders];
};

// model.cpp:17-26 (contains) evaluated at the cell centre in FP32; the last
// collider containing the centre wins (model.cpp:61-68).  Returns -1 if none.
__device__ __forceinline__ int collider_at(const ColliderSet& cs, int x, int y, int z, float h) {
    const float px = (static_cast<float>(x) + 0.5f) * h, py = (static_cast<float>(y) + 0.5f) * h, pz = (static_cast<float>(z) + 0.5f) * h;
    int hit = -1;
    for (uint32_t k = 0; k < cs.count; ++k) {
        const XsCollider& c = cs.items[k];
        bool inside;
        if (c.shape == 0u) {
            const float a = (px - c.center[0]) / c.size[0], b = (py - c.center[1]) / c.size[1], d = (pz - c.center[2]) / c.size[2];
            inside = a * a + b * b + d * d <= 1.0f;
        } else {
            inside = fabsf(px - c.center[0]) <= c.size[0] && fabsf(py - c.center[1]) <= c.size[1] && fabsf(pz - c.center[2]) <= c.size[2];
        }
        if (inside) hit = static_cast<int>(k);
    }
    return hit;
}

__global__ void rasterize_kernel(Grid g, ColliderSet cs, uint32_t* __restrict__ mask, float* __restrict__ density,
                                 float* __restrict__ temperature) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const int k = collider_at(cs, x, y, z, g.h);
    mask[i] = k >= 0 ? 1u : 0u;
    density[i] = k >= 0 ? cs.items[k].density : 0.0f;
    temperature[i] = k >= 0 ? cs.items[k].temperature : 0.0f;
}

// model.cpp:79-150: mean collider velocity component of the solid cells on
// either side of a face, in the order (lower, upper) as the reference sums.
__global__ void collider_face_kernel(Grid g, ColliderSet cs, int axis, float* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= face_count(g, axis)) return;
    int x, y, z;
    decode(i, extent(g, axis, 0), extent(g, axis, 1), x, y, z);
    float sum = 0.0f, count = 0.0f;
    const int lx = x - (axis == 0), ly = y - (axis == 1), lz = z - (axis == 2);
    if (in_grid(g, lx, ly, lz)) {
        const int k = collider_at(cs, lx, ly, lz, g.h);
        if (k >= 0) { sum += cs.items[k].velocity[axis]; count += 1.0f; }
    }
    if (in_grid(g, x, y, z)) {
        const int k = collider_at(cs, x, y, z, g.h);
        if (k >= 0) { sum += cs.items[k].velocity[axis]; count += 1.0f; }
    }
    out[i] = count == 0.0f ? 0.0f : sum / count;
}

}  // namespace xs

using namespace xs;

extern "C" XsStatus xs_smoke_build_domain(cudaStream_t stream, XsGrid grid, XsScalarBoundary pressure_boundary, const XsCollider* colliders,
                                          uint32_t collider_count, uint32_t* cell_mask, XsVector collider_velocity,
                                          float* collider_density, float* collider_temperature, uint32_t* pressure_anchor) {
    if (!valid_grid(grid) || !cell_mask || !valid(collider_velocity) || !collider_density || !collider_temperature || !pressure_anchor ||
        collider_count > static_cast<uint32_t>(kMaxColliders) || (collider_count && !colliders))
        return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    ColliderSet cs{};
    cs.count = collider_count;
    for (uint32_t k = 0; k < collider_count; ++k) cs.items[k] = colliders[k];
    rasterize_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(g, cs, cell_mask, collider_density, collider_temperature);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    for (int a = 0; a < 3; ++a) {
        collider_face_kernel<<<blocks_for(face_count(g, a)), kBlock, 0, stream>>>(g, cs, a,
                                                                                  component(collider_velocity.x, collider_velocity.y,
                                                                                            collider_velocity.z, a));
        if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    }
    // model.cpp:72-77: no anchor ("cell_count") if any pressure face is fixed,
    // else the first fluid cell.
    bool fixed = false;
    for (int f = 0; f < 6; ++f) fixed = fixed || pressure_boundary.modes[f] == 0u;
    const uint64_t n = cell_count(g);
    if (fixed) {
        *pressure_anchor = static_cast<uint32_t>(n);
    } else if (collider_count == 0) {
        *pressure_anchor = 0u;
    } else {
        std::vector<uint32_t> host(n);
        if (cudaMemcpyAsync(host.data(), cell_mask, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return XS_CUDA_ERROR;
        if (cudaStreamSynchronize(stream) != cudaSuccess) return XS_CUDA_ERROR;
        uint64_t a = 0;
        while (a < n && host[a] != 0u) ++a;
        *pressure_anchor = static_cast<uint32_t>(a);
    }
    return check_cuda(cudaStreamSynchronize(stream));
}
