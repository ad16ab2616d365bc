// Forward smoke operators on sm_100a: sources and inflow, buoyancy, force
// integration, MAC advection with boundary constraints, scalar advection,
// divergence and projection.  Operator-level C ABI (operators.h:40-72).
#include <atomic>

#include "advect_tile.cuh"
#include "common.cuh"
#include "launch.cuh"
#include "ops.cuh"

namespace xs {

// ------------------------------------------------------------ sources
// operators.cu:286-290, plus inflow spheres that set the value.
__global__ void source_forward_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ state,
                                      const float* __restrict__ source, InflowSet inflows, uint32_t which, float* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { out[i] = 0.0f; return; }
    if (inflows.count) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        const int k = inflow_hit(inflows, x, y, z, g);
        if (k >= 0) { out[i] = which == 0 ? inflows.items[k].density : inflows.items[k].temperature; return; }
    }
    out[i] = state[i] + g.dt * source[i];
}

// Sources of density and temperature and the buoyancy force in one pass
// (operators.cu:286-290 twice, then :304-313 on the sourced fields, as
// model.cpp:342-344 composes them).
__global__ void source_buoyancy_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ rho,
                                       const float* __restrict__ temp, const float* __restrict__ rho_src,
                                       const float* __restrict__ temp_src, const float* __restrict__ ax,
                                       const float* __restrict__ ay, const float* __restrict__ az,
                                       const float* __restrict__ ambient, const float* __restrict__ beta_rho,
                                       const float* __restrict__ beta_temp, InflowSet inflows, float* __restrict__ rho_out,
                                       float* __restrict__ temp_out, float* __restrict__ fx, float* __restrict__ fy,
                                       float* __restrict__ fz) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) {
        rho_out[i] = 0.0f; temp_out[i] = 0.0f; fx[i] = 0.0f; fy[i] = 0.0f; fz[i] = 0.0f;
        return;
    }
    float r, t;
    int k = -1;
    if (inflows.count) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        k = inflow_hit(inflows, x, y, z, g);
    }
    if (k >= 0) {
        r = inflows.items[k].density;
        t = inflows.items[k].temperature;
    } else {
        r = rho[i] + g.dt * rho_src[i];
        t = temp[i] + g.dt * temp_src[i];
    }
    rho_out[i] = r;
    temp_out[i] = t;
    fx[i] = ax[i];
    fy[i] = ay[i] + __ldg(beta_rho) * r + __ldg(beta_temp) * (t - __ldg(ambient));
    fz[i] = az[i];
}

// ------------------------------------------------------------ buoyancy
// operators.cu:304-313
__global__ void buoyancy_forward_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ rho,
                                        const float* __restrict__ temp, const float* __restrict__ ax, const float* __restrict__ ay,
                                        const float* __restrict__ az, const float* __restrict__ ambient,
                                        const float* __restrict__ beta_rho, const float* __restrict__ beta_temp,
                                        float* __restrict__ fx, float* __restrict__ fy, float* __restrict__ fz) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { fx[i] = 0.0f; fy[i] = 0.0f; fz[i] = 0.0f; return; }
    fx[i] = ax[i];
    fy[i] = ay[i] + __ldg(beta_rho) * rho[i] + __ldg(beta_temp) * (temp[i] - __ldg(ambient));
    fz[i] = az[i];
}

// ------------------------------------------------------------ integrate
// Face index space of all three components, concatenated.
struct FaceSpace {
    uint64_t f0, f1, f2;
    __host__ __device__ uint64_t total() const { return f0 + f1 + f2; }
    __device__ __forceinline__ int locate(uint64_t i, uint64_t& local) const {
        if (i < f0) { local = i; return 0; }
        if (i < f0 + f1) { local = i - f0; return 1; }
        local = i - f0 - f1;
        return 2;
    }
};

inline FaceSpace face_space(const Grid& g) { return FaceSpace{face_count(g, 0), face_count(g, 1), face_count(g, 2)}; }

// operators.cu:339-356: mean force of the fluid cells either side of a face.
__device__ __forceinline__ float averaged_center_force(const float* __restrict__ f, int axis, int x, int y, int z, const Grid& g,
                                                       const uint32_t* __restrict__ mask) {
    const int fx = x - (axis == 0), fy = y - (axis == 1), fz = z - (axis == 2);
    float sum = 0.0f, count = 0.0f;
    if (in_grid(g, fx, fy, fz)) {
        const uint64_t c = idx3(fx, fy, fz, g.nx, g.ny);
        if (!is_solid(mask, c)) { sum += __ldg(f + c); count += 1.0f; }
    }
    if (in_grid(g, x, y, z)) {
        const uint64_t c = idx3(x, y, z, g.nx, g.ny);
        if (!is_solid(mask, c)) { sum += __ldg(f + c); count += 1.0f; }
    }
    return count == 0.0f ? 0.0f : sum / count;
}

// operators.cu:358-364 for all three components in one launch.
__global__ void integrate_kernel(Grid g, FaceSpace fs, const uint32_t* __restrict__ mask, XsVector u, XsVector f, XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= fs.total()) return;
    uint64_t local;
    const int a = fs.locate(i, local);
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    const float* ua = component(u.x, u.y, u.z, a);
    const float* fa = component(f.x, f.y, f.z, a);
    float* oa = component(out.x, out.y, out.z, a);
    oa[local] = ua[local] + g.dt * averaged_center_force(fa, a, x, y, z, g, mask);
}

// ------------------------------------------------------------ advection
// operators.cu:441-449
__device__ __forceinline__ bool adjacent_solid(int a, int x, int y, int z, const Grid& g, const uint32_t* __restrict__ mask) {
    if (mask == nullptr) return false;
    const int fx = x - (a == 0), fy = y - (a == 1), fz = z - (a == 2);
    if (in_grid(g, fx, fy, fz) && __ldg(mask + idx3(fx, fy, fz, g.nx, g.ny)) != 0u) return true;
    if (in_grid(g, x, y, z) && __ldg(mask + idx3(x, y, z, g.nx, g.ny)) != 0u) return true;
    return false;
}

// operators.cu:451-464
__device__ __forceinline__ bool constrained_boundary(int a, int x, int y, int z, const Grid& g, const XsVelocityBoundary& b,
                                                     float& value) {
    const int coord = a == 0 ? x : (a == 1 ? y : z);
    const int mx = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
    if (coord != 0 && coord != mx) return false;
    const int face = a * 2 + (coord == mx);
    const uint32_t mode = b.modes[face];
    if (mode != 0u && mode != 2u) return false;
    value = b.values[face * 3 + a];
    return true;
}

// operators.cu:381-388: one face, RK2 trace through u, sample own component.
__device__ __forceinline__ float advect_face(int a, int x, int y, int z, const Grid& g, const uint32_t* __restrict__ mask,
                                             const XsVector& u, const XsVelocityBoundary& b) {
    const Trace t = trace_rk2(face_position(a, x, y, z, g), u.x, u.y, u.z, mask, g, b);
    return sample_face<false>(component<const float>(u.x, u.y, u.z, a), a, t.position, g, b).value;
}

__global__ void advect_velocity_kernel(const __grid_constant__ Grid g, FaceSpace fs, const uint32_t* __restrict__ mask, XsVector u, const __grid_constant__ XsVelocityBoundary b,
                                       XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= fs.total()) return;
    uint64_t local;
    const int a = fs.locate(i, local);
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    component(out.x, out.y, out.z, a)[local] = advect_face(a, x, y, z, g, mask, u, b);
}

// operators.cu:466-481 (collider components may be null: zero).
__global__ void constrain_kernel(Grid g, FaceSpace fs, const uint32_t* __restrict__ mask, XsVector col, XsVector u,
                                 XsVelocityBoundary b, XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= fs.total()) return;
    uint64_t local;
    const int a = fs.locate(i, local);
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    float* oa = component(out.x, out.y, out.z, a);
    float v;
    if (constrained_boundary(a, x, y, z, g, b, v)) { oa[local] = v; return; }
    if (adjacent_solid(a, x, y, z, g, mask)) {
        const float* ca = component(col.x, col.y, col.z, a);
        oa[local] = ca == nullptr ? 0.0f : ca[local];
        return;
    }
    const float* ua = component(u.x, u.y, u.z, a);
    if (periodic(b, a) && (a == 0 ? x == g.nx : (a == 1 ? y == g.ny : z == g.nz))) {
        if (a == 0) x = 0;
        if (a == 1) y = 0;
        if (a == 2) z = 0;
        oa[local] = ua[idx3(x, y, z, extent(g, a, 0), extent(g, a, 1))];
        return;
    }
    oa[local] = ua[local];
}

// Advection and constraint fused for one face (operators.cu:381-388 then
// :466-481): the constrained value is produced directly; a periodic face at
// the upper end takes the advected value of its wrapped partner at
// coordinate 0.
__device__ __forceinline__ float advect_constrain_face(int a, int x, int y, int z, uint64_t local, const Grid& g,
                                                       const uint32_t* __restrict__ mask, const XsVector& col, const XsVector& u,
                                                       const XsVelocityBoundary& b) {
    float v;
    if (constrained_boundary(a, x, y, z, g, b, v)) return v;
    if (adjacent_solid(a, x, y, z, g, mask)) {
        const float* ca = component(col.x, col.y, col.z, a);
        return ca == nullptr ? 0.0f : ca[local];
    }
    if (periodic(b, a) && (a == 0 ? x == g.nx : (a == 1 ? y == g.ny : z == g.nz))) {
        if (a == 0) x = 0;
        if (a == 1) y = 0;
        if (a == 2) z = 0;
    }
    return advect_face(a, x, y, z, g, mask, u, b);
}

// General form (colliders, any spacing), one thread per face.  Latency-bound
// on its ~56 L1 gathers per face: the launch bounds trade a few registers for
// a fourth resident block per SM.
__global__ void __launch_bounds__(kBlock, 4) advect_constrain_kernel(const __grid_constant__ Grid g, FaceSpace fs, const uint32_t* __restrict__ mask, XsVector col, XsVector u,
                                        const __grid_constant__ XsVelocityBoundary b, XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= fs.total()) return;
    uint64_t local;
    const int a = fs.locate(i, local);
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    component(out.x, out.y, out.z, a)[local] = advect_constrain_face(a, x, y, z, local, g, mask, col, u, b);
}

// ------------------------------------------------ tile-staged advection
// Grids without colliders and with a power-of-two spacing (advect_tile.cuh).
// A CTA stages u over its box once and advects the three faces at each of
// its kTX x kTY x kTZ positions (x, y, z < nx, ny, nz): every face whose
// coordinate along its own axis is below the grid size.  The faces at the
// upper end of their axis (x = nx for u, ...) are left to the remainder
// kernel below.  Bit-identical to advect_constrain_kernel.
// Halo 1: every stencil of traces shorter than half a cell per step (the
// plume benchmark's CFL number stays near 0.06); longer traces read the
// stencils outside the box from global memory, same values.  Against halo 2
// (traces up to 1.5 cells): 41 % fewer staged nodes, 3-4 % more steps/s at
// 256^3.
using ForwardTile = tile::Shape<32, 8, 4, 1>;

template <class S, int A, bool kConstrain>
__device__ __forceinline__ void advect_constrain_tile_face(int x, int y, int z, int li, const tile::StagedVelocity& sv, const tile::Origin& o,
                                                           const tile::TileConsts& k, const Grid& g, const XsVelocityBoundary& b,
                                                           float* __restrict__ out) {
    float v;
    if (!kConstrain || !constrained_boundary(A, x, y, z, g, b, v)) {
        const Vec3 s = face_position(A, x, y, z, g);
        const Vec3 p = tile::staged_trace<S>(sv, s, tile::face_start_velocity<S, A>(sv, li), o, k, g, b);
        v = tile::staged_face<S, A, false>(sv.s[A], component<const float>(sv.u.x, sv.u.y, sv.u.z, A), p, o, k, g, b).value;
    }
    const uint32_t ex = static_cast<uint32_t>(extent(g, A, 0)), ey = static_cast<uint32_t>(extent(g, A, 1));
    out[static_cast<uint32_t>(x) + ex * (static_cast<uint32_t>(y) + ey * static_cast<uint32_t>(z))] = v;
}

// kConstrain = false: the raw advected field of advect_velocity_kernel.
template <class S, bool kConstrain>
__global__ void __launch_bounds__(S::kThreads, 4) advect_constrain_tile_kernel(const __grid_constant__ Grid g, XsVector u, const __grid_constant__ XsVelocityBoundary b, XsVector out) {
    __shared__ float box[3][S::kNodes];
    const tile::Origin o = tile::tile_origin<S>();
    tile::stage_face<S, 0>(box[0], u.x, o, g, b);
    tile::stage_face<S, 1>(box[1], u.y, o, g, b);
    tile::stage_face<S, 2>(box[2], u.z, o, g, b);
    tile::stage_wait();
    __syncthreads();
    const tile::StagedVelocity sv{{box[0], box[1], box[2]}, u};
    const tile::TileConsts k = tile::tile_consts(g, b);
    const int x = static_cast<int>(blockIdx.x) * S::TX + static_cast<int>(threadIdx.x);
    const int y = static_cast<int>(blockIdx.y) * S::TY + static_cast<int>(threadIdx.y);
    if (x >= g.nx || y >= g.ny) return;
#pragma unroll 1
    for (int kz = 0; kz < S::TZ; ++kz) {
        const int z = static_cast<int>(blockIdx.z) * S::TZ + kz;
        if (z >= g.nz) break;
        const int li = tile::local_index<S>(kz);
        advect_constrain_tile_face<S, 0, kConstrain>(x, y, z, li, sv, o, k, g, b, out.x);
        advect_constrain_tile_face<S, 1, kConstrain>(x, y, z, li, sv, o, k, g, b, out.y);
        advect_constrain_tile_face<S, 2, kConstrain>(x, y, z, li, sv, o, k, g, b, out.z);
    }
}

// The faces at the upper end of their own axis (ny nz + nx nz + nx ny of
// them), general form.
template <bool kConstrain>
__global__ void advect_constrain_upper_kernel(const __grid_constant__ Grid g, const uint32_t* __restrict__ mask, XsVector col, XsVector u, const __grid_constant__ XsVelocityBoundary b,
                                              XsVector out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t sx = static_cast<uint32_t>(g.ny) * g.nz, sy = static_cast<uint32_t>(g.nx) * g.nz, sz = static_cast<uint32_t>(g.nx) * g.ny;
    int a, x, y, z;
    if (i < sx) {
        a = 0; x = g.nx; y = static_cast<int>(i % g.ny); z = static_cast<int>(i / g.ny);
    } else if (i < sx + sy) {
        const uint32_t j = i - sx;
        a = 1; x = static_cast<int>(j % g.nx); y = g.ny; z = static_cast<int>(j / g.nx);
    } else if (i < sx + sy + sz) {
        const uint32_t j = i - sx - sy;
        a = 2; x = static_cast<int>(j % g.nx); y = static_cast<int>(j / g.nx); z = g.nz;
    } else {
        return;
    }
    const uint64_t local = idx3(x, y, z, extent(g, a, 0), extent(g, a, 1));
    component(out.x, out.y, out.z, a)[local] =
        kConstrain ? advect_constrain_face(a, x, y, z, local, g, mask, col, u, b) : advect_face(a, x, y, z, g, mask, u, b);
}

// Both tile launches of the MAC advection (with or without the constraint).
template <bool kConstrain>
XsStatus launch_advect_tiled(cudaStream_t st, const Grid& g, const XsVector& col, const XsVector& u, const XsVelocityBoundary& b,
                             const XsVector& out) {
    advect_constrain_tile_kernel<ForwardTile, kConstrain><<<tile::tile_grid<ForwardTile>(g), tile::tile_block<ForwardTile>(), 0, st>>>(g, u, b, out);
    XsStatus s = check_launch();
    if (s != XS_OK) return s;
    const uint64_t upper = static_cast<uint64_t>(g.ny) * g.nz + static_cast<uint64_t>(g.nx) * g.nz + static_cast<uint64_t>(g.nx) * g.ny;
    advect_constrain_upper_kernel<kConstrain><<<blocks_for(upper), kBlock, 0, st>>>(g, nullptr, col, u, b, out);
    return check_launch();
}

// operators.cu:499-507
__global__ void advect_scalar_kernel(const __grid_constant__ Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ collider,
                                     const float* __restrict__ src, XsVector u, const __grid_constant__ XsScalarBoundary sb, const __grid_constant__ XsVelocityBoundary vb,
                                     float* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { out[i] = collider == nullptr ? 0.0f : collider[i]; return; }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const Trace t = trace_rk2(cell_position(x, y, z, g), u.x, u.y, u.z, mask, g, vb);
    out[i] = sample_scalar<false>(src, t.position, g, sb).value;
}

// Density and temperature advected along one shared trace (the reference
// traces twice, model.cpp:347-348).
__global__ void __launch_bounds__(kBlock, 4) advect_scalar_pair_kernel(const __grid_constant__ Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ col_rho,
                                          const float* __restrict__ col_temp, const float* __restrict__ src_rho,
                                          const float* __restrict__ src_temp, XsVector u, const __grid_constant__ XsScalarBoundary rb,
                                          const __grid_constant__ XsScalarBoundary tb, const __grid_constant__ XsVelocityBoundary vb, float* __restrict__ out_rho,
                                          float* __restrict__ out_temp) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) {
        out_rho[i] = col_rho == nullptr ? 0.0f : col_rho[i];
        out_temp[i] = col_temp == nullptr ? 0.0f : col_temp[i];
        return;
    }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const Trace t = trace_rk2(cell_position(x, y, z, g), u.x, u.y, u.z, mask, g, vb);
    out_rho[i] = sample_scalar<false>(src_rho, t.position, g, rb).value;
    out_temp[i] = sample_scalar<false>(src_temp, t.position, g, tb).value;
}

// Tile-staged form of advect_scalar_pair_kernel for grids without colliders
// and with a power-of-two spacing: u, the sourced density and the sourced
// temperature are staged over the box (5 boxes, dynamic shared memory).
// Bit-identical to advect_scalar_pair_kernel; kFields = 1 advects one field
// (advect_scalar_kernel).
template <class S>
constexpr size_t scalar_tile_smem(int fields) { return (3 + fields) * sizeof(float) * S::kNodes; }

template <class S, int kFields>
__global__ void __launch_bounds__(S::kThreads, 3) advect_scalar_pair_tile_kernel(const __grid_constant__ Grid g, const float* __restrict__ src_rho,
                                                                                      const float* __restrict__ src_temp, XsVector u,
                                                                                      const __grid_constant__ XsScalarBoundary rb, const __grid_constant__ XsScalarBoundary tb,
                                                                                      const __grid_constant__ XsVelocityBoundary vb, float* __restrict__ out_rho,
                                                                                      float* __restrict__ out_temp) {
    extern __shared__ float smem[];
    float* box[5] = {smem, smem + S::kNodes, smem + 2 * S::kNodes, smem + 3 * S::kNodes, smem + 4 * S::kNodes};
    const tile::Origin o = tile::tile_origin<S>();
    tile::stage_face<S, 0>(box[0], u.x, o, g, vb);
    tile::stage_face<S, 1>(box[1], u.y, o, g, vb);
    tile::stage_face<S, 2>(box[2], u.z, o, g, vb);
    tile::stage_cells<S>(box[3], src_rho, o, g, rb);
    if (kFields == 2) tile::stage_cells<S>(box[4], src_temp, o, g, tb);
    tile::stage_wait();
    __syncthreads();
    const tile::StagedVelocity sv{{box[0], box[1], box[2]}, u};
    const tile::TileConsts k = tile::tile_consts(g, vb);
    const int x = static_cast<int>(blockIdx.x) * S::TX + static_cast<int>(threadIdx.x);
    const int y = static_cast<int>(blockIdx.y) * S::TY + static_cast<int>(threadIdx.y);
    if (x >= g.nx || y >= g.ny) return;
#pragma unroll 1
    for (int kz = 0; kz < S::TZ; ++kz) {
        const int z = static_cast<int>(blockIdx.z) * S::TZ + kz;
        if (z >= g.nz) break;
        const int li = tile::local_index<S>(kz);
        const Vec3 s = cell_position(x, y, z, g);
        const Vec3 p = tile::staged_trace<S>(sv, s, tile::cell_start_velocity<S>(sv, li), o, k, g, vb);
        const uint32_t i = static_cast<uint32_t>(x) + static_cast<uint32_t>(g.nx) * (static_cast<uint32_t>(y) + static_cast<uint32_t>(g.ny) *
                                                                                                                static_cast<uint32_t>(z));
        out_rho[i] = tile::staged_scalar<S, false>(box[3], src_rho, p, o, k, g, rb).value;
        if (kFields == 2) out_temp[i] = tile::staged_scalar<S, false>(box[4], src_temp, p, o, k, g, tb).value;
    }
}

// ------------------------------------------------------------ projection
// operators.cu:904-910
__device__ __forceinline__ bool projectable_face(const Grid& g, int a, int x, int y, int z, const uint32_t* __restrict__ mask,
                                                 uint64_t& first, uint64_t& second) {
    const int fx = x - (a == 0), fy = y - (a == 1), fz = z - (a == 2);
    if (!in_grid(g, fx, fy, fz) || !in_grid(g, x, y, z)) return false;
    first = idx3(fx, fy, fz, g.nx, g.ny);
    second = idx3(x, y, z, g.nx, g.ny);
    return !is_solid(mask, first) && !is_solid(mask, second);
}

// operators.cu:912-920 with an FP32 pressure.
__global__ void project_kernel(Grid g, FaceSpace fs, const uint32_t* __restrict__ mask, XsVector u, const float* __restrict__ p,
                               XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= fs.total()) return;
    uint64_t local;
    const int a = fs.locate(i, local);
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    const float* ua = component(u.x, u.y, u.z, a);
    float* oa = component(out.x, out.y, out.z, a);
    uint64_t f, s;
    if (!projectable_face(g, a, x, y, z, mask, f, s)) { oa[local] = ua[local]; return; }
    oa[local] = ua[local] - g.dt * (__ldg(p + s) - __ldg(p + f)) / g.h;
}

// The same with the FP64 pressure iterate of the PCG solve: the pressure
// difference is taken in FP64 and the velocity rounded once.
__global__ void project64_kernel(Grid g, FaceSpace fs, const uint32_t* __restrict__ mask, XsVector u, const double* __restrict__ p,
                                 XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= fs.total()) return;
    uint64_t local;
    const int a = fs.locate(i, local);
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    const float* ua = component(u.x, u.y, u.z, a);
    float* oa = component(out.x, out.y, out.z, a);
    uint64_t f, s;
    if (!projectable_face(g, a, x, y, z, mask, f, s)) { oa[local] = ua[local]; return; }
    const double dp = __ldg(p + s) - __ldg(p + f);
    oa[local] = static_cast<float>(static_cast<double>(ua[local]) - static_cast<double>(g.dt) * dp / static_cast<double>(g.h));
}

// operators.cu:875-883
__global__ void pressure_rhs_kernel(Grid g, uint32_t anchor, const uint32_t* __restrict__ mask, XsVector u, float* __restrict__ rhs) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i) || i == anchor) { rhs[i] = 0.0f; return; }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const float div = (__ldg(u.x + idx3(x + 1, y, z, g.nx + 1, g.ny)) - __ldg(u.x + idx3(x, y, z, g.nx + 1, g.ny)) +
                       __ldg(u.y + idx3(x, y + 1, z, g.nx, g.ny + 1)) - __ldg(u.y + idx3(x, y, z, g.nx, g.ny + 1)) +
                       __ldg(u.z + idx3(x, y, z + 1, g.nx, g.ny)) - __ldg(u.z + idx3(x, y, z, g.nx, g.ny))) / g.h;
    rhs[i] = -g.h * g.h * div / g.dt;
}

// pressure_rhs_kernel without colliders, 3D-indexed: a thread takes kFaceZ
// cells of one (x, y) column, loading all their face velocities before the
// first store; the same arithmetic per cell.
template <int kZ>
__global__ void __launch_bounds__(256) pressure_rhs_cells_kernel(const __grid_constant__ Grid g, uint32_t anchor, XsVector u, float* __restrict__ rhs) {
    const int x = static_cast<int>(blockIdx.x * 32 + threadIdx.x), y = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    const int z0 = static_cast<int>(blockIdx.z) * kZ;
    if (x >= g.nx || y >= g.ny) return;
    float d[kZ][6];
#pragma unroll
    for (int k = 0; k < kZ; ++k) {
        const int z = z0 + k;
        if (z >= g.nz) continue;
        d[k][0] = __ldg(u.x + tile::index32(x + 1, y, z, g.nx + 1, g.ny));
        d[k][1] = __ldg(u.x + tile::index32(x, y, z, g.nx + 1, g.ny));
        d[k][2] = __ldg(u.y + tile::index32(x, y + 1, z, g.nx, g.ny + 1));
        d[k][3] = __ldg(u.y + tile::index32(x, y, z, g.nx, g.ny + 1));
        d[k][4] = __ldg(u.z + tile::index32(x, y, z + 1, g.nx, g.ny));
        d[k][5] = __ldg(u.z + tile::index32(x, y, z, g.nx, g.ny));
    }
#pragma unroll
    for (int k = 0; k < kZ; ++k) {
        const int z = z0 + k;
        if (z >= g.nz) continue;
        const uint32_t i = tile::index32(x, y, z, g.nx, g.ny);
        const float div = (d[k][0] - d[k][1] + d[k][2] - d[k][3] + d[k][4] - d[k][5]) / g.h;
        rhs[i] = i == anchor ? 0.0f : -g.h * g.h * div / g.dt;
    }
}

__global__ void accumulate_kernel(const double* __restrict__ src, double* __restrict__ dst, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] += src[i];
}

// ------------------------------------------------ collider-free face passes
// Faces of all three components addressed in 3D: blockIdx.z runs over the
// z-slices of u, then v, then w (each component's own z extent); threads
// cover (x, y) with x fastest, so loads and stores are coalesced and no index
// is decoded.  The arithmetic is the general kernels' (bit-identical).
// Each thread handles kFaceZ consecutive z-slices of its component: all of
// their loads are issued before the first store (four times the bytes in
// flight of one face per thread).
constexpr int kFaceZ = 4;

struct FaceSlice {
    int a, z;  // component and first z-slice of the block
};

__host__ __device__ __forceinline__ int face_blocks_z(int extent_z) { return (extent_z + kFaceZ - 1) / kFaceZ; }

__device__ __forceinline__ FaceSlice face_slice(const Grid& g) {
    const int zi = static_cast<int>(blockIdx.z);
    const int z0 = face_blocks_z(g.nz), z1 = 2 * z0;  // u and v have nz slices, w has nz + 1
    if (zi < z0) return FaceSlice{0, kFaceZ * zi};
    if (zi < z1) return FaceSlice{1, kFaceZ * (zi - z0)};
    return FaceSlice{2, kFaceZ * (zi - z1)};
}

inline dim3 face_pass_grid(const Grid& g) {
    return dim3(static_cast<unsigned>((g.nx + 1 + 31) / 32), static_cast<unsigned>((g.ny + 1 + 7) / 8),
                static_cast<unsigned>(2 * face_blocks_z(g.nz) + face_blocks_z(g.nz + 1)));
}

// operators.cu:358-364 without colliders, for kFaceZ z-slices of face
// component A: the mean of
// the one or two in-grid cell forces beside the face (division by a count
// of 2 is the exact product with 0.5).
template <int A>
__device__ __forceinline__ void integrate_faces(const Grid& g, int x, int y, int z0, const XsVector& u, const XsVector& f, const XsVector& out) {
    const int ex = extent(g, A, 0), ey = extent(g, A, 1), ez = extent(g, A, 2);
    if (x >= ex || y >= ey) return;
    const float* fa = component<const float>(f.x, f.y, f.z, A);
    const float* ua = component<const float>(u.x, u.y, u.z, A);
    const int n = A == 0 ? g.nx : (A == 1 ? g.ny : g.nz);
    const uint32_t step = static_cast<uint32_t>(A == 0 ? 1 : (A == 1 ? g.nx : g.nx * g.ny));
    float uv[kFaceZ], lo[kFaceZ], hi[kFaceZ];
#pragma unroll
    for (int k = 0; k < kFaceZ; ++k) {
        const int z = z0 + k;
        uv[k] = lo[k] = hi[k] = 0.0f;
        if (z >= ez) continue;
        const int c = A == 0 ? x : (A == 1 ? y : z);
        const uint32_t upper = tile::index32(x, y, z, g.nx, g.ny);
        uv[k] = __ldg(ua + tile::index32(x, y, z, ex, ey));
        if (c != n) hi[k] = __ldg(fa + upper);
        if (c != 0) lo[k] = __ldg(fa + upper - step);
    }
    float* oa = component(out.x, out.y, out.z, A);
#pragma unroll
    for (int k = 0; k < kFaceZ; ++k) {
        const int z = z0 + k;
        if (z >= ez) continue;
        const int c = A == 0 ? x : (A == 1 ? y : z);
        float sum = 0.0f, mean;
        if (c == 0) {
            sum += hi[k];
            mean = sum;
        } else if (c == n) {
            sum += lo[k];
            mean = sum;
        } else {
            sum += lo[k];
            sum += hi[k];
            mean = sum * 0.5f;
        }
        oa[tile::index32(x, y, z, ex, ey)] = uv[k] + g.dt * mean;
    }
}

__global__ void __launch_bounds__(256) integrate_faces_kernel(const __grid_constant__ Grid g, XsVector u, XsVector f, XsVector out) {
    const FaceSlice fsl = face_slice(g);
    const int x = static_cast<int>(blockIdx.x * 32 + threadIdx.x), y = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (fsl.a == 0) integrate_faces<0>(g, x, y, fsl.z, u, f, out);
    else if (fsl.a == 1) integrate_faces<1>(g, x, y, fsl.z, u, f, out);
    else integrate_faces<2>(g, x, y, fsl.z, u, f, out);
}

// operators.cu:912-920 with the FP64 pressure iterate, without colliders, for
// kFaceZ z-slices of face component A.  For a power-of-two spacing the FP64 division by h is the
// exact product with inv_h = 1/h (computed on the host; the same IEEE result).
template <int A, bool kPow2>
__device__ __forceinline__ void project64_faces(const Grid& g, double inv_h, int x, int y, int z0, const XsVector& u, const double* __restrict__ p,
                                                const XsVector& out) {
    const int ex = extent(g, A, 0), ey = extent(g, A, 1), ez = extent(g, A, 2);
    if (x >= ex || y >= ey) return;
    const float* ua = component<const float>(u.x, u.y, u.z, A);
    const int n = A == 0 ? g.nx : (A == 1 ? g.ny : g.nz);
    const uint32_t step = static_cast<uint32_t>(A == 0 ? 1 : (A == 1 ? g.nx : g.nx * g.ny));
    float uv[kFaceZ];
    double p0[kFaceZ], p1[kFaceZ];
#pragma unroll
    for (int k = 0; k < kFaceZ; ++k) {
        const int z = z0 + k;
        uv[k] = 0.0f;
        p0[k] = p1[k] = 0.0;
        if (z >= ez) continue;
        const int c = A == 0 ? x : (A == 1 ? y : z);
        uv[k] = __ldg(ua + tile::index32(x, y, z, ex, ey));
        if (c == 0 || c == n) continue;  // projectable_face: both cells in the grid
        const uint32_t second = tile::index32(x, y, z, g.nx, g.ny);
        p1[k] = __ldg(p + second);
        p0[k] = __ldg(p + second - step);
    }
    float* oa = component(out.x, out.y, out.z, A);
#pragma unroll
    for (int k = 0; k < kFaceZ; ++k) {
        const int z = z0 + k;
        if (z >= ez) continue;
        const int c = A == 0 ? x : (A == 1 ? y : z);
        const uint32_t i = tile::index32(x, y, z, ex, ey);
        if (c == 0 || c == n) {
            oa[i] = uv[k];
            continue;
        }
        const double dp = p1[k] - p0[k];
        const double scaled = static_cast<double>(g.dt) * dp;
        oa[i] = static_cast<float>(static_cast<double>(uv[k]) - (kPow2 ? scaled * inv_h : scaled / static_cast<double>(g.h)));
    }
}

template <bool kPow2>
__global__ void __launch_bounds__(256) project64_faces_kernel(const __grid_constant__ Grid g, double inv_h, XsVector u, const double* __restrict__ p,
                                                              XsVector out) {
    const FaceSlice fsl = face_slice(g);
    const int x = static_cast<int>(blockIdx.x * 32 + threadIdx.x), y = static_cast<int>(blockIdx.y * 8 + threadIdx.y);
    if (fsl.a == 0) project64_faces<0, kPow2>(g, inv_h, x, y, fsl.z, u, p, out);
    else if (fsl.a == 1) project64_faces<1, kPow2>(g, inv_h, x, y, fsl.z, u, p, out);
    else project64_faces<2, kPow2>(g, inv_h, x, y, fsl.z, u, p, out);
}

// ------------------------------------------------------------ launchers
template <class S, int kFields>
XsStatus launch_scalar_tiled_shape(cudaStream_t st, const Grid& g, const float* src_rho, const float* src_temp, const XsVector& u,
                                   const XsScalarBoundary& rb, const XsScalarBoundary& tb, const XsVelocityBoundary& vb, float* out_rho,
                                   float* out_temp) {
    static DeviceOnce configured;
    if (!configured.run([] {
            return cudaFuncSetAttribute(advect_scalar_pair_tile_kernel<S, kFields>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(scalar_tile_smem<S>(kFields)));
        }))
        return XS_CUDA_ERROR;
    advect_scalar_pair_tile_kernel<S, kFields><<<tile::tile_grid<S>(g), tile::tile_block<S>(), scalar_tile_smem<S>(kFields), st>>>(
        g, src_rho, src_temp, u, rb, tb, vb, out_rho, out_temp);
    return check_launch();
}

template <int kFields>
XsStatus launch_scalar_tiled(cudaStream_t st, const Grid& g, const float* src_rho, const float* src_temp, const XsVector& u,
                             const XsScalarBoundary& rb, const XsScalarBoundary& tb, const XsVelocityBoundary& vb, float* out_rho,
                             float* out_temp) {
    return launch_scalar_tiled_shape<ForwardTile, kFields>(st, g, src_rho, src_temp, u, rb, tb, vb, out_rho, out_temp);
}

InflowSet make_inflows(const XsInflow* inflows, uint32_t count) {
    InflowSet s{};
    s.count = inflows == nullptr ? 0u : count;
    for (uint32_t k = 0; k < s.count; ++k) s.items[k] = inflows[k];
    return s;
}

XsStatus launch_source_buoyancy(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho, const float* temp,
                                const float* rho_src, const float* temp_src, const XsVector& acc, const float* ambient,
                                const float* beta_rho, const float* beta_temp, const InflowSet& inflows, float* rho_out,
                                float* temp_out, const XsVector& force) {
    source_buoyancy_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, rho, temp, rho_src, temp_src, acc.x, acc.y, acc.z,
                                                                          ambient, beta_rho, beta_temp, inflows, rho_out, temp_out,
                                                                          force.x, force.y, force.z);
    return check_launch();
}

XsStatus launch_integrate(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVector& f, const XsVector& out) {
    if (mask == nullptr) {
        integrate_faces_kernel<<<face_pass_grid(g), dim3(32, 8), 0, st>>>(g, u, f, out);
        return check_launch();
    }
    const FaceSpace fs = face_space(g);
    integrate_kernel<<<blocks_for(fs.total()), kBlock, 0, st>>>(g, fs, mask, u, f, out);
    return check_launch();
}

XsStatus launch_advect_constrain(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& col, const XsVector& u,
                                 const XsVelocityBoundary& b, const XsVector& out) {
    if (tile::tiled_advection(g, mask)) return launch_advect_tiled<true>(st, g, col, u, b, out);
    const FaceSpace fs = face_space(g);
    advect_constrain_kernel<<<blocks_for(fs.total()), kBlock, 0, st>>>(g, fs, mask, col, u, b, out);
    return check_launch();
}

XsStatus launch_constrain(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& col, const XsVector& u,
                          const XsVelocityBoundary& b, const XsVector& out) {
    const FaceSpace fs = face_space(g);
    constrain_kernel<<<blocks_for(fs.total()), kBlock, 0, st>>>(g, fs, mask, col, u, b, out);
    return check_launch();
}

XsStatus launch_advect_scalar_pair(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* col_rho, const float* col_temp,
                                   const float* src_rho, const float* src_temp, const XsVector& u, const XsScalarBoundary& rb,
                                   const XsScalarBoundary& tb, const XsVelocityBoundary& vb, float* out_rho, float* out_temp) {
    if (tile::tiled_advection(g, mask)) return launch_scalar_tiled<2>(st, g, src_rho, src_temp, u, rb, tb, vb, out_rho, out_temp);
    advect_scalar_pair_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, col_rho, col_temp, src_rho, src_temp, u, rb, tb,
                                                                             vb, out_rho, out_temp);
    return check_launch();
}

XsStatus launch_pressure_rhs(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsVector& u, float* rhs) {
    if (mask == nullptr && g.nz <= 4 * 65535) {
        const dim3 grid(static_cast<unsigned>((g.nx + 31) / 32), static_cast<unsigned>((g.ny + 7) / 8), static_cast<unsigned>((g.nz + kFaceZ - 1) / kFaceZ));
        pressure_rhs_cells_kernel<kFaceZ><<<grid, dim3(32, 8), 0, st>>>(g, anchor, u, rhs);
        return check_launch();
    }
    pressure_rhs_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, anchor, mask, u, rhs);
    return check_launch();
}

XsStatus launch_project(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const float* p, const XsVector& out) {
    const FaceSpace fs = face_space(g);
    project_kernel<<<blocks_for(fs.total()), kBlock, 0, st>>>(g, fs, mask, u, p, out);
    return check_launch();
}

XsStatus launch_project64(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const double* p, const XsVector& out) {
    if (mask == nullptr) {
        const double inv_h = 1.0 / static_cast<double>(g.h);
        if (tile::tiled_advection(g, mask))
            project64_faces_kernel<true><<<face_pass_grid(g), dim3(32, 8), 0, st>>>(g, inv_h, u, p, out);
        else
            project64_faces_kernel<false><<<face_pass_grid(g), dim3(32, 8), 0, st>>>(g, inv_h, u, p, out);
        return check_launch();
    }
    const FaceSpace fs = face_space(g);
    project64_kernel<<<blocks_for(fs.total()), kBlock, 0, st>>>(g, fs, mask, u, p, out);
    return check_launch();
}

}  // namespace xs

using namespace xs;

extern "C" {

XsStatus xs_accumulate(cudaStream_t stream, const double* source, double* destination, uint64_t count) {
    if (count == 0) return XS_OK;
    if (!source || !destination) return XS_INVALID_ARGUMENT;
    accumulate_kernel<<<blocks_for(count), kBlock, 0, stream>>>(source, destination, count);
    return check_launch();
}

XsStatus xs_source_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* state, const float* source,
                           const XsInflow* inflows, uint32_t inflow_count, uint32_t which, float* output) {
    if (!valid_grid(grid) || !state || !source || !output || inflow_count > XS_MAX_INFLOWS) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    source_forward_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(g, cell_mask, state, source, make_inflows(inflows, inflow_count),
                                                                             which, output);
    return check_launch();
}

XsStatus xs_buoyancy_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* density, const float* temperature,
                             XsVector external_acceleration, const float* ambient_temperature, const float* density_buoyancy,
                             const float* temperature_buoyancy, XsVector force) {
    if (!valid_grid(grid) || !density || !temperature || !ambient_temperature || !density_buoyancy || !temperature_buoyancy ||
        !valid(external_acceleration) || !valid(force))
        return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    buoyancy_forward_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(
        g, cell_mask, density, temperature, external_acceleration.x, external_acceleration.y, external_acceleration.z, ambient_temperature,
        density_buoyancy, temperature_buoyancy, force.x, force.y, force.z);
    return check_launch();
}

XsStatus xs_integrate_velocity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, XsVector force,
                                       XsVector output) {
    if (!valid_grid(grid) || !valid(velocity) || !valid(force) || !valid(output)) return XS_INVALID_ARGUMENT;
    return launch_integrate(stream, make_grid(grid), cell_mask, velocity, force, output);
}

XsStatus xs_advect_velocity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity,
                                    XsVelocityBoundary boundary, XsVector output) {
    if (!valid_grid(grid) || !valid(velocity) || !valid(output)) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    if (tile::tiled_advection(g, cell_mask)) return launch_advect_tiled<false>(stream, g, XsVector{nullptr, nullptr, nullptr}, velocity, boundary, output);
    const FaceSpace fs = face_space(g);
    advect_velocity_kernel<<<blocks_for(fs.total()), kBlock, 0, stream>>>(g, fs, cell_mask, velocity, boundary, output);
    return check_launch();
}

XsStatus xs_constrain_velocity_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector collider_velocity,
                                       XsVector velocity, XsVelocityBoundary boundary, XsVector output) {
    if (!valid_grid(grid) || !valid(velocity) || !valid(output)) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    const FaceSpace fs = face_space(g);
    constrain_kernel<<<blocks_for(fs.total()), kBlock, 0, stream>>>(g, fs, cell_mask, collider_velocity, velocity, boundary, output);
    return check_launch();
}

XsStatus xs_advect_scalar_forward(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* collider_value,
                                  const float* source, XsVector velocity, XsScalarBoundary scalar_boundary,
                                  XsVelocityBoundary velocity_boundary, float* output) {
    if (!valid_grid(grid) || !source || !valid(velocity) || !output) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    if (tile::tiled_advection(g, cell_mask))
        return launch_scalar_tiled<1>(stream, g, source, nullptr, velocity, scalar_boundary, scalar_boundary, velocity_boundary, output, nullptr);
    advect_scalar_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(g, cell_mask, collider_value, source, velocity, scalar_boundary,
                                                                            velocity_boundary, output);
    return check_launch();
}

}  // extern "C"
