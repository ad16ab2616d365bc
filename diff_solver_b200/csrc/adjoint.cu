// Adjoint (VJP) smoke operators on sm_100a
// (solvers/smoke/operators.cu:196-240, 297-302, 326-337, 366-379, 415-439,
// 483-497, 537-561, 922-969).
//
// Operators whose transpose has a fixed, local sparsity (sources, buoyancy,
// integration, constraints, projection and the divergence) are written in
// gather form: each output element sums what the reference would have
// scattered into it, so they need no atomics and are deterministic.  The
// transposes of the trilinear gathers along backtraced paths (advection)
// scatter with FP64 atomics to the 8 corners, as their targets depend on the
// velocity field.  Parameter adjoints are reduced per block first.
#include "ops.cuh"
#include "advect_tile.cuh"
#include "common.cuh"
#include "launch.cuh"

namespace xs {

// ---------------------------------------------------------------- sources
// operators.cu:297-302; inflow cells are set, not sourced: no adjoint flows.
__global__ void source_vjp_kernel(Grid g, const uint32_t* __restrict__ mask, const double* __restrict__ oa, InflowSet inflows,
                                  double* __restrict__ sa, double* __restrict__ ra) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g) || is_solid(mask, i)) return;
    if (inflows.count) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        if (inflow_hit(inflows, x, y, z, g) >= 0) return;
    }
    sa[i] += oa[i];
    ra[i] += static_cast<double>(g.dt) * oa[i];
}

// operators.cu:326-337 with block-reduced parameter adjoints.
__global__ void buoyancy_vjp_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ rho, const float* __restrict__ temp,
                                    const float* __restrict__ ambient, const float* __restrict__ beta_rho,
                                    const float* __restrict__ beta_temp, XsAdjointVector fa, double* __restrict__ rho_a,
                                    double* __restrict__ temp_a, XsAdjointVector ea, double* __restrict__ amb_a,
                                    double* __restrict__ br_a, double* __restrict__ bt_a) {
    __shared__ double red[4 * 32];
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double part[3] = {0.0, 0.0, 0.0};
    if (i < cell_count(g) && !is_solid(mask, i)) {
        const double fy = fa.y[i];
        ea.x[i] += fa.x[i];
        ea.y[i] += fy;
        ea.z[i] += fa.z[i];
        const float bt = __ldg(beta_temp);
        rho_a[i] += static_cast<double>(__ldg(beta_rho)) * fy;
        temp_a[i] += static_cast<double>(bt) * fy;
        part[0] = -static_cast<double>(bt) * fy;
        part[1] = static_cast<double>(rho[i]) * fy;
        part[2] = static_cast<double>(temp[i] - __ldg(ambient)) * fy;
    }
    block_sum<3>(part, red);
    if (threadIdx.x == 0) {
        if (part[0] != 0.0) atomicAdd(amb_a, part[0]);
        if (part[1] != 0.0) atomicAdd(br_a, part[1]);
        if (part[2] != 0.0) atomicAdd(bt_a, part[2]);
    }
}

// ---------------------------------------------------------------- integrate
__device__ __forceinline__ int fluid_neighbours_of_face(const Grid& g, const uint32_t* mask, int a, int x, int y, int z) {
    int count = 0;
    const int lx = x - (a == 0), ly = y - (a == 1), lz = z - (a == 2);
    if (in_grid(g, lx, ly, lz) && !is_solid(mask, idx3(lx, ly, lz, g.nx, g.ny))) ++count;
    if (in_grid(g, x, y, z) && !is_solid(mask, idx3(x, y, z, g.nx, g.ny))) ++count;
    return count;
}

// operators.cu:366-379, face part: velocity adjoint += output adjoint.
__global__ void integrate_vjp_faces_kernel(uint64_t n, const double* __restrict__ oa, double* __restrict__ ua) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) ua[i] += oa[i];
}

// operators.cu:366-379, force part gathered per fluid cell: each of the cell's
// two faces along axis a hands dt * oa / (fluid cells beside that face).
// kAssign: the force adjoint is written instead of accumulated (a caller
// whose force adjoint starts at zero skips clearing it).
template <bool kAssign>
__global__ void integrate_vjp_cells_kernel(Grid g, const uint32_t* __restrict__ mask, XsAdjointVector oa, XsAdjointVector fa) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g) || is_solid(mask, i)) return;
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int ex = extent(g, a, 0), ey = extent(g, a, 1);
        const double* o = component<double>(oa.x, oa.y, oa.z, a);
        const int ux = x + (a == 0), uy = y + (a == 1), uz = z + (a == 2);
        const double lo = o[idx3(x, y, z, ex, ey)] / fluid_neighbours_of_face(g, mask, a, x, y, z);
        const double hi = o[idx3(ux, uy, uz, ex, ey)] / fluid_neighbours_of_face(g, mask, a, ux, uy, uz);
        double* f = component<double>(fa.x, fa.y, fa.z, a);
        const double v = static_cast<double>(g.dt) * lo + static_cast<double>(g.dt) * hi;
        if (kAssign) f[i] = v; else f[i] += v;
    }
}

// The same without colliders: a face has two fluid cells beside it unless it
// lies on the domain boundary (one), so the division by the count is an exact
// halving or nothing; bit-identical to integrate_vjp_cells_kernel.
template <bool kAssign>
__global__ void integrate_vjp_open_cells_kernel(Grid g, XsAdjointVector oa, XsAdjointVector fa) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int ex = extent(g, a, 0), ey = extent(g, a, 1);
        const double* o = component<double>(oa.x, oa.y, oa.z, a);
        const int ux = x + (a == 0), uy = y + (a == 1), uz = z + (a == 2);
        const int c = a == 0 ? x : (a == 1 ? y : z), n = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
        double lo = o[idx3(x, y, z, ex, ey)], hi = o[idx3(ux, uy, uz, ex, ey)];
        if (c > 0) lo *= 0.5;
        if (c + 1 < n) hi *= 0.5;
        double* f = component<double>(fa.x, fa.y, fa.z, a);
        const double v = static_cast<double>(g.dt) * lo + static_cast<double>(g.dt) * hi;
        if (kAssign) f[i] = v; else f[i] += v;
    }
}

// Shared tail of both advection adjoints (operators.cu:426-438, 548-560):
// adjoint of value1 through the final position, midpoint sample gradients,
// then of value0 at the start.
__device__ __forceinline__ void trace_adjoint(const Vec3& start, const Vec3& mid, const Trace& t, const Vec3& src_gradient, double o,
                                              const XsVector& u, const Grid& g, const XsVelocityBoundary& vb, const XsAdjointVector& ua) {
    const double v1x = -static_cast<double>(t.derivative.x * g.dt * src_gradient.x) * o;
    const double v1y = -static_cast<double>(t.derivative.y * g.dt * src_gradient.y) * o;
    const double v1z = -static_cast<double>(t.derivative.z * g.dt * src_gradient.z) * o;
    const Sample m0 = sample_face<true>(u.x, 0, mid, g, vb);
    const Sample m1 = sample_face<true>(u.y, 1, mid, g, vb);
    const Sample m2 = sample_face<true>(u.z, 2, mid, g, vb);
    scatter_face(ua.x, 0, mid, v1x, g, vb);
    scatter_face(ua.y, 1, mid, v1y, g, vb);
    scatter_face(ua.z, 2, mid, v1z, g, vb);
    const double mx = m0.gradient.x * v1x + m1.gradient.x * v1y + m2.gradient.x * v1z;
    const double my = m0.gradient.y * v1x + m1.gradient.y * v1y + m2.gradient.y * v1z;
    const double mz = m0.gradient.z * v1x + m1.gradient.z * v1y + m2.gradient.z * v1z;
    scatter_face(ua.x, 0, start, -0.5 * static_cast<double>(g.dt) * mx, g, vb);
    scatter_face(ua.y, 1, start, -0.5 * static_cast<double>(g.dt) * my, g, vb);
    scatter_face(ua.z, 2, start, -0.5 * static_cast<double>(g.dt) * mz, g, vb);
}

// operators.cu:415-439, one face (general form: colliders, any spacing).
__device__ __forceinline__ void advect_velocity_vjp_face(int a, int x, int y, int z, double o, const Grid& g, const uint32_t* __restrict__ mask,
                                                         const XsVector& u, const XsVelocityBoundary& vb, const XsAdjointVector& ua) {
    const Vec3 s = face_position(a, x, y, z, g);
    const Vec3 v0 = sample_velocity(u.x, u.y, u.z, s, g, vb);
    const Vec3 mid{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    const Trace t = trace_rk2(s, u.x, u.y, u.z, mask, g, vb);
    const Sample src = sample_face<true>(component<const float>(u.x, u.y, u.z, a), a, t.position, g, vb);
    scatter_face(component<double>(ua.x, ua.y, ua.z, a), a, t.position, o, g, vb);
    trace_adjoint(s, mid, t, src.gradient, o, u, g, vb, ua);
}

// operators.cu:415-439 for all three components in one launch.
__global__ void advect_velocity_vjp_kernel(const __grid_constant__ Grid g, uint64_t f0, uint64_t f1, uint64_t f2, const uint32_t* __restrict__ mask, XsVector u,
                                           const __grid_constant__ XsVelocityBoundary vb, XsAdjointVector oa, XsAdjointVector ua) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= f0 + f1 + f2) return;
    int a;
    uint64_t local;
    if (i < f0) { a = 0; local = i; } else if (i < f0 + f1) { a = 1; local = i - f0; } else { a = 2; local = i - f0 - f1; }
    const double o = component<double>(oa.x, oa.y, oa.z, a)[local];
    if (o == 0.0) return;
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    advect_velocity_vjp_face(a, x, y, z, o, g, mask, u, vb, ua);
}

// ------------------------------------------------ tile-staged adjoints
// Grids without colliders and with a power-of-two spacing (advect_tile.cuh).
// u is staged over the tile's box; every scatter of the transposed trilinear
// gathers goes to FP64 box accumulators in shared memory, and each touched
// box node is added to global memory once at the end (instead of 56 global
// atomics per face).  The same products as the general kernels; only the
// order of the FP64 additions differs.
// Halo 1: the box holds every stencil of traces shorter than half a cell per
// step (longer ones scatter to global memory); the smaller boxes give five
// velocity-adjoint CTAs per SM (96 registers: 6.49 against 6.88 ms at 256^3
// with four; six spill) and three density-and-temperature ones.
using AdjointTile = tile::Shape<32, 4, 4, 1>;
constexpr size_t kVelocityVjpSmem = 3 * AdjointTile::kNodes * (sizeof(double) + sizeof(float));
constexpr size_t kScalarVjpSmem = 5 * AdjointTile::kNodes * (sizeof(double) + sizeof(float));

// The trace adjoint of one sample at the trace end (operators.cu:426-438):
// through the end position to the midpoint samples (their gradients m), and
// through the midpoint to the start (exact start weights).  A is the face
// component at run time (a cell centre for the scalar adjoints: cell).
__device__ __forceinline__ void staged_trace_adjoint(int A, const Vec3& mid, const Sample (&m)[3], const Vec3& der, const Vec3& src_gradient,
                                                     double o, int li, double* const (&acc)[3], const tile::Origin& org,
                                                     const tile::TileConsts& k, const Grid& g, const XsVelocityBoundary& vb,
                                                     const XsAdjointVector& ua, bool cell) {
    using S = AdjointTile;
    const double v1x = -static_cast<double>(der.x * g.dt * src_gradient.x) * o;
    const double v1y = -static_cast<double>(der.y * g.dt * src_gradient.y) * o;
    const double v1z = -static_cast<double>(der.z * g.dt * src_gradient.z) * o;
    tile::staged_face_scatter<S, 0>(acc[0], ua.x, mid, v1x, org, k, g, vb);
    tile::staged_face_scatter<S, 1>(acc[1], ua.y, mid, v1y, org, k, g, vb);
    tile::staged_face_scatter<S, 2>(acc[2], ua.z, mid, v1z, org, k, g, vb);
    const double mx = m[0].gradient.x * v1x + m[1].gradient.x * v1y + m[2].gradient.x * v1z;
    const double my = m[0].gradient.y * v1x + m[1].gradient.y * v1y + m[2].gradient.y * v1z;
    const double mz = m[0].gradient.z * v1x + m[1].gradient.z * v1y + m[2].gradient.z * v1z;
    const double h = -0.5 * static_cast<double>(g.dt);
    if (cell) {
        tile::cell_start_scatter<S, 0>(acc[0], li, h * mx);
        tile::cell_start_scatter<S, 1>(acc[1], li, h * my);
        tile::cell_start_scatter<S, 2>(acc[2], li, h * mz);
    } else {
        tile::face_start_scatter_rt<S, 0>(acc[0], li, A, h * mx);
        tile::face_start_scatter_rt<S, 1>(acc[1], li, A, h * my);
        tile::face_start_scatter_rt<S, 2>(acc[2], li, A, h * mz);
    }
}

// Midpoint samples (values and gradients) and the clamped end of the trace
// from a start with known velocity.
__device__ __forceinline__ Vec3 staged_trace_with_samples(const tile::StagedVelocity& sv, const Vec3& s, const Vec3& v0, const tile::Origin& org,
                                                          const tile::TileConsts& k, const Grid& g, const XsVelocityBoundary& vb, Vec3& mid,
                                                          Sample (&m)[3], Vec3& der) {
    using S = AdjointTile;
    mid = Vec3{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    m[0] = tile::staged_face<S, 0, true>(sv.s[0], sv.u.x, mid, org, k, g, vb);
    m[1] = tile::staged_face<S, 1, true>(sv.s[1], sv.u.y, mid, org, k, g, vb);
    m[2] = tile::staged_face<S, 2, true>(sv.s[2], sv.u.z, mid, org, k, g, vb);
    Vec3 raw{s.x - g.dt * m[0].value, s.y - g.dt * m[1].value, s.z - g.dt * m[2].value};
    der = Vec3{1.0f, 1.0f, 1.0f};
    tile::clamp_trace(raw, der, k);
    return raw;
}

// One face of component A (run time: the kernel loops over the components
// with one copy of this body).
__device__ __forceinline__ void advect_velocity_vjp_tile_face(int A, int x, int y, int z, int li, const tile::StagedVelocity& sv,
                                                              double* const (&acc)[3], const tile::Origin& org, const tile::TileConsts& k,
                                                              const Grid& g, const XsVelocityBoundary& vb, const XsAdjointVector& oa,
                                                              const XsAdjointVector& ua) {
    using S = AdjointTile;
    const double o = component<const double>(oa.x, oa.y, oa.z, A)[tile::index32(x, y, z, extent(g, A, 0), extent(g, A, 1))];
    if (o == 0.0) return;
    const Vec3 s = face_position(A, x, y, z, g);
    Vec3 mid, der;
    Sample m[3];
    const Vec3 end = staged_trace_with_samples(sv, s, tile::face_start_velocity_rt<S>(sv, li, A), org, k, g, vb, mid, m, der);
    const Sample src = tile::staged_face_rt<S>(sv.s[A], component<const float>(sv.u.x, sv.u.y, sv.u.z, A), A, end, org, k, g, vb);
    tile::staged_face_scatter_rt<S>(acc[A], component<double>(ua.x, ua.y, ua.z, A), A, end, o, org, k, g, vb);
    staged_trace_adjoint(A, mid, m, der, src.gradient, o, li, acc, org, k, g, vb, ua, false);
}

__global__ void __launch_bounds__(AdjointTile::kThreads, 5) advect_velocity_vjp_tile_kernel(const __grid_constant__ Grid g, XsVector u, const __grid_constant__ XsVelocityBoundary vb,
                                                                                          XsAdjointVector oa, XsAdjointVector ua) {
    using S = AdjointTile;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* const acc[3] = {reinterpret_cast<double*>(smem_raw), reinterpret_cast<double*>(smem_raw) + S::kNodes,
                            reinterpret_cast<double*>(smem_raw) + 2 * S::kNodes};
    float* box = reinterpret_cast<float*>(acc[0] + 3 * S::kNodes);
    const tile::Origin org = tile::tile_origin<S>();
    tile::stage_face<S, 0>(box, u.x, org, g, vb);
    tile::stage_face<S, 1>(box + S::kNodes, u.y, org, g, vb);
    tile::stage_face<S, 2>(box + 2 * S::kNodes, u.z, org, g, vb);
    tile::zero_box<S>(acc[0]);
    tile::zero_box<S>(acc[1]);
    tile::zero_box<S>(acc[2]);
    tile::stage_wait();
    __syncthreads();
    const tile::StagedVelocity sv{{box, box + S::kNodes, box + 2 * S::kNodes}, u};
    const tile::TileConsts k = tile::tile_consts(g, vb);
    const int x = static_cast<int>(blockIdx.x) * S::TX + static_cast<int>(threadIdx.x);
    const int y = static_cast<int>(blockIdx.y) * S::TY + static_cast<int>(threadIdx.y);
    if (x < g.nx && y < g.ny) {
#pragma unroll 1
        for (int kz = 0; kz < S::TZ; ++kz) {
            const int z = static_cast<int>(blockIdx.z) * S::TZ + kz;
            if (z >= g.nz) break;
            const int li = tile::local_index<S>(kz);
#pragma unroll 1
            for (int A = 0; A < 3; ++A) advect_velocity_vjp_tile_face(A, x, y, z, li, sv, acc, org, k, g, vb, oa, ua);
        }
    }
    __syncthreads();
    tile::flush_face<S, 0>(acc[0], ua.x, org, g, vb);
    tile::flush_face<S, 1>(acc[1], ua.y, org, g, vb);
    tile::flush_face<S, 2>(acc[2], ua.z, org, g, vb);
}

// The faces at the upper end of their own axis, general form.
__global__ void advect_velocity_vjp_upper_kernel(const __grid_constant__ Grid g, const uint32_t* __restrict__ mask, XsVector u, const __grid_constant__ XsVelocityBoundary vb,
                                                 XsAdjointVector oa, XsAdjointVector ua) {
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
    const double o = component<double>(oa.x, oa.y, oa.z, a)[idx3(x, y, z, extent(g, a, 0), extent(g, a, 1))];
    if (o == 0.0) return;
    advect_velocity_vjp_face(a, x, y, z, o, g, mask, u, vb, ua);
}

// Density and temperature together (operators.cu:537-561 twice on one
// trace): u and both sources staged, the velocity and both source adjoints
// accumulated in the box.
__global__ void __launch_bounds__(AdjointTile::kThreads, 3) advect_scalar_vjp_tile_kernel(const __grid_constant__ Grid g, const float* __restrict__ src,
                                                                                        const __grid_constant__ XsScalarBoundary sb, const double* __restrict__ oa,
                                                                                        double* __restrict__ sa, const float* __restrict__ src2,
                                                                                        const __grid_constant__ XsScalarBoundary sb2, const double* __restrict__ oa2,
                                                                                        double* __restrict__ sa2, XsVector u,
                                                                                        const __grid_constant__ XsVelocityBoundary vb, XsAdjointVector ua) {
    using S = AdjointTile;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* const acc[3] = {reinterpret_cast<double*>(smem_raw), reinterpret_cast<double*>(smem_raw) + S::kNodes,
                            reinterpret_cast<double*>(smem_raw) + 2 * S::kNodes};
    double* const sacc[2] = {acc[0] + 3 * S::kNodes, acc[0] + 4 * S::kNodes};
    float* box = reinterpret_cast<float*>(acc[0] + 5 * S::kNodes);
    const bool two = oa2 != nullptr;
    const tile::Origin org = tile::tile_origin<S>();
    tile::stage_face<S, 0>(box, u.x, org, g, vb);
    tile::stage_face<S, 1>(box + S::kNodes, u.y, org, g, vb);
    tile::stage_face<S, 2>(box + 2 * S::kNodes, u.z, org, g, vb);
    tile::stage_cells<S>(box + 3 * S::kNodes, src, org, g, sb);
    if (two) tile::stage_cells<S>(box + 4 * S::kNodes, src2, org, g, sb2);
    for (int k = 0; k < 5; ++k) tile::zero_box<S>(acc[0] + k * S::kNodes);
    tile::stage_wait();
    __syncthreads();
    const tile::StagedVelocity sv{{box, box + S::kNodes, box + 2 * S::kNodes}, u};
    const tile::TileConsts k = tile::tile_consts(g, vb);
    const int x = static_cast<int>(blockIdx.x) * S::TX + static_cast<int>(threadIdx.x);
    const int y = static_cast<int>(blockIdx.y) * S::TY + static_cast<int>(threadIdx.y);
    if (x < g.nx && y < g.ny) {
#pragma unroll 1
        for (int kz = 0; kz < S::TZ; ++kz) {
            const int z = static_cast<int>(blockIdx.z) * S::TZ + kz;
            if (z >= g.nz) break;
            const uint32_t i = tile::index32(x, y, z, g.nx, g.ny);
            const double o1 = oa[i];
            const double o2 = two ? oa2[i] : 0.0;
            if (o1 == 0.0 && o2 == 0.0) continue;
            const int li = tile::local_index<S>(kz);
            const Vec3 s = cell_position(x, y, z, g);
            Vec3 mid, der;
            Sample m[3];
            const Vec3 end = staged_trace_with_samples(sv, s, tile::cell_start_velocity<S>(sv, li), org, k, g, vb, mid, m, der);
            const Sample smp = tile::staged_scalar<S, true>(box + 3 * S::kNodes, src, end, org, k, g, sb);
            tile::staged_scalar_scatter<S>(sacc[0], sa, end, o1, org, k, g, sb);
            if (o1 != 0.0) staged_trace_adjoint(0, mid, m, der, smp.gradient, o1, li, acc, org, k, g, vb, ua, true);
            if (two && o2 != 0.0) {
                const Sample smp2 = tile::staged_scalar<S, true>(box + 4 * S::kNodes, src2, end, org, k, g, sb2);
                tile::staged_scalar_scatter<S>(sacc[1], sa2, end, o2, org, k, g, sb2);
                staged_trace_adjoint(0, mid, m, der, smp2.gradient, o2, li, acc, org, k, g, vb, ua, true);
            }
        }
    }
    __syncthreads();
    tile::flush_face<S, 0>(acc[0], ua.x, org, g, vb);
    tile::flush_face<S, 1>(acc[1], ua.y, org, g, vb);
    tile::flush_face<S, 2>(acc[2], ua.z, org, g, vb);
    tile::flush_cells<S>(sacc[0], sa, org, g, sb);
    if (two) tile::flush_cells<S>(sacc[1], sa2, org, g, sb2);
}

// operators.cu:537-561; density and temperature share one trace when both
// adjoints are requested (sa2/oa2 non-null).
__global__ void advect_scalar_vjp_kernel(const __grid_constant__ Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ src, const __grid_constant__ XsScalarBoundary sb,
                                         const double* __restrict__ oa, double* __restrict__ sa, const float* __restrict__ src2,
                                         const __grid_constant__ XsScalarBoundary sb2, const double* __restrict__ oa2, double* __restrict__ sa2, XsVector u,
                                         const __grid_constant__ XsVelocityBoundary vb, XsAdjointVector ua) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g) || is_solid(mask, i)) return;
    const double o1 = oa[i];
    const double o2 = oa2 ? oa2[i] : 0.0;
    if (o1 == 0.0 && o2 == 0.0) return;
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const Vec3 s = cell_position(x, y, z, g);
    const Vec3 v0 = sample_velocity(u.x, u.y, u.z, s, g, vb);
    const Vec3 mid{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    const Trace t = trace_rk2(s, u.x, u.y, u.z, mask, g, vb);
    const Sample smp = sample_scalar<true>(src, t.position, g, sb);
    scatter_scalar(sa, t.position, o1, g, sb);
    trace_adjoint(s, mid, t, smp.gradient, o1, u, g, vb, ua);
    if (oa2 && o2 != 0.0) {
        const Sample smp2 = sample_scalar<true>(src2, t.position, g, sb2);
        scatter_scalar(sa2, t.position, o2, g, sb2);
        trace_adjoint(s, mid, t, smp2.gradient, o2, u, g, vb, ua);
    }
}

// ---------------------------------------------------------------- constrain
// operators.cu:483-497 gathered per face: a face receives its own output
// adjoint unless it is constrained or beside a solid; on a periodic axis
// the face at coordinate 0 also receives its upper partner's.
__device__ __forceinline__ bool constrained_or_solid(int a, int x, int y, int z, const Grid& g, const uint32_t* mask,
                                                     const XsVelocityBoundary& b) {
    const int coord = a == 0 ? x : (a == 1 ? y : z);
    const int mx = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
    if (coord == 0 || coord == mx) {
        const uint32_t mode = b.modes[a * 2 + (coord == mx)];
        if (mode == 0u || mode == 2u) return true;
    }
    if (mask != nullptr) {
        const int lx = x - (a == 0), ly = y - (a == 1), lz = z - (a == 2);
        if (in_grid(g, lx, ly, lz) && __ldg(mask + idx3(lx, ly, lz, g.nx, g.ny)) != 0u) return true;
        if (in_grid(g, x, y, z) && __ldg(mask + idx3(x, y, z, g.nx, g.ny)) != 0u) return true;
    }
    return false;
}

template <bool kAssign>
__global__ void constrain_vjp_kernel(Grid g, uint64_t f0, uint64_t f1, uint64_t f2, const uint32_t* __restrict__ mask, XsAdjointVector oa,
                                     XsVelocityBoundary b, XsAdjointVector ua) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= f0 + f1 + f2) return;
    int a;
    uint64_t local;
    if (i < f0) { a = 0; local = i; } else if (i < f0 + f1) { a = 1; local = i - f0; } else { a = 2; local = i - f0 - f1; }
    int x, y, z;
    const int ex = extent(g, a, 0), ey = extent(g, a, 1);
    decode(local, ex, ey, x, y, z);
    const double* o = component<double>(oa.x, oa.y, oa.z, a);
    const int coord = a == 0 ? x : (a == 1 ? y : z);
    const int mx = a == 0 ? g.nx : (a == 1 ? g.ny : g.nz);
    const bool per = periodic(b, a);
    double acc = 0.0;
    if (!constrained_or_solid(a, x, y, z, g, mask, b) && !(per && coord == mx)) acc += o[local];
    if (per && coord == 0) {
        const int px = a == 0 ? mx : x, py = a == 1 ? mx : y, pz = a == 2 ? mx : z;
        if (!constrained_or_solid(a, px, py, pz, g, mask, b)) acc += o[idx3(px, py, pz, ex, ey)];
    }
    if (kAssign) component<double>(ua.x, ua.y, ua.z, a)[local] = acc;
    else if (acc != 0.0) component<double>(ua.x, ua.y, ua.z, a)[local] += acc;
}

// ---------------------------------------------------------------- projection
// operators.cu:904-910 for the two cells beside a face.
__device__ __forceinline__ bool projectable(const Grid& g, int a, int x, int y, int z, const uint32_t* mask) {
    const int fx = x - (a == 0), fy = y - (a == 1), fz = z - (a == 2);
    if (!in_grid(g, fx, fy, fz) || !in_grid(g, x, y, z)) return false;
    return !is_solid(mask, idx3(fx, fy, fz, g.nx, g.ny)) && !is_solid(mask, idx3(x, y, z, g.nx, g.ny));
}

// operators.cu:922-933, cell part gathered: lambda_p of a cell from the
// output adjoint of its projectable faces (+ on the upper face, - on the lower).
__global__ void project_reverse_cells_kernel(Grid g, const uint32_t* __restrict__ mask, XsAdjointVector oa, double* __restrict__ pa) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const double s = static_cast<double>(g.dt) / g.h;
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int ex = extent(g, a, 0), ey = extent(g, a, 1);
        const double* o = component<double>(oa.x, oa.y, oa.z, a);
        const int ux = x + (a == 0), uy = y + (a == 1), uz = z + (a == 2);
        if (projectable(g, a, ux, uy, uz, mask)) acc += s * o[idx3(ux, uy, uz, ex, ey)];
        if (projectable(g, a, x, y, z, mask)) acc -= s * o[idx3(x, y, z, ex, ey)];
    }
    pa[i] = acc;
}

// operators.cu:957-969 gathered per face, plus the face part of :922-933
// (velocity adjoint += output adjoint).  scale(c) = -h * rhs_adj(c) / dt for
// fluid, non-anchor cells; the face gets scale(lower) - scale(upper).
template <bool kAssign>
__global__ void pressure_rhs_reverse_kernel(Grid g, uint64_t f0, uint64_t f1, uint64_t f2, uint32_t anchor, const uint32_t* __restrict__ mask,
                                            const double* __restrict__ rhs_adj, XsAdjointVector oa, XsAdjointVector ua) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= f0 + f1 + f2) return;
    int a;
    uint64_t local;
    if (i < f0) { a = 0; local = i; } else if (i < f0 + f1) { a = 1; local = i - f0; } else { a = 2; local = i - f0 - f1; }
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    double acc = oa.x ? component<double>(oa.x, oa.y, oa.z, a)[local] : 0.0;
    const double k = -static_cast<double>(g.h) / static_cast<double>(g.dt);
    const int lx = x - (a == 0), ly = y - (a == 1), lz = z - (a == 2);
    if (in_grid(g, lx, ly, lz)) {
        const uint64_t c = idx3(lx, ly, lz, g.nx, g.ny);
        if (!is_solid(mask, c) && c != anchor) acc += k * rhs_adj[c];
    }
    if (in_grid(g, x, y, z)) {
        const uint64_t c = idx3(x, y, z, g.nx, g.ny);
        if (!is_solid(mask, c) && c != anchor) acc -= k * rhs_adj[c];
    }
    if (kAssign) component<double>(ua.x, ua.y, ua.z, a)[local] = acc;
    else component<double>(ua.x, ua.y, ua.z, a)[local] += acc;
}

// ---------------------------------------------------------------- launchers
XsStatus launch_source_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const double* oa, const InflowSet& inflows, double* sa,
                           double* ra) {
    source_vjp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, oa, inflows, sa, ra);
    return check_launch();
}

XsStatus launch_buoyancy_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho, const float* temp, const float* ambient,
                             const float* beta_rho, const float* beta_temp, const XsAdjointVector& fa, double* rho_a, double* temp_a,
                             const XsAdjointVector& ea, double* amb_a, double* br_a, double* bt_a) {
    buoyancy_vjp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, rho, temp, ambient, beta_rho, beta_temp, fa, rho_a, temp_a,
                                                                       ea, amb_a, br_a, bt_a);
    return check_launch();
}

XsStatus launch_integrate_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsAdjointVector& oa, const XsAdjointVector& ua,
                              const XsAdjointVector& fa, bool assign_force) {
    for (int a = 0; a < 3; ++a) {
        const uint64_t n = face_count(g, a);
        integrate_vjp_faces_kernel<<<blocks_for(n), kBlock, 0, st>>>(n, component<double>(oa.x, oa.y, oa.z, a),
                                                                     component<double>(ua.x, ua.y, ua.z, a));
        if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    }
    const unsigned blocks = blocks_for(cell_count(g));
    if (mask == nullptr && assign_force)
        integrate_vjp_open_cells_kernel<true><<<blocks, kBlock, 0, st>>>(g, oa, fa);
    else if (mask == nullptr)
        integrate_vjp_open_cells_kernel<false><<<blocks, kBlock, 0, st>>>(g, oa, fa);
    else if (assign_force)
        integrate_vjp_cells_kernel<true><<<blocks, kBlock, 0, st>>>(g, mask, oa, fa);
    else
        integrate_vjp_cells_kernel<false><<<blocks, kBlock, 0, st>>>(g, mask, oa, fa);
    return check_launch();
}

XsStatus launch_advect_velocity_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVelocityBoundary& vb,
                                    const XsAdjointVector& oa, const XsAdjointVector& ua) {
    if (tile::tiled_advection(g, mask)) {
        static DeviceOnce configured;
        if (!configured.run([] {
                return cudaFuncSetAttribute(advect_velocity_vjp_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kVelocityVjpSmem));
            }))
            return XS_CUDA_ERROR;
        advect_velocity_vjp_tile_kernel<<<tile::tile_grid<AdjointTile>(g), tile::tile_block<AdjointTile>(), kVelocityVjpSmem, st>>>(g, u, vb,
                                                                                                                                  oa, ua);
        XsStatus s = check_launch();
        if (s != XS_OK) return s;
        const uint64_t upper = static_cast<uint64_t>(g.ny) * g.nz + static_cast<uint64_t>(g.nx) * g.nz + static_cast<uint64_t>(g.nx) * g.ny;
        advect_velocity_vjp_upper_kernel<<<blocks_for(upper), kBlock, 0, st>>>(g, mask, u, vb, oa, ua);
        return check_launch();
    }
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    advect_velocity_vjp_kernel<<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, mask, u, vb, oa, ua);
    return check_launch();
}

XsStatus launch_advect_scalar_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* src, const XsScalarBoundary& sb,
                                  const double* oa, double* sa, const float* src2, const XsScalarBoundary& sb2, const double* oa2,
                                  double* sa2, const XsVector& u, const XsVelocityBoundary& vb, const XsAdjointVector& ua) {
    if (tile::tiled_advection(g, mask)) {
        static DeviceOnce configured;
        if (!configured.run([] {
                return cudaFuncSetAttribute(advect_scalar_vjp_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(kScalarVjpSmem));
            }))
            return XS_CUDA_ERROR;
        advect_scalar_vjp_tile_kernel<<<tile::tile_grid<AdjointTile>(g), tile::tile_block<AdjointTile>(), kScalarVjpSmem, st>>>(
            g, src, sb, oa, sa, src2, sb2, oa2, sa2, u, vb, ua);
        return check_launch();
    }
    advect_scalar_vjp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, src, sb, oa, sa, src2, sb2, oa2, sa2, u, vb, ua);
    return check_launch();
}

XsStatus launch_constrain_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsAdjointVector& oa, const XsVelocityBoundary& b,
                              const XsAdjointVector& ua, bool assign) {
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    if (assign)
        constrain_vjp_kernel<true><<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, mask, oa, b, ua);
    else
        constrain_vjp_kernel<false><<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, mask, oa, b, ua);
    return check_launch();
}

// projection_vjp (operators.cu:1020-1031): pa, ra are cell scratch; the
// output adjoint passes to velocity_adjoint, lambda_p is solved (PCG kind)
// or reverse-swept (RBGS kind), and the divergence transpose is added.
XsStatus projection_vjp(cudaStream_t st, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                        const XsAdjointVector& oa, const XsScalarBoundary& pb, double* pa, double* ra, const XsAdjointVector& ua,
                        void* workspace, const WarmHistory* history, bool assign) {
    project_reverse_cells_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, oa, pa);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    XsStatus s;
    if (solve.kind == XS_SOLVER_RED_BLACK_GAUSS_SEIDEL) {
        if (cudaMemsetAsync(ra, 0, sizeof(double) * cell_count(g), st) != cudaSuccess) return XS_CUDA_ERROR;
        s = reverse_rbgs(st, g, solve.max_iterations, anchor, mask, pb, pa, ra, workspace);
    } else {
        XsPressureSolve adj = solve;
        adj.initial_guess = nullptr;
        adj.scale_guess = 0u;
        const bool ring = history && history->history > 0;
        const bool coarse = ring && history->coarsening != 0 && mask == nullptr;
        if (ring) {
            // successive adjoint solves of a reverse pass are related: Galerkin
            // start from the ring of previous adjoint solutions, then (with
            // coarsening) kAdjointStartCycles rounds of sweeps and an
            // energy-optimal step along the coarse-grid correction of the
            // residual (the forward solve takes one)
            const WarmHistory& h = *history;
            if ((s = galerkin_combine(st, g, anchor, mask, pb, h, true, nullptr, 0, nullptr, h.ring_start, pa)) != XS_OK) return s;
            adj.initial_guess = h.ring_start;
            if (coarse) {
                const float* x = nullptr;
                if ((s = coarse_cycles(st, g, anchor, pb, h, nullptr, pa, kAdjointStartCycles, &x)) != XS_OK) return s;
                adj.initial_guess = x;
            }
        }
        s = solve_pressure(st, g, adj, anchor, mask, pb, nullptr, pa, nullptr, ra, workspace, nullptr);
        if (s == XS_OK && coarse) s = record_coarse_iterations(st, *history, workspace, g);
        if (s == XS_OK && ring) s = history_push(st, g, anchor, mask, pb, *history, nullptr, ra);
    }
    if (s != XS_OK) return s;
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    if (assign)
        pressure_rhs_reverse_kernel<true><<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, anchor, mask, ra, oa, ua);
    else
        pressure_rhs_reverse_kernel<false><<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, anchor, mask, ra, oa, ua);
    return check_launch();
}

}  // namespace xs

using namespace xs;

extern "C" {

XsStatus xs_source_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const double* output_adjoint, const XsInflow* inflows,
                       uint32_t inflow_count, double* state_adjoint, double* source_adjoint) {
    if (!valid_grid(grid) || !output_adjoint || !state_adjoint || !source_adjoint || inflow_count > XS_MAX_INFLOWS) return XS_INVALID_ARGUMENT;
    return launch_source_vjp(stream, make_grid(grid), cell_mask, output_adjoint, make_inflows(inflows, inflow_count), state_adjoint,
                             source_adjoint);
}

XsStatus xs_buoyancy_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* density, const float* temperature,
                         const float* ambient_temperature, const float* density_buoyancy, const float* temperature_buoyancy,
                         XsAdjointVector force_adjoint, double* density_adjoint, double* temperature_adjoint,
                         XsAdjointVector external_acceleration_adjoint, double* ambient_temperature_adjoint,
                         double* density_buoyancy_adjoint, double* temperature_buoyancy_adjoint) {
    if (!valid_grid(grid) || !density || !temperature || !ambient_temperature || !density_buoyancy || !temperature_buoyancy ||
        !valid(force_adjoint) || !density_adjoint || !temperature_adjoint || !valid(external_acceleration_adjoint) ||
        !ambient_temperature_adjoint || !density_buoyancy_adjoint || !temperature_buoyancy_adjoint)
        return XS_INVALID_ARGUMENT;
    return launch_buoyancy_vjp(stream, make_grid(grid), cell_mask, density, temperature, ambient_temperature, density_buoyancy,
                               temperature_buoyancy, force_adjoint, density_adjoint, temperature_adjoint, external_acceleration_adjoint,
                               ambient_temperature_adjoint, density_buoyancy_adjoint, temperature_buoyancy_adjoint);
}

XsStatus xs_integrate_velocity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsAdjointVector output_adjoint,
                                   XsAdjointVector velocity_adjoint, XsAdjointVector force_adjoint) {
    if (!valid_grid(grid) || !valid(output_adjoint) || !valid(velocity_adjoint) || !valid(force_adjoint)) return XS_INVALID_ARGUMENT;
    return launch_integrate_vjp(stream, make_grid(grid), cell_mask, output_adjoint, velocity_adjoint, force_adjoint);
}

XsStatus xs_advect_velocity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, XsVelocityBoundary boundary,
                                XsAdjointVector output_adjoint, XsAdjointVector velocity_adjoint) {
    if (!valid_grid(grid) || !valid(velocity) || !valid(output_adjoint) || !valid(velocity_adjoint)) return XS_INVALID_ARGUMENT;
    return launch_advect_velocity_vjp(stream, make_grid(grid), cell_mask, velocity, boundary, output_adjoint, velocity_adjoint);
}

XsStatus xs_constrain_velocity_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsAdjointVector output_adjoint,
                                   XsVelocityBoundary boundary, XsAdjointVector velocity_adjoint) {
    if (!valid_grid(grid) || !valid(output_adjoint) || !valid(velocity_adjoint)) return XS_INVALID_ARGUMENT;
    return launch_constrain_vjp(stream, make_grid(grid), cell_mask, output_adjoint, boundary, velocity_adjoint);
}

XsStatus xs_advect_scalar_vjp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* source, XsVector velocity,
                              XsScalarBoundary scalar_boundary, XsVelocityBoundary velocity_boundary, const double* output_adjoint,
                              double* source_adjoint, XsAdjointVector velocity_adjoint) {
    if (!valid_grid(grid) || !source || !valid(velocity) || !output_adjoint || !source_adjoint || !valid(velocity_adjoint))
        return XS_INVALID_ARGUMENT;
    return launch_advect_scalar_vjp(stream, make_grid(grid), cell_mask, source, scalar_boundary, output_adjoint, source_adjoint, nullptr,
                                    scalar_boundary, nullptr, nullptr, velocity, velocity_boundary, velocity_adjoint);
}

XsStatus xs_projection_vjp(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                           const uint32_t* cell_mask, XsAdjointVector output_adjoint, XsVelocityBoundary velocity_boundary,
                           XsScalarBoundary pressure_boundary, double* pressure_adjoint, double* rhs_adjoint,
                           XsAdjointVector velocity_adjoint, void* workspace) {
    (void)velocity_boundary;
    if (!valid_grid(grid) || !solve || !valid(output_adjoint) || !pressure_adjoint || !rhs_adjoint || !valid(velocity_adjoint) || !workspace)
        return XS_INVALID_ARGUMENT;
    return projection_vjp(stream, make_grid(grid), *solve, pressure_anchor, cell_mask, output_adjoint, pressure_boundary, pressure_adjoint,
                          rhs_adjoint, velocity_adjoint, workspace);
}

}  // extern "C"
