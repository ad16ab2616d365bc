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
        f[i] += static_cast<double>(g.dt) * lo + static_cast<double>(g.dt) * hi;
    }
}

// ---------------------------------------------------------------- scatter
__device__ __forceinline__ void scatter_scalar(double* v, const Vec3& p, double adj, const Grid& g, const XsScalarBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates(p, g.h, -1, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const double wx[2] = {1.0 - (gx - x0), static_cast<double>(gx - x0)};
    const double wy[2] = {1.0 - (gy - y0), static_cast<double>(gy - y0)};
    const double wz[2] = {1.0 - (gz - z0), static_cast<double>(gz - z0)};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int x = x0 + dx, y = y0 + dy, z = z0 + dz;
                if ((x < 0 && b.modes[0] == 0u) || (beyond(x, g.nx) && b.modes[1] == 0u) || (y < 0 && b.modes[2] == 0u) ||
                    (beyond(y, g.ny) && b.modes[3] == 0u) || (z < 0 && b.modes[4] == 0u) || (beyond(z, g.nz) && b.modes[5] == 0u))
                    continue;
                atomicAdd(v + mapped_cell(x, y, z, g, periodic(b, 0), periodic(b, 1), periodic(b, 2)), adj * wx[dx] * wy[dy] * wz[dz]);
            }
}

// operators.cu:217-240
__device__ __forceinline__ void scatter_face(double* v, int axis, const Vec3& p, double adj, const Grid& g, const XsVelocityBoundary& b) {
    if (adj == 0.0) return;
    float gx, gy, gz;
    grid_coordinates(p, g.h, axis, gx, gy, gz);
    const int x0 = static_cast<int>(floorf(gx)), y0 = static_cast<int>(floorf(gy)), z0 = static_cast<int>(floorf(gz));
    const double wx[2] = {1.0 - (gx - x0), static_cast<double>(gx - x0)};
    const double wy[2] = {1.0 - (gy - y0), static_cast<double>(gy - y0)};
    const double wz[2] = {1.0 - (gz - z0), static_cast<double>(gz - z0)};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int c[3] = {x0 + dx, y0 + dy, z0 + dz};
                bool constant = false;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int size = extent(g, axis, d);
                    if (c[d] >= 0 && c[d] < size) continue;
                    const int face = 2 * d + (c[d] >= size);
                    if (b.modes[face] == 0u || (b.modes[face] == 2u && axis == d)) constant = true;
                }
                if (!constant) atomicAdd(v + mapped_face(c[0], c[1], c[2], g, axis, b), adj * wx[dx] * wy[dy] * wz[dz]);
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

// operators.cu:415-439 for all three components in one launch.
__global__ void advect_velocity_vjp_kernel(Grid g, uint64_t f0, uint64_t f1, uint64_t f2, const uint32_t* __restrict__ mask, XsVector u,
                                           XsVelocityBoundary vb, XsAdjointVector oa, XsAdjointVector ua) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= f0 + f1 + f2) return;
    int a;
    uint64_t local;
    if (i < f0) { a = 0; local = i; } else if (i < f0 + f1) { a = 1; local = i - f0; } else { a = 2; local = i - f0 - f1; }
    const double o = component<double>(oa.x, oa.y, oa.z, a)[local];
    if (o == 0.0) return;
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    const Vec3 s = face_position(a, x, y, z, g);
    const Vec3 v0 = sample_velocity(u.x, u.y, u.z, s, g, vb);
    const Vec3 mid{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    const Trace t = trace_rk2(s, u.x, u.y, u.z, mask, g, vb);
    const Sample src = sample_face<true>(component<const float>(u.x, u.y, u.z, a), a, t.position, g, vb);
    scatter_face(component<double>(ua.x, ua.y, ua.z, a), a, t.position, o, g, vb);
    trace_adjoint(s, mid, t, src.gradient, o, u, g, vb, ua);
}

// operators.cu:537-561; density and temperature share one trace when both
// adjoints are requested (sa2/oa2 non-null).
__global__ void advect_scalar_vjp_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ src, XsScalarBoundary sb,
                                         const double* __restrict__ oa, double* __restrict__ sa, const float* __restrict__ src2,
                                         XsScalarBoundary sb2, const double* __restrict__ oa2, double* __restrict__ sa2, XsVector u,
                                         XsVelocityBoundary vb, XsAdjointVector ua) {
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
    if (acc != 0.0) component<double>(ua.x, ua.y, ua.z, a)[local] += acc;
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
    component<double>(ua.x, ua.y, ua.z, a)[local] += acc;
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
                              const XsAdjointVector& fa) {
    for (int a = 0; a < 3; ++a) {
        const uint64_t n = face_count(g, a);
        integrate_vjp_faces_kernel<<<blocks_for(n), kBlock, 0, st>>>(n, component<double>(oa.x, oa.y, oa.z, a),
                                                                     component<double>(ua.x, ua.y, ua.z, a));
        if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    }
    integrate_vjp_cells_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, oa, fa);
    return check_launch();
}

XsStatus launch_advect_velocity_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVelocityBoundary& vb,
                                    const XsAdjointVector& oa, const XsAdjointVector& ua) {
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    advect_velocity_vjp_kernel<<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, mask, u, vb, oa, ua);
    return check_launch();
}

XsStatus launch_advect_scalar_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* src, const XsScalarBoundary& sb,
                                  const double* oa, double* sa, const float* src2, const XsScalarBoundary& sb2, const double* oa2,
                                  double* sa2, const XsVector& u, const XsVelocityBoundary& vb, const XsAdjointVector& ua) {
    advect_scalar_vjp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, src, sb, oa, sa, src2, sb2, oa2, sa2, u, vb, ua);
    return check_launch();
}

XsStatus launch_constrain_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsAdjointVector& oa, const XsVelocityBoundary& b,
                              const XsAdjointVector& ua) {
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    constrain_vjp_kernel<<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, mask, oa, b, ua);
    return check_launch();
}

// projection_vjp (operators.cu:1020-1031): pa, ra are cell scratch; the
// output adjoint passes to velocity_adjoint, lambda_p is solved (PCG kind)
// or reverse-swept (RBGS kind), and the divergence transpose is added.
XsStatus projection_vjp(cudaStream_t st, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                        const XsAdjointVector& oa, const XsScalarBoundary& pb, double* pa, double* ra, const XsAdjointVector& ua,
                        void* workspace, const WarmHistory* history) {
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
            // successive adjoint solves of a reverse pass are close: Galerkin
            // start from the ring of previous adjoint solutions, then (with
            // coarsening) one energy-optimal step along the coarse-grid
            // correction of its residual, as in the forward solve
            const WarmHistory& h = *history;
            if ((s = galerkin_combine(st, g, anchor, mask, pb, h, true, nullptr, 0, nullptr, h.ring_start, pa)) != XS_OK) return s;
            adj.initial_guess = h.ring_start;
            if (coarse) {
                if ((s = jacobi_sweeps(st, g, anchor, mask, pb, nullptr, pa, h.ring_start, h.extra_product, h.start)) != XS_OK) return s;
                if ((s = start_residual(st, g, anchor, mask, pb, nullptr, h.start, h.residual, pa)) != XS_OK) return s;
                if ((s = coarse_correction(st, g, anchor, pb, h, h.residual)) != XS_OK) return s;
                if ((s = line_step(st, g, anchor, mask, pb, h, h.correction, h.start, h.residual, h.start)) != XS_OK) return s;
                adj.initial_guess = h.start;
            }
        }
        s = solve_pressure(st, g, adj, anchor, mask, pb, nullptr, pa, nullptr, ra, workspace, nullptr);
        if (s == XS_OK && coarse) s = record_coarse_iterations(st, *history, workspace, g);
        if (s == XS_OK && ring) s = history_push(st, g, anchor, mask, pb, *history, nullptr, ra);
    }
    if (s != XS_OK) return s;
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    pressure_rhs_reverse_kernel<<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, anchor, mask, ra, oa, ua);
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
