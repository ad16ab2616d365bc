// Tangent (JVP) smoke operators on sm_100a
// (solvers/smoke/operators.cu:315-324, 390-413, 509-535, 575-577, 604-606,
// 633-638, 1015-1018).
#include "common.cuh"
#include "launch.cuh"
#include "ops.cuh"

namespace xs {

// operators.cu:575-577 (source_jvp is source_forward on tangents) for both
// scalars; inflow cells are set, so their tangent is zero.
__global__ void source_jvp_pair_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ rt, const float* __restrict__ tt,
                                       const float* __restrict__ rst, const float* __restrict__ tst, InflowSet inflows,
                                       float* __restrict__ ro, float* __restrict__ to) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    bool zero = is_solid(mask, i);
    if (!zero && inflows.count) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        zero = inflow_hit(inflows, x, y, z, g) >= 0;
    }
    if (zero) { ro[i] = 0.0f; to[i] = 0.0f; return; }
    ro[i] = rt[i] + g.dt * rst[i];
    to[i] = tt[i] + g.dt * tst[i];
}

__global__ void source_jvp_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ st, const float* __restrict__ sr,
                                  InflowSet inflows, float* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    bool zero = is_solid(mask, i);
    if (!zero && inflows.count) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        zero = inflow_hit(inflows, x, y, z, g) >= 0;
    }
    out[i] = zero ? 0.0f : st[i] + g.dt * sr[i];
}

// operators.cu:315-324
__global__ void buoyancy_jvp_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ rho, const float* __restrict__ temp,
                                    const float* __restrict__ rho_t, const float* __restrict__ temp_t, XsVector acc_t,
                                    const float* __restrict__ amb, const float* __restrict__ br, const float* __restrict__ bt,
                                    const float* __restrict__ amb_t, const float* __restrict__ br_t, const float* __restrict__ bt_t,
                                    XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) { out.x[i] = 0.0f; out.y[i] = 0.0f; out.z[i] = 0.0f; return; }
    out.x[i] = acc_t.x[i];
    out.y[i] = acc_t.y[i] + __ldg(br) * rho_t[i] + __ldg(br_t) * rho[i] + __ldg(bt) * (temp_t[i] - __ldg(amb_t)) +
               __ldg(bt_t) * (temp[i] - __ldg(amb));
    out.z[i] = acc_t.z[i];
}

// Tangent of the RK2 trace: returns the tangent of the final position
// (operators.cu:398-410 / 520-532).
__device__ __forceinline__ Vec3 trace_tangent(const Vec3& s, const XsVector& u, const XsVector& ut, const Trace& t, const Grid& g,
                                              const XsVelocityBoundary& vb, const XsVelocityBoundary& tvb) {
    const Vec3 v0 = sample_velocity(u.x, u.y, u.z, s, g, vb);
    const Vec3 t0 = sample_velocity(ut.x, ut.y, ut.z, s, g, tvb);
    const Vec3 mid{s.x - 0.5f * g.dt * v0.x, s.y - 0.5f * g.dt * v0.y, s.z - 0.5f * g.dt * v0.z};
    const Vec3 midt{-0.5f * g.dt * t0.x, -0.5f * g.dt * t0.y, -0.5f * g.dt * t0.z};
    const Sample a = sample_face<true>(u.x, 0, mid, g, vb);
    const Sample b = sample_face<true>(u.y, 1, mid, g, vb);
    const Sample c = sample_face<true>(u.z, 2, mid, g, vb);
    const Vec3 st = sample_velocity(ut.x, ut.y, ut.z, mid, g, tvb);
    const Vec3 v1t{st.x + a.gradient.x * midt.x + a.gradient.y * midt.y + a.gradient.z * midt.z,
                   st.y + b.gradient.x * midt.x + b.gradient.y * midt.y + b.gradient.z * midt.z,
                   st.z + c.gradient.x * midt.x + c.gradient.y * midt.y + c.gradient.z * midt.z};
    return Vec3{-t.derivative.x * g.dt * v1t.x, -t.derivative.y * g.dt * v1t.y, -t.derivative.z * g.dt * v1t.z};
}

// operators.cu:390-413 for all three components in one launch.
__global__ void advect_velocity_jvp_kernel(const __grid_constant__ Grid g, uint64_t f0, uint64_t f1, uint64_t f2, const uint32_t* __restrict__ mask, XsVector u,
                                           XsVector ut, const __grid_constant__ XsVelocityBoundary vb, XsVector out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= f0 + f1 + f2) return;
    int a;
    uint64_t local;
    if (i < f0) { a = 0; local = i; } else if (i < f0 + f1) { a = 1; local = i - f0; } else { a = 2; local = i - f0 - f1; }
    int x, y, z;
    decode(local, extent(g, a, 0), extent(g, a, 1), x, y, z);
    const XsVelocityBoundary tvb = zero_values(vb);
    const Vec3 s = face_position(a, x, y, z, g);
    const Trace t = trace_rk2(s, u.x, u.y, u.z, mask, g, vb);
    const Vec3 pt = trace_tangent(s, u, ut, t, g, vb, tvb);
    const Sample src = sample_face<true>(component<const float>(u.x, u.y, u.z, a), a, t.position, g, vb);
    component<float>(out.x, out.y, out.z, a)[local] =
        sample_face<false>(component<const float>(ut.x, ut.y, ut.z, a), a, t.position, g, tvb).value + src.gradient.x * pt.x +
        src.gradient.y * pt.y + src.gradient.z * pt.z;
}

// operators.cu:509-535; the second scalar (src2 non-null) shares the trace.
__global__ void advect_scalar_jvp_kernel(const __grid_constant__ Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ src,
                                         const float* __restrict__ src_t, const __grid_constant__ XsScalarBoundary sb, float* __restrict__ out,
                                         const float* __restrict__ src2, const float* __restrict__ src2_t, const __grid_constant__ XsScalarBoundary sb2,
                                         float* __restrict__ out2, XsVector u, XsVector ut, const __grid_constant__ XsVelocityBoundary vb) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cell_count(g)) return;
    if (is_solid(mask, i)) {
        out[i] = 0.0f;
        if (out2) out2[i] = 0.0f;
        return;
    }
    int x, y, z;
    decode(i, g.nx, g.ny, x, y, z);
    const XsVelocityBoundary tvb = zero_values(vb);
    const Vec3 s = cell_position(x, y, z, g);
    const Trace t = trace_rk2(s, u.x, u.y, u.z, mask, g, vb);
    const Vec3 pt = trace_tangent(s, u, ut, t, g, vb, tvb);
    const Sample a = sample_scalar<true>(src, t.position, g, sb);
    out[i] = sample_scalar<false>(src_t, t.position, g, zero_values(sb)).value + a.gradient.x * pt.x + a.gradient.y * pt.y + a.gradient.z * pt.z;
    if (out2) {
        const Sample b = sample_scalar<true>(src2, t.position, g, sb2);
        out2[i] = sample_scalar<false>(src2_t, t.position, g, zero_values(sb2)).value + b.gradient.x * pt.x + b.gradient.y * pt.y +
                  b.gradient.z * pt.z;
    }
}

// ------------------------------------------------------------ launchers
XsStatus launch_source_jvp_pair(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho_t, const float* temp_t,
                                const float* rho_src_t, const float* temp_src_t, const InflowSet& inflows, float* rho_out,
                                float* temp_out) {
    source_jvp_pair_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, rho_t, temp_t, rho_src_t, temp_src_t, inflows, rho_out,
                                                                          temp_out);
    return check_launch();
}

XsStatus launch_buoyancy_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho, const float* temp, const float* rho_t,
                             const float* temp_t, const XsVector& acc_t, const float* ambient, const float* beta_rho,
                             const float* beta_temp, const float* ambient_t, const float* beta_rho_t, const float* beta_temp_t,
                             const XsVector& force_t) {
    buoyancy_jvp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, rho, temp, rho_t, temp_t, acc_t, ambient, beta_rho, beta_temp,
                                                                       ambient_t, beta_rho_t, beta_temp_t, force_t);
    return check_launch();
}

XsStatus launch_advect_velocity_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVector& ut,
                                    const XsVelocityBoundary& vb, const XsVector& out) {
    const uint64_t f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    advect_velocity_jvp_kernel<<<blocks_for(f0 + f1 + f2), kBlock, 0, st>>>(g, f0, f1, f2, mask, u, ut, vb, out);
    return check_launch();
}

XsStatus launch_advect_scalar_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* src, const float* src_t,
                                  const XsScalarBoundary& sb, float* out, const float* src2, const float* src2_t,
                                  const XsScalarBoundary& sb2, float* out2, const XsVector& u, const XsVector& ut,
                                  const XsVelocityBoundary& vb) {
    advect_scalar_jvp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, st>>>(g, mask, src, src_t, sb, out, src2, src2_t, sb2, out2, u, ut, vb);
    return check_launch();
}

}  // namespace xs

using namespace xs;

extern "C" {

XsStatus xs_source_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* state_tangent, const float* source_tangent,
                       const XsInflow* inflows, uint32_t inflow_count, float* output_tangent) {
    if (!valid_grid(grid) || !state_tangent || !source_tangent || !output_tangent || inflow_count > XS_MAX_INFLOWS) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(grid);
    source_jvp_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(g, cell_mask, state_tangent, source_tangent,
                                                                         make_inflows(inflows, inflow_count), output_tangent);
    return check_launch();
}

XsStatus xs_buoyancy_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* density, const float* temperature,
                         const float* density_tangent, const float* temperature_tangent, XsVector external_acceleration_tangent,
                         const float* ambient_temperature, const float* density_buoyancy, const float* temperature_buoyancy,
                         const float* ambient_temperature_tangent, const float* density_buoyancy_tangent,
                         const float* temperature_buoyancy_tangent, XsVector force_tangent) {
    if (!valid_grid(grid) || !density || !temperature || !density_tangent || !temperature_tangent || !valid(external_acceleration_tangent) ||
        !ambient_temperature || !density_buoyancy || !temperature_buoyancy || !ambient_temperature_tangent || !density_buoyancy_tangent ||
        !temperature_buoyancy_tangent || !valid(force_tangent))
        return XS_INVALID_ARGUMENT;
    return launch_buoyancy_jvp(stream, make_grid(grid), cell_mask, density, temperature, density_tangent, temperature_tangent,
                               external_acceleration_tangent, ambient_temperature, density_buoyancy, temperature_buoyancy,
                               ambient_temperature_tangent, density_buoyancy_tangent, temperature_buoyancy_tangent, force_tangent);
}

XsStatus xs_integrate_velocity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity_tangent,
                                   XsVector force_tangent, XsVector output_tangent) {
    return xs_integrate_velocity_forward(stream, grid, cell_mask, velocity_tangent, force_tangent, output_tangent);
}

XsStatus xs_advect_velocity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity, XsVector velocity_tangent,
                                XsVelocityBoundary boundary, XsVector output_tangent) {
    if (!valid_grid(grid) || !valid(velocity) || !valid(velocity_tangent) || !valid(output_tangent)) return XS_INVALID_ARGUMENT;
    return launch_advect_velocity_jvp(stream, make_grid(grid), cell_mask, velocity, velocity_tangent, boundary, output_tangent);
}

// operators.cu:633-638: the forward constraint with zero collider velocity
// and zeroed boundary values.
XsStatus xs_constrain_velocity_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, XsVector velocity_tangent,
                                   XsVelocityBoundary boundary, XsVector output_tangent) {
    for (float& v : boundary.values) v = 0.0f;
    return xs_constrain_velocity_forward(stream, grid, cell_mask, XsVector{nullptr, nullptr, nullptr}, velocity_tangent, boundary,
                                         output_tangent);
}

XsStatus xs_advect_scalar_jvp(cudaStream_t stream, XsGrid grid, const uint32_t* cell_mask, const float* source, const float* source_tangent,
                              XsVector velocity, XsVector velocity_tangent, XsScalarBoundary scalar_boundary,
                              XsVelocityBoundary velocity_boundary, float* output_tangent) {
    if (!valid_grid(grid) || !source || !source_tangent || !valid(velocity) || !valid(velocity_tangent) || !output_tangent)
        return XS_INVALID_ARGUMENT;
    return launch_advect_scalar_jvp(stream, make_grid(grid), cell_mask, source, source_tangent, scalar_boundary, output_tangent, nullptr,
                                    nullptr, scalar_boundary, nullptr, velocity, velocity_tangent, velocity_boundary);
}

}  // extern "C"
