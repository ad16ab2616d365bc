// Step-level composition of the smoke model (solvers/smoke/model.cpp:341-389)
// and the projection entry points (operators.cu:1004-1031), over a
// caller-owned workspace that plays the ExecutionContext scratch
// (model.ixx:17-49).
#include <cstring>

#include "common.cuh"
#include "launch.cuh"
#include "ops.cuh"
#include "unet.cuh"

namespace xs {

// ------------------------------------------------------------ projection
// operators.cu:1004-1013: rhs, pressure solve, gradient subtraction.  With
// the PCG kind the velocity is corrected from the FP64 iterate.
XsStatus projection_forward(cudaStream_t st, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                            const XsVector& u, const XsScalarBoundary& pb, float* pressure, float* rhs, const XsVector& out,
                            void* workspace, cudaEvent_t begin, cudaEvent_t end, WarmStartNet* warm_start, const WarmHistory* history,
                            cudaEvent_t* stages) {
    // stages (optional): the step's events [4..8], here indexed 0..4
    XsStatus s = launch_pressure_rhs(st, g, anchor, mask, u, rhs);
    if (s != XS_OK) return s;
    if ((s = mark_stage(st, stages, 0)) != XS_OK) return s;
    PressureWorkspace w{};
    if (begin && cudaEventRecord(begin, st) != cudaSuccess) return XS_CUDA_ERROR;
    XsPressureSolve used = solve;
    const bool pcg = solve.kind == XS_SOLVER_JACOBI_PCG;
    const bool ring = pcg && history && history->history > 0;
    // warm start (inside the timed solve); PCG falls back to zero whenever the
    // start is worse than zero:
    //  * ring of previous solutions: their Galerkin (A-norm-optimal)
    //    combination x0; then, in turn, the coarse grid's solution for the
    //    residual (coarsening) and the network's correction for the residual
    //    left by that, each as one energy-optimal step on the running
    //    residual.  Sequential steps, not one joint Galerkin combination:
    //    the joint A-norm optimum trades the smooth error these corrections
    //    remove (the error CG is slowest on) for high-frequency error (which
    //    CG removes in a few iterations), and measured 1.3-2x more CG
    //    iterations at 256^3;
    //  * network alone: its guess for b, scaled by the energy-optimal factor.
    float* guess = nullptr;
    const bool coarse = ring && history->coarsening != 0 && mask == nullptr;
    if (ring) {
        const WarmHistory& h = *history;
        if ((s = galerkin_combine(st, g, anchor, mask, pb, h, true, nullptr, 0, rhs, h.ring_start)) != XS_OK) return s;
        used.initial_guess = h.ring_start;
        if (warm_start || coarse) {
            // smooth the start before each coarse-grid step: the coarse grid
            // then sees its smooth error alone
            const float* x = h.ring_start;
            if (coarse) {
                const int cycles = h.forward_rounds ? static_cast<int>(h.forward_rounds)
                                                    : (warm_start ? kForwardStartCyclesLearned : kForwardStartCycles);
                if ((s = coarse_cycles(st, g, anchor, pb, h, rhs, nullptr, cycles, &x, warm_start != nullptr)) != XS_OK) return s;
            } else if ((s = start_residual(st, g, anchor, mask, pb, rhs, x, h.residual)) != XS_OK) {
                return s;
            }
            if (warm_start) {
                float* out = x == h.start ? h.ring_start : h.start;
                if ((s = warm_start_guess(warm_start, st, g, h.residual, &guess)) != XS_OK) return s;
                if ((s = line_step(st, g, anchor, mask, pb, h, guess, x, h.residual, out, false)) != XS_OK) return s;
                x = out;
            }
            used.initial_guess = x;
        }
        used.scale_guess = 0u;
    } else if (warm_start && pcg) {
        if ((s = warm_start_guess(warm_start, st, g, rhs, &guess)) != XS_OK) return s;
        used.initial_guess = guess;
        used.scale_guess = 1u;
    }
    if ((s = mark_stage(st, stages, 1)) != XS_OK) return s;
    s = solve_pressure(st, g, used, anchor, mask, pb, rhs, nullptr, pressure, nullptr, workspace, &w);
    if (s != XS_OK) return s;
    if ((s = mark_stage(st, stages, 2)) != XS_OK) return s;
    if (coarse && (s = record_coarse_iterations(st, *history, workspace, g)) != XS_OK) return s;
    if (ring && (s = history_push(st, g, anchor, mask, pb, *history, pressure)) != XS_OK) return s;
    if (end && cudaEventRecord(end, st) != cudaSuccess) return XS_CUDA_ERROR;
    if ((s = mark_stage(st, stages, 3)) != XS_OK) return s;
    s = solve.kind == XS_SOLVER_RED_BLACK_GAUSS_SEIDEL ? launch_project(st, g, mask, u, pressure, out) : launch_project64(st, g, mask, u, w.x64, out);
    if (s != XS_OK) return s;
    return mark_stage(st, stages, 4);
}

// ------------------------------------------------------------ workspace
struct StepWorkspace {
    // forward (ExecutionContext: raw_advected_velocity_, pressure_, pressure_rhs_)
    float* pressure;
    float* rhs;
    void* solver;
    // tangent scratch (model.ixx:32-43)
    float* sourced_rho_t;
    float* sourced_temp_t;
    XsVector force_t;
    float* vort_t;  // 10 N
    XsVector forced_t;
    XsVector raw_t;
    XsVector advected_t;
    float* pressure_t;
    float* rhs_t;
    // adjoint scratch (model.ixx:44-52)
    double* sourced_rho_a;
    double* sourced_temp_a;
    XsAdjointVector force_a;
    double* vort_a;  // 10 N
    XsAdjointVector projected_a;
    XsAdjointVector advected_a;
    XsAdjointVector raw_a;
    XsAdjointVector forced_a;
    double* pressure_a;
    double* rhs_a;
    WarmHistory history;
    WarmHistory adjoint_history;  // ring of previous adjoint pressure solutions
    size_t bytes;
};

StepWorkspace carve_step(void* base, const Grid& g, uint32_t mode, uint32_t history, uint32_t coarsening) {
    StepWorkspace w{};
    char* p = static_cast<char*>(base);
    size_t off = 0;
    auto take = [&](size_t bytes) -> void* {
        void* r = p ? p + off : nullptr;
        off = (off + bytes + 255) / 256 * 256;
        return r;
    };
    const uint64_t n = cell_count(g), f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    auto fvec = [&]() { XsVector v; v.x = static_cast<float*>(take(4 * f0)); v.y = static_cast<float*>(take(4 * f1)); v.z = static_cast<float*>(take(4 * f2)); return v; };
    auto cvec = [&]() { XsVector v; v.x = static_cast<float*>(take(4 * n)); v.y = static_cast<float*>(take(4 * n)); v.z = static_cast<float*>(take(4 * n)); return v; };
    auto fadj = [&]() { XsAdjointVector v; v.x = static_cast<double*>(take(8 * f0)); v.y = static_cast<double*>(take(8 * f1)); v.z = static_cast<double*>(take(8 * f2)); return v; };
    auto cadj = [&]() { XsAdjointVector v; v.x = static_cast<double*>(take(8 * n)); v.y = static_cast<double*>(take(8 * n)); v.z = static_cast<double*>(take(8 * n)); return v; };
    w.solver = take(pressure_workspace_bytes(g));
    w.pressure = static_cast<float*>(take(4 * n));
    w.rhs = static_cast<float*>(take(4 * n));
    // warm-start ring, in every mode at the same place
    w.history = carve_warm_history(take(warm_history_bytes(g, history, coarsening)), g, history, coarsening);
    if (mode == XS_MODE_DIFFERENTIABLE) {
        w.sourced_rho_t = static_cast<float*>(take(4 * n));
        w.sourced_temp_t = static_cast<float*>(take(4 * n));
        w.force_t = cvec();
        w.vort_t = static_cast<float*>(take(40 * n));
        w.forced_t = fvec();
        w.raw_t = fvec();
        w.advected_t = fvec();
        w.pressure_t = static_cast<float*>(take(4 * n));
        w.rhs_t = static_cast<float*>(take(4 * n));
        w.sourced_rho_a = static_cast<double*>(take(8 * n));
        w.sourced_temp_a = static_cast<double*>(take(8 * n));
        w.force_a = cadj();
        w.vort_a = static_cast<double*>(take(80 * n));
        w.projected_a = fadj();
        w.advected_a = fadj();
        w.raw_a = fadj();
        w.forced_a = fadj();
        w.pressure_a = static_cast<double*>(take(8 * n));
        w.rhs_a = static_cast<double*>(take(8 * n));
        w.adjoint_history = carve_warm_history(take(warm_history_bytes(g, history, coarsening)), g, history, coarsening);
    }
    w.bytes = off;
    return w;
}

bool valid_model(const XsSmokeModel* m) {
    if (m == nullptr || !valid_grid(m->grid) || m->inflow_count > XS_MAX_INFLOWS || (m->inflow_count != 0 && m->inflows == nullptr) ||
        m->warm_start_history > static_cast<uint32_t>(kMaxHistory) || m->warm_start_rounds > kMaxStartRounds)
        return false;
    if (m->warm_start_coarsening != 0) {  // a divisible grid, a ring, no colliders
        Grid c;
        if (!coarse_grid(make_grid(m->grid), m->warm_start_coarsening, c) || m->warm_start_history == 0 || m->cell_mask != nullptr) return false;
    }
    return true;
}

XsStatus zero(cudaStream_t st, void* p, size_t bytes) { return check_cuda(cudaMemsetAsync(p, 0, bytes, st)); }

// ------------------------------------------------------------ metrics
__device__ __forceinline__ void atomic_max_double(double* address, double value) {
    unsigned long long* a = reinterpret_cast<unsigned long long*>(address);
    unsigned long long old = *a;
    while (__longlong_as_double(static_cast<long long>(old)) < value) {
        const unsigned long long assumed = old;
        old = atomicCAS(a, assumed, static_cast<unsigned long long>(__double_as_longlong(value)));
        if (old == assumed) break;
    }
}

// examples/smoke/forward/simulation.cu:59-85: density mass, density and
// temperature maxima, maximum centred speed and the squared divergence
// before and after projection, over fluid cells; one atomic per block.
__global__ void reduce_metrics_kernel(Grid g, const uint32_t* __restrict__ mask, const float* __restrict__ rho, const float* __restrict__ temp,
                                      XsVector pre, XsVector post, double* __restrict__ metrics) {
    __shared__ double red[4 * 32];
    __shared__ double mx[3][32];
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double sums[3] = {0.0, 0.0, 0.0};
    double maxima[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (i < cell_count(g) && !is_solid(mask, i)) {
        int x, y, z;
        decode(i, g.nx, g.ny, x, y, z);
        const uint64_t x0 = idx3(x, y, z, g.nx + 1, g.ny), x1 = idx3(x + 1, y, z, g.nx + 1, g.ny);
        const uint64_t y0 = idx3(x, y, z, g.nx, g.ny + 1), y1 = idx3(x, y + 1, z, g.nx, g.ny + 1);
        const uint64_t z0 = idx3(x, y, z, g.nx, g.ny), z1 = idx3(x, y, z + 1, g.nx, g.ny);
        const double vx = 0.5 * static_cast<double>(post.x[x0] + post.x[x1]);
        const double vy = 0.5 * static_cast<double>(post.y[y0] + post.y[y1]);
        const double vz = 0.5 * static_cast<double>(post.z[z0] + post.z[z1]);
        const double inv = 1.0 / g.h;
        const double dpre = (pre.x[x1] - pre.x[x0] + pre.y[y1] - pre.y[y0] + pre.z[z1] - pre.z[z0]) * inv;
        const double dpost = (post.x[x1] - post.x[x0] + post.y[y1] - post.y[y0] + post.z[z1] - post.z[z0]) * inv;
        sums[0] = rho[i];
        sums[1] = dpre * dpre;
        sums[2] = dpost * dpost;
        maxima[0] = rho[i];
        maxima[1] = temp[i];
        maxima[2] = sqrt(vx * vx + vy * vy + vz * vz);
    }
    block_sum<3>(sums, red);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = maxima[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) mx[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int w = 0; w < (blockDim.x + 31) / 32; ++w)
            for (int k = 0; k < 3; ++k) m[k] = fmax(m[k], mx[k][w]);
        atomicAdd(metrics + 0, sums[0]);
        atomic_max_double(metrics + 1, m[0]);
        atomic_max_double(metrics + 2, m[1]);
        atomic_max_double(metrics + 3, m[2]);
        atomicAdd(metrics + 4, sums[1]);
        atomicAdd(metrics + 5, sums[2]);
    }
}

// The example zeroes its metrics buffer before each reduction
// (simulation.cpp:97-98): sums and maxima start at 0.
__global__ void metrics_init_kernel(double* metrics) {
    if (threadIdx.x < 6) metrics[threadIdx.x] = 0.0;
}

}  // namespace xs

using namespace xs;

extern "C" {

XsStatus xs_projection_forward(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                               const uint32_t* cell_mask, XsVector velocity, XsVelocityBoundary velocity_boundary,
                               XsScalarBoundary pressure_boundary, float* pressure, float* rhs, XsVector output, void* workspace) {
    (void)velocity_boundary;
    if (!valid_grid(grid) || !solve || !valid(velocity) || !pressure || !rhs || !valid(output) || !workspace) return XS_INVALID_ARGUMENT;
    return projection_forward(stream, make_grid(grid), *solve, pressure_anchor, cell_mask, velocity, pressure_boundary, pressure, rhs, output,
                              workspace);
}

// operators.cu:1015-1018: the forward projection of the tangent with zeroed
// pressure boundary values.
XsStatus xs_projection_jvp(cudaStream_t stream, XsGrid grid, const XsPressureSolve* solve, uint32_t pressure_anchor,
                           const uint32_t* cell_mask, XsVector velocity_tangent, XsVelocityBoundary velocity_boundary,
                           XsScalarBoundary pressure_boundary, float* pressure_tangent, float* rhs_tangent, XsVector output_tangent,
                           void* workspace) {
    for (float& v : pressure_boundary.values) v = 0.0f;
    if (!solve) return XS_INVALID_ARGUMENT;
    XsPressureSolve s = *solve;
    s.initial_guess = nullptr;
    return xs_projection_forward(stream, grid, &s, pressure_anchor, cell_mask, velocity_tangent, velocity_boundary, pressure_boundary,
                                 pressure_tangent, rhs_tangent, output_tangent, workspace);
}

size_t xs_smoke_workspace_bytes(const XsSmokeModel* model, uint32_t mode) {
    if (!valid_model(model)) return 0;
    return carve_step(nullptr, make_grid(model->grid), mode, model->warm_start_history, model->warm_start_coarsening).bytes;
}

// model.cpp:341-349
XsStatus xs_smoke_forward_step(cudaStream_t stream, const XsSmokeModel* m, XsState state, XsControl control, XsParameters parameters,
                               XsState next_state, XsStepCache cache, void* workspace) {
    if (!valid_model(m) || !workspace || !state.density || !state.temperature || !valid(state.velocity) || !control.density_source ||
        !control.temperature_source || !valid(control.external_acceleration) || !parameters.ambient_temperature ||
        !parameters.density_buoyancy || !parameters.temperature_buoyancy || !next_state.density || !next_state.temperature ||
        !valid(next_state.velocity) || !cache.sourced_density || !cache.sourced_temperature || !valid(cache.force) ||
        !valid(cache.forced_velocity) || !valid(cache.advected_velocity))
        return XS_INVALID_ARGUMENT;
    if (m->vorticity_confinement_enabled && (!cache.vorticity || !parameters.vorticity_confinement)) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(m->grid);
    const StepWorkspace w = carve_step(workspace, g, XS_MODE_FORWARD, m->warm_start_history, m->warm_start_coarsening);
    const InflowSet inflows = make_inflows(m->inflows, m->inflow_count);
    cudaEvent_t* ev = m->stage_events;
    XsStatus s;
    if ((s = mark_stage(stream, ev, 0)) != XS_OK) return s;
    // sources of density and temperature, then buoyancy on the sourced fields
    s = launch_source_buoyancy(stream, g, m->cell_mask, state.density, state.temperature, control.density_source,
                               control.temperature_source, control.external_acceleration, parameters.ambient_temperature,
                               parameters.density_buoyancy, parameters.temperature_buoyancy, inflows, cache.sourced_density,
                               cache.sourced_temperature, cache.force);
    if (s != XS_OK) return s;
    if (m->vorticity_confinement_enabled) {
        s = vorticity_forward(stream, g, m->cell_mask, state.velocity, parameters.vorticity_confinement, cache.vorticity, cache.force);
        if (s != XS_OK) return s;
    }
    if ((s = mark_stage(stream, ev, 1)) != XS_OK) return s;
    // velocity evolution: integrate, advect (through the forced velocity), constrain
    s = launch_integrate(stream, g, m->cell_mask, state.velocity, cache.force, cache.forced_velocity);
    if (s != XS_OK) return s;
    if ((s = mark_stage(stream, ev, 2)) != XS_OK) return s;
    s = launch_advect_constrain(stream, g, m->cell_mask, m->collider_velocity, cache.forced_velocity, m->velocity_boundary,
                                cache.advected_velocity);
    if (s != XS_OK) return s;
    if ((s = mark_stage(stream, ev, 3)) != XS_OK) return s;
    // projection
    WarmHistory history = w.history;
    history.forward_rounds = m->warm_start_rounds;
    s = projection_forward(stream, g, m->pressure, m->pressure_anchor, m->cell_mask, cache.advected_velocity, m->pressure_boundary,
                           w.pressure, w.rhs, next_state.velocity, w.solver, m->solve_begin, m->solve_end,
                           reinterpret_cast<WarmStartNet*>(m->warm_start), &history, ev ? ev + 4 : nullptr);
    if (s != XS_OK) return s;
    // scalar advection of the sourced fields through the projected velocity
    s = launch_advect_scalar_pair(stream, g, m->cell_mask, m->collider_density, m->collider_temperature, cache.sourced_density,
                                  cache.sourced_temperature, next_state.velocity, m->density_boundary, m->temperature_boundary,
                                  m->velocity_boundary, next_state.density, next_state.temperature);
    if (s != XS_OK) return s;
    return mark_stage(stream, ev, 9);
}

// model.cpp:351-359
XsStatus xs_smoke_jvp_step(cudaStream_t stream, const XsSmokeModel* m, XsState state, XsParameters parameters, XsState next_state,
                           XsStepCache cache, XsState st, XsControl ct, XsParameters pt, XsState nt, void* workspace) {
    (void)state;
    if (!valid_model(m) || !workspace || !st.density || !st.temperature || !valid(st.velocity) || !ct.density_source ||
        !ct.temperature_source || !valid(ct.external_acceleration) || !pt.ambient_temperature || !pt.density_buoyancy ||
        !pt.temperature_buoyancy || !nt.density || !nt.temperature || !valid(nt.velocity) || !valid(next_state.velocity))
        return XS_INVALID_ARGUMENT;
    if (m->vorticity_confinement_enabled && (!cache.vorticity || !parameters.vorticity_confinement || !pt.vorticity_confinement))
        return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(m->grid);
    const StepWorkspace w = carve_step(workspace, g, XS_MODE_DIFFERENTIABLE, m->warm_start_history, m->warm_start_coarsening);
    const InflowSet inflows = make_inflows(m->inflows, m->inflow_count);
    XsStatus s;
    s = launch_source_jvp_pair(stream, g, m->cell_mask, st.density, st.temperature, ct.density_source, ct.temperature_source, inflows,
                               w.sourced_rho_t, w.sourced_temp_t);
    if (s != XS_OK) return s;
    s = launch_buoyancy_jvp(stream, g, m->cell_mask, cache.sourced_density, cache.sourced_temperature, w.sourced_rho_t, w.sourced_temp_t,
                            ct.external_acceleration, parameters.ambient_temperature, parameters.density_buoyancy,
                            parameters.temperature_buoyancy, pt.ambient_temperature, pt.density_buoyancy, pt.temperature_buoyancy,
                            w.force_t);
    if (s != XS_OK) return s;
    if (m->vorticity_confinement_enabled) {
        s = vorticity_jvp(stream, g, m->cell_mask, st.velocity, parameters.vorticity_confinement, pt.vorticity_confinement, cache.vorticity,
                          w.force_t, w.vort_t);
        if (s != XS_OK) return s;
    }
    s = launch_integrate(stream, g, m->cell_mask, st.velocity, w.force_t, w.forced_t);
    if (s != XS_OK) return s;
    s = launch_advect_velocity_jvp(stream, g, m->cell_mask, cache.forced_velocity, w.forced_t, m->velocity_boundary, w.raw_t);
    if (s != XS_OK) return s;
    XsVelocityBoundary tvb = m->velocity_boundary;
    for (float& v : tvb.values) v = 0.0f;
    s = launch_constrain(stream, g, m->cell_mask, XsVector{nullptr, nullptr, nullptr}, w.raw_t, tvb, w.advected_t);
    if (s != XS_OK) return s;
    XsScalarBoundary tpb = m->pressure_boundary;
    for (float& v : tpb.values) v = 0.0f;
    XsPressureSolve solve = m->pressure;
    solve.initial_guess = nullptr;
    s = projection_forward(stream, g, solve, m->pressure_anchor, m->cell_mask, w.advected_t, tpb, w.pressure_t, w.rhs_t, nt.velocity,
                           w.solver);
    if (s != XS_OK) return s;
    return launch_advect_scalar_jvp(stream, g, m->cell_mask, cache.sourced_density, w.sourced_rho_t, m->density_boundary, nt.density,
                                    cache.sourced_temperature, w.sourced_temp_t, m->temperature_boundary, nt.temperature,
                                    next_state.velocity, nt.velocity, m->velocity_boundary);
}

// model.cpp:361-389
XsStatus xs_smoke_vjp_step(cudaStream_t stream, const XsSmokeModel* m, XsState state, XsParameters parameters, XsState next_state,
                           XsStepCache cache, XsStateAdjoint na, XsStateAdjoint pa, XsControlAdjoint ca, XsParameterAdjoint qa,
                           void* workspace) {
    (void)state;
    if (!valid_model(m) || !workspace || !na.density || !na.temperature || !valid(na.velocity) || !pa.density || !pa.temperature ||
        !valid(pa.velocity) || !ca.density_source || !ca.temperature_source || !valid(ca.external_acceleration) ||
        !qa.ambient_temperature || !qa.density_buoyancy || !qa.temperature_buoyancy || !valid(next_state.velocity))
        return XS_INVALID_ARGUMENT;
    if (m->vorticity_confinement_enabled && (!cache.vorticity || !parameters.vorticity_confinement || !qa.vorticity_confinement))
        return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(m->grid);
    const StepWorkspace w = carve_step(workspace, g, XS_MODE_DIFFERENTIABLE, m->warm_start_history, m->warm_start_coarsening);
    const InflowSet inflows = make_inflows(m->inflows, m->inflow_count);
    const uint64_t n = cell_count(g), f0 = face_count(g, 0), f1 = face_count(g, 1), f2 = face_count(g, 2);
    XsStatus s;
    // scratch adjoints start at zero (model.cpp:362-378): those accumulated
    // by scatters are cleared; the advected, raw and force adjoints are
    // written whole by the first operator that produces them instead
    if ((s = zero(stream, w.sourced_rho_a, 8 * n)) != XS_OK) return s;
    if ((s = zero(stream, w.sourced_temp_a, 8 * n)) != XS_OK) return s;
    const size_t fb[3] = {8 * f0, 8 * f1, 8 * f2};
    if ((s = zero(stream, w.forced_a.x, fb[0])) != XS_OK) return s;
    if ((s = zero(stream, w.forced_a.y, fb[1])) != XS_OK) return s;
    if ((s = zero(stream, w.forced_a.z, fb[2])) != XS_OK) return s;
    // lambda of the projected velocity starts as the incoming adjoint (model.cpp:379-381)
    if ((s = check_cuda(cudaMemcpyAsync(w.projected_a.x, na.velocity.x, fb[0], cudaMemcpyDeviceToDevice, stream))) != XS_OK) return s;
    if ((s = check_cuda(cudaMemcpyAsync(w.projected_a.y, na.velocity.y, fb[1], cudaMemcpyDeviceToDevice, stream))) != XS_OK) return s;
    if ((s = check_cuda(cudaMemcpyAsync(w.projected_a.z, na.velocity.z, fb[2], cudaMemcpyDeviceToDevice, stream))) != XS_OK) return s;
    // scalar advection of density and temperature, one shared trace
    s = launch_advect_scalar_vjp(stream, g, m->cell_mask, cache.sourced_density, m->density_boundary, na.density, w.sourced_rho_a,
                                 cache.sourced_temperature, m->temperature_boundary, na.temperature, w.sourced_temp_a, next_state.velocity,
                                 m->velocity_boundary, w.projected_a);
    if (s != XS_OK) return s;
    // projection
    s = projection_vjp(stream, g, m->pressure, m->pressure_anchor, m->cell_mask, w.projected_a, m->pressure_boundary, w.pressure_a, w.rhs_a,
                       w.advected_a, w.solver, &w.adjoint_history, true);
    if (s != XS_OK) return s;
    // velocity evolution: constrain, advect, integrate (operators.cpp:152-156)
    s = launch_constrain_vjp(stream, g, m->cell_mask, w.advected_a, m->velocity_boundary, w.raw_a, true);
    if (s != XS_OK) return s;
    s = launch_advect_velocity_vjp(stream, g, m->cell_mask, cache.forced_velocity, m->velocity_boundary, w.raw_a, w.forced_a);
    if (s != XS_OK) return s;
    s = launch_integrate_vjp(stream, g, m->cell_mask, w.forced_a, pa.velocity, w.force_a, true);
    if (s != XS_OK) return s;
    // forces: buoyancy then vorticity (operators.cpp:135-138)
    s = launch_buoyancy_vjp(stream, g, m->cell_mask, cache.sourced_density, cache.sourced_temperature, parameters.ambient_temperature,
                            parameters.density_buoyancy, parameters.temperature_buoyancy, w.force_a, w.sourced_rho_a, w.sourced_temp_a,
                            ca.external_acceleration, qa.ambient_temperature, qa.density_buoyancy, qa.temperature_buoyancy);
    if (s != XS_OK) return s;
    if (m->vorticity_confinement_enabled) {
        s = vorticity_vjp(stream, g, m->cell_mask, parameters.vorticity_confinement, cache.vorticity, w.force_a, pa.velocity,
                          qa.vorticity_confinement, w.vort_a);
        if (s != XS_OK) return s;
    }
    // sources
    s = launch_source_vjp(stream, g, m->cell_mask, w.sourced_rho_a, inflows, pa.density, ca.density_source);
    if (s != XS_OK) return s;
    return launch_source_vjp(stream, g, m->cell_mask, w.sourced_temp_a, inflows, pa.temperature, ca.temperature_source);
}

XsStatus xs_smoke_reduce_metrics(cudaStream_t stream, const XsSmokeModel* m, const float* density, const float* temperature,
                                 XsVector pre_projection_velocity, XsVector post_projection_velocity, double* metrics) {
    if (!valid_model(m) || !density || !temperature || !valid(pre_projection_velocity) || !valid(post_projection_velocity) || !metrics)
        return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(m->grid);
    metrics_init_kernel<<<1, 32, 0, stream>>>(metrics);
    if (check_launch() != XS_OK) return XS_CUDA_ERROR;
    reduce_metrics_kernel<<<blocks_for(cell_count(g)), kBlock, 0, stream>>>(g, m->cell_mask, density, temperature, pre_projection_velocity,
                                                                             post_projection_velocity, metrics);
    return check_launch();
}

XsStatus xs_smoke_read_solve_stats(cudaStream_t stream, const XsSmokeModel* model, const void* workspace, uint32_t mode,
                                   XsSolveStats* forward_stats, XsSolveStats* adjoint_stats) {
    (void)mode;
    if (!valid_model(model) || !workspace) return XS_INVALID_ARGUMENT;
    const StepWorkspace w =
        carve_step(const_cast<void*>(workspace), make_grid(model->grid), XS_MODE_FORWARD, model->warm_start_history, model->warm_start_coarsening);
    XsSolveStats st{};
    const XsStatus s = xs_read_solve_stats(stream, w.solver, &st);
    if (forward_stats) *forward_stats = st;
    if (adjoint_stats) *adjoint_stats = st;
    return s;
}

XsStatus xs_smoke_warm_start_fields(cudaStream_t stream, const XsSmokeModel* model, void* workspace, float** ring_start, float** residual) {
    if (!valid_model(model) || !workspace || model->warm_start_history == 0) return XS_INVALID_ARGUMENT;
    const Grid g = make_grid(model->grid);
    const StepWorkspace w = carve_step(workspace, g, XS_MODE_FORWARD, model->warm_start_history, model->warm_start_coarsening);
    const XsStatus s = start_residual(stream, g, model->pressure_anchor, model->cell_mask, model->pressure_boundary, w.rhs, w.history.ring_start,
                                      w.history.residual);
    if (s != XS_OK) return s;
    if (ring_start) *ring_start = w.history.ring_start;
    if (residual) *residual = w.history.residual;
    return XS_OK;
}

XsStatus xs_smoke_reset_warm_start(cudaStream_t stream, const XsSmokeModel* model, void* workspace, uint32_t mode) {
    if (!valid_model(model) || !workspace || mode > XS_MODE_DIFFERENTIABLE) return XS_INVALID_ARGUMENT;
    const StepWorkspace w = carve_step(workspace, make_grid(model->grid), mode, model->warm_start_history, model->warm_start_coarsening);
    const XsStatus s = history_reset(stream, w.history);
    if (s != XS_OK || mode != XS_MODE_DIFFERENTIABLE) return s;
    return history_reset(stream, w.adjoint_history);
}

XsStatus xs_smoke_pressure_fields(const XsSmokeModel* model, void* workspace, float** pressure, float** rhs) {
    if (!valid_model(model) || !workspace) return XS_INVALID_ARGUMENT;
    const StepWorkspace w = carve_step(workspace, make_grid(model->grid), XS_MODE_FORWARD, model->warm_start_history, model->warm_start_coarsening);
    if (pressure) *pressure = w.pressure;
    if (rhs) *rhs = w.rhs;
    return XS_OK;
}

}  // extern "C"
