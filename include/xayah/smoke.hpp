// xayah::smoke -- the smoke solver's data layout and model for C++ callers.
//
// Header-only counterpart of the reference modules xayah.smoke.data
// (solvers/smoke/data.ixx:8-204) and xayah.smoke.model (model.ixx:10-96),
// with the same type and member names, enum values and call signatures.
// Every step runs on the B200 kernels of libdiffsmoke.so through the C ABI
// in diff_smoke.h.  Additions (no reference counterpart): inflow spheres,
// the pressure-solver choice with tolerance, and warm starts.
#pragma once

#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>

#include "diff_smoke.h"
#include "xayah/cuda.hpp"

namespace xayah::smoke {

inline void check(XsStatus status, const char* what) {
    if (status != XS_OK) {
        std::string msg = std::string{what} + ": " + xs_status_string(status);
        if (status == XS_CUDA_ERROR) msg += std::string{" ("} + cudaGetErrorString(static_cast<cudaError_t>(xs_last_cuda_error())) + ")";
        throw std::runtime_error(msg);
    }
}

// ------------------------------------------------------------- data.ixx:8-83
struct Vector3 {
    float x;
    float y;
    float z;
};

enum class ScalarBoundaryMode : std::uint32_t { fixed_value, zero_gradient, periodic };
enum class VelocityBoundaryMode : std::uint32_t { fixed_value, zero_gradient, normal_fixed_tangent_zero_gradient, periodic };

struct ScalarBoundaryFace {
    ScalarBoundaryMode mode{ScalarBoundaryMode::zero_gradient};
    float value{};
};
struct VelocityBoundaryFace {
    VelocityBoundaryMode mode{VelocityBoundaryMode::zero_gradient};
    Vector3 value{};
};
struct ScalarBoundary {
    ScalarBoundaryFace x_min{}, x_max{}, y_min{}, y_max{}, z_min{}, z_max{};
};
struct VelocityBoundary {
    VelocityBoundaryFace x_min{}, x_max{}, y_min{}, y_max{}, z_min{}, z_max{};
};
struct Ellipsoid {
    Vector3 center{};
    Vector3 radius{1.0F, 1.0F, 1.0F};
};
struct Box {
    Vector3 center{};
    Vector3 half_extent{1.0F, 1.0F, 1.0F};
};
struct Collider {
    std::variant<Ellipsoid, Box> shape{Ellipsoid{}};
    Vector3 velocity{};
    float density{};
    float temperature{};
};
struct Inflow {
    Vector3 center{};
    float radius{};
    float density{1.0F};
    float temperature{1.0F};
};
enum class PressureSolver : std::uint32_t { jacobi_pcg = XS_SOLVER_JACOBI_PCG, red_black_gauss_seidel = XS_SOLVER_RED_BLACK_GAUSS_SEIDEL };

struct Configuration {
    std::array<std::uint32_t, 3u> resolution{32u, 48u, 32u};
    float cell_size{1.0F / 32.0F};
    float time_step{1.0F / 60.0F};
    std::uint32_t pressure_iterations{80u};
    VelocityBoundary velocity_boundary{};
    ScalarBoundary pressure_boundary{};
    ScalarBoundary density_boundary{};
    ScalarBoundary temperature_boundary{};
    std::vector<Collider> colliders{};
    bool vorticity_confinement_enabled{true};
    // additions
    std::vector<Inflow> inflows{};
    PressureSolver pressure_solver{PressureSolver::jacobi_pcg};
    double pressure_tolerance{1.0e-6};
    std::uint32_t pressure_max_iterations{4000u};
    // previous forward solutions kept for the Galerkin warm start (0..5; 0: off)
    std::uint32_t warm_start_history{0u};
    // coarse-grid correction of that start (0: off; else the coarsening factor
    // per axis, dividing the grid; needs a ring and no colliders)
    std::uint32_t warm_start_coarsening{0u};
    // rounds of sweeps and coarse-grid correction before a forward solve (0: defaults)
    std::uint32_t warm_start_rounds{0u};
};

// ------------------------------------------------------------- data.ixx:85-204
struct ScalarField {
    cuda::Buffer<float> values;
};
struct CenteredVectorField {
    ScalarField x, y, z;
};
struct StaggeredVectorField {
    cuda::Buffer<float> x, y, z;
};
struct ScalarAdjointField {
    cuda::Buffer<double> values;
};
struct CenteredVectorAdjointField {
    ScalarAdjointField x, y, z;
};
struct StaggeredVectorAdjointField {
    cuda::Buffer<double> x, y, z;
};
struct State {
    ScalarField density;
    ScalarField temperature;
    StaggeredVectorField velocity;
};
struct Control {
    ScalarField density_source;
    ScalarField temperature_source;
    CenteredVectorField external_acceleration;
};
struct Parameters {
    cuda::Buffer<float> ambient_temperature, density_buoyancy, temperature_buoyancy, vorticity_confinement;
};
using StateTangent = State;
using ControlTangent = Control;
using ParameterTangent = Parameters;
struct StateAdjoint {
    ScalarAdjointField density;
    ScalarAdjointField temperature;
    StaggeredVectorAdjointField velocity;
};
struct ControlAdjoint {
    ScalarAdjointField density_source;
    ScalarAdjointField temperature_source;
    CenteredVectorAdjointField external_acceleration;
};
struct ParameterAdjoint {
    cuda::Buffer<double> ambient_temperature, density_buoyancy, temperature_buoyancy, vorticity_confinement;
};
// data.ixx:174-180, held as one block of 11 cell arrays: centred velocity
// (3), vorticity (3), magnitude, normal (3), normalizer.
struct VorticityCache {
    cuda::Buffer<float> storage;
    std::size_t cell_count{};
    [[nodiscard]] float* array(int i) const { return storage.data + static_cast<std::size_t>(i) * cell_count; }
};
struct StepCache {
    ScalarField sourced_density;
    ScalarField sourced_temperature;
    CenteredVectorField force;
    VorticityCache vorticity;
    StaggeredVectorField forced_velocity;
    StaggeredVectorField advected_velocity;
};
struct DeviceDomain {
    cuda::Buffer<std::uint32_t> cell_mask;
    StaggeredVectorField collider_velocity;
    ScalarField collider_density;
    ScalarField collider_temperature;
    std::uint32_t pressure_anchor{};
};

// ------------------------------------------------------------- model.ixx
enum class ExecutionMode : std::uint32_t { forward = XS_MODE_FORWARD, differentiable = XS_MODE_DIFFERENTIABLE };

struct Model;

struct ExecutionContext {
public:
    std::shared_ptr<cuda::Resource> resource;
    DeviceDomain domain;

    // Statistics of the last pressure solve run in this context (synchronises).
    [[nodiscard]] XsSolveStats solve_stats() const {
        XsSolveStats s{};
        check(xs_smoke_read_solve_stats(resource->stream(), &native_, workspace_.data, static_cast<std::uint32_t>(mode_), &s, nullptr),
              "xs_smoke_read_solve_stats");
        return s;
    }
    // Warm start (N device floats) for the following PCG solves; nullptr: zero.
    void set_warm_start(const float* guess) { native_.pressure.initial_guess = guess; }
    // Learned warm start of the forward pressure solves (a network whose grid
    // times its factor is this model's grid); nullptr: none.  The guess is
    // energy-scaled and PCG falls back to zero when it does not help.
    void set_learned_warm_start(XsWarmStartNet* net) { native_.warm_start = net; }
    // The model block the C ABI's step-level entry points take.
    [[nodiscard]] const XsSmokeModel& native() const { return native_; }

private:
    ExecutionMode mode_{ExecutionMode::forward};
    XsSmokeModel native_{};
    std::vector<XsInflow> inflows_;
    cuda::Buffer<unsigned char> workspace_;

    friend struct Model;
};

struct Model {
public:
    const Configuration configuration;

    explicit Model(Configuration c) : configuration(std::move(c)) {
        if (configuration.inflows.size() > XS_MAX_INFLOWS) throw std::invalid_argument("too many inflows");
    }

    [[nodiscard]] ExecutionContext allocate_context(ExecutionMode mode) const {
        ExecutionContext ctx{};
        ctx.resource = std::make_shared<cuda::Resource>();
        ctx.mode_ = mode;
        const std::size_t n = cell_count();
        ctx.domain.cell_mask = cuda::Buffer<std::uint32_t>(ctx.resource, n);
        ctx.domain.collider_velocity = staggered(ctx);
        ctx.domain.collider_density = scalar(ctx);
        ctx.domain.collider_temperature = scalar(ctx);
        std::vector<XsCollider> cols;
        for (const Collider& k : configuration.colliders) {
            XsCollider c{};
            if (const auto* e = std::get_if<Ellipsoid>(&k.shape)) {
                c.shape = 0u;
                c.center[0] = e->center.x; c.center[1] = e->center.y; c.center[2] = e->center.z;
                c.size[0] = e->radius.x; c.size[1] = e->radius.y; c.size[2] = e->radius.z;
            } else {
                const Box& b = std::get<Box>(k.shape);
                c.shape = 1u;
                c.center[0] = b.center.x; c.center[1] = b.center.y; c.center[2] = b.center.z;
                c.size[0] = b.half_extent.x; c.size[1] = b.half_extent.y; c.size[2] = b.half_extent.z;
            }
            c.velocity[0] = k.velocity.x; c.velocity[1] = k.velocity.y; c.velocity[2] = k.velocity.z;
            c.density = k.density;
            c.temperature = k.temperature;
            cols.push_back(c);
        }
        XsSmokeModel& m = ctx.native_;
        m.grid = grid();
        m.velocity_boundary = pack(configuration.velocity_boundary);
        m.pressure_boundary = pack(configuration.pressure_boundary);
        m.density_boundary = pack(configuration.density_boundary);
        m.temperature_boundary = pack(configuration.temperature_boundary);
        check(xs_smoke_build_domain(ctx.resource->stream(), m.grid, m.pressure_boundary, cols.data(), static_cast<std::uint32_t>(cols.size()),
                                    ctx.domain.cell_mask.data, view(ctx.domain.collider_velocity), ctx.domain.collider_density.values.data,
                                    ctx.domain.collider_temperature.values.data, &ctx.domain.pressure_anchor),
              "xs_smoke_build_domain");
        const bool colliders = !configuration.colliders.empty();
        m.vorticity_confinement_enabled = configuration.vorticity_confinement_enabled ? 1u : 0u;
        m.pressure_anchor = ctx.domain.pressure_anchor;
        if (configuration.pressure_solver == PressureSolver::red_black_gauss_seidel)
            m.pressure = XsPressureSolve{XS_SOLVER_RED_BLACK_GAUSS_SEIDEL, configuration.pressure_iterations, 0.0, nullptr};
        else
            m.pressure = XsPressureSolve{XS_SOLVER_JACOBI_PCG, configuration.pressure_max_iterations, configuration.pressure_tolerance, nullptr};
        for (const Inflow& f : configuration.inflows)
            ctx.inflows_.push_back(XsInflow{{f.center.x, f.center.y, f.center.z}, f.radius, f.density, f.temperature});
        m.inflows = ctx.inflows_.data();
        m.inflow_count = static_cast<std::uint32_t>(ctx.inflows_.size());
        m.cell_mask = colliders ? ctx.domain.cell_mask.data : nullptr;
        m.collider_velocity = colliders ? view(ctx.domain.collider_velocity) : XsVector{nullptr, nullptr, nullptr};
        m.collider_density = colliders ? ctx.domain.collider_density.values.data : nullptr;
        m.collider_temperature = colliders ? ctx.domain.collider_temperature.values.data : nullptr;
        m.warm_start_history = configuration.warm_start_history;
        m.warm_start_coarsening = configuration.warm_start_coarsening;
        m.warm_start_rounds = configuration.warm_start_rounds;
        const std::size_t bytes = xs_smoke_workspace_bytes(&m, static_cast<std::uint32_t>(mode));
        if (bytes == 0) throw std::invalid_argument("invalid smoke configuration");
        ctx.workspace_ = cuda::Buffer<unsigned char>(ctx.resource, bytes);
        check(xs_smoke_reset_warm_start(ctx.resource->stream(), &m, ctx.workspace_.data, static_cast<std::uint32_t>(mode)),
              "xs_smoke_reset_warm_start");
        ctx.resource->synchronize();
        return ctx;
    }

    [[nodiscard]] State allocate_state(ExecutionContext& c) const {
        State s{scalar(c), scalar(c), staggered(c)};
        zero(c, s);
        return s;
    }
    [[nodiscard]] Control allocate_control(ExecutionContext& c) const {
        Control v{scalar(c), scalar(c), centered(c)};
        for (float* p : {v.density_source.values.data, v.temperature_source.values.data, v.external_acceleration.x.values.data,
                         v.external_acceleration.y.values.data, v.external_acceleration.z.values.data})
            c.resource->zero(p, cell_count() * sizeof(float));
        return v;
    }
    [[nodiscard]] Parameters allocate_parameters(ExecutionContext& c) const {
        Parameters p{cuda::Buffer<float>(c.resource, 1u), cuda::Buffer<float>(c.resource, 1u), cuda::Buffer<float>(c.resource, 1u),
                     cuda::Buffer<float>(c.resource, 1u)};
        for (float* q : {p.ambient_temperature.data, p.density_buoyancy.data, p.temperature_buoyancy.data, p.vorticity_confinement.data})
            c.resource->zero(q, sizeof(float));
        return p;
    }
    [[nodiscard]] StepCache allocate_step_cache(ExecutionContext& c) const {
        StepCache k{scalar(c), scalar(c), centered(c), VorticityCache{cuda::Buffer<float>(c.resource, 11u * cell_count()), cell_count()},
                    staggered(c), staggered(c)};
        return k;
    }
    [[nodiscard]] StateTangent allocate_state_tangent(ExecutionContext& c) const { return allocate_state(c); }
    [[nodiscard]] ControlTangent allocate_control_tangent(ExecutionContext& c) const { return allocate_control(c); }
    [[nodiscard]] ParameterTangent allocate_parameter_tangent(ExecutionContext& c) const { return allocate_parameters(c); }
    [[nodiscard]] StateAdjoint allocate_state_adjoint(ExecutionContext& c) const {
        StateAdjoint s{scalar64(c), scalar64(c), staggered64(c)};
        zero(c, s);
        return s;
    }
    [[nodiscard]] ControlAdjoint allocate_control_adjoint(ExecutionContext& c) const {
        ControlAdjoint v{scalar64(c), scalar64(c), CenteredVectorAdjointField{scalar64(c), scalar64(c), scalar64(c)}};
        for (double* p : {v.density_source.values.data, v.temperature_source.values.data, v.external_acceleration.x.values.data,
                          v.external_acceleration.y.values.data, v.external_acceleration.z.values.data})
            c.resource->zero(p, cell_count() * sizeof(double));
        return v;
    }
    [[nodiscard]] ParameterAdjoint allocate_parameter_adjoint(ExecutionContext& c) const {
        ParameterAdjoint p{cuda::Buffer<double>(c.resource, 1u), cuda::Buffer<double>(c.resource, 1u), cuda::Buffer<double>(c.resource, 1u),
                           cuda::Buffer<double>(c.resource, 1u)};
        for (double* q : {p.ambient_temperature.data, p.density_buoyancy.data, p.temperature_buoyancy.data, p.vorticity_confinement.data})
            c.resource->zero(q, sizeof(double));
        return p;
    }

    // model.cpp:308-339
    void copy_state(const State& s, State& d, ExecutionContext& c) const { copy(c, s, d); }
    void copy_state_tangent(const StateTangent& s, StateTangent& d, ExecutionContext& c) const { copy(c, s, d); }
    void copy_state_adjoint(const StateAdjoint& s, StateAdjoint& d, ExecutionContext& c) const { copy(c, s, d); }
    void accumulate_state_adjoint(const StateAdjoint& s, StateAdjoint& d, ExecutionContext& c) const {
        const cudaStream_t st = c.resource->stream();
        check(xs_accumulate(st, s.density.values.data, d.density.values.data, s.density.values.size), "xs_accumulate");
        check(xs_accumulate(st, s.temperature.values.data, d.temperature.values.data, s.temperature.values.size), "xs_accumulate");
        check(xs_accumulate(st, s.velocity.x.data, d.velocity.x.data, s.velocity.x.size), "xs_accumulate");
        check(xs_accumulate(st, s.velocity.y.data, d.velocity.y.data, s.velocity.y.size), "xs_accumulate");
        check(xs_accumulate(st, s.velocity.z.data, d.velocity.z.data, s.velocity.z.size), "xs_accumulate");
    }

    // model.cpp:341-349
    void forward_step(const State& s, const Control& u, const Parameters& p, State& next, StepCache& k, ExecutionContext& c) const {
        check(xs_smoke_forward_step(c.resource->stream(), &c.native_, view(s), view(u), view(p), view(next), view(k), c.workspace_.data),
              "xs_smoke_forward_step");
    }
    // model.cpp:351-359
    void jvp_step(const State& s, const Control&, const Parameters& p, const State& next, const StepCache& k, const StateTangent& st,
                  const ControlTangent& ct, const ParameterTangent& pt, StateTangent& nt, ExecutionContext& c) const {
        require_differentiable(c);
        check(xs_smoke_jvp_step(c.resource->stream(), &c.native_, view(s), view(p), view(next), view(k), view(st), view(ct), view(pt), view(nt),
                                c.workspace_.data),
              "xs_smoke_jvp_step");
    }
    // model.cpp:361-389
    void vjp_step(const State& s, const Control&, const Parameters& p, const State& next, const StepCache& k, const StateAdjoint& na,
                  StateAdjoint& pa, ControlAdjoint& ca, ParameterAdjoint& qa, ExecutionContext& c) const {
        require_differentiable(c);
        check(xs_smoke_vjp_step(c.resource->stream(), &c.native_, view(s), view(p), view(next), view(k), view(na), view(pa), view(ca), view(qa),
                                c.workspace_.data),
              "xs_smoke_vjp_step");
    }

    [[nodiscard]] std::size_t cell_count() const {
        return static_cast<std::size_t>(configuration.resolution[0]) * configuration.resolution[1] * configuration.resolution[2];
    }
    [[nodiscard]] std::array<std::size_t, 3u> face_counts() const {
        const auto& r = configuration.resolution;
        return {static_cast<std::size_t>(r[0] + 1u) * r[1] * r[2], static_cast<std::size_t>(r[0]) * (r[1] + 1u) * r[2],
                static_cast<std::size_t>(r[0]) * r[1] * (r[2] + 1u)};
    }

private:
    [[nodiscard]] XsGrid grid() const {
        return XsGrid{configuration.resolution[0], configuration.resolution[1], configuration.resolution[2], configuration.cell_size,
                      configuration.time_step};
    }
    static XsScalarBoundary pack(const ScalarBoundary& b) {  // operators.cpp:85-93
        const ScalarBoundaryFace f[6] = {b.x_min, b.x_max, b.y_min, b.y_max, b.z_min, b.z_max};
        XsScalarBoundary out{};
        for (int i = 0; i < 6; ++i) {
            out.modes[i] = static_cast<std::uint32_t>(f[i].mode);
            out.values[i] = f[i].value;
        }
        return out;
    }
    static XsVelocityBoundary pack(const VelocityBoundary& b) {  // operators.cpp:95-105
        const VelocityBoundaryFace f[6] = {b.x_min, b.x_max, b.y_min, b.y_max, b.z_min, b.z_max};
        XsVelocityBoundary out{};
        for (int i = 0; i < 6; ++i) {
            out.modes[i] = static_cast<std::uint32_t>(f[i].mode);
            out.values[3 * i] = f[i].value.x;
            out.values[3 * i + 1] = f[i].value.y;
            out.values[3 * i + 2] = f[i].value.z;
        }
        return out;
    }
    ScalarField scalar(ExecutionContext& c) const { return ScalarField{cuda::Buffer<float>(c.resource, cell_count())}; }
    ScalarAdjointField scalar64(ExecutionContext& c) const { return ScalarAdjointField{cuda::Buffer<double>(c.resource, cell_count())}; }
    CenteredVectorField centered(ExecutionContext& c) const { return CenteredVectorField{scalar(c), scalar(c), scalar(c)}; }
    StaggeredVectorField staggered(ExecutionContext& c) const {
        const auto f = face_counts();
        return StaggeredVectorField{cuda::Buffer<float>(c.resource, f[0]), cuda::Buffer<float>(c.resource, f[1]), cuda::Buffer<float>(c.resource, f[2])};
    }
    StaggeredVectorAdjointField staggered64(ExecutionContext& c) const {
        const auto f = face_counts();
        return StaggeredVectorAdjointField{cuda::Buffer<double>(c.resource, f[0]), cuda::Buffer<double>(c.resource, f[1]),
                                           cuda::Buffer<double>(c.resource, f[2])};
    }
    template <class S>
    static void zero(ExecutionContext& c, S& s) {
        using E = std::remove_pointer_t<decltype(s.density.values.data)>;
        c.resource->zero(s.density.values.data, s.density.values.size * sizeof(E));
        c.resource->zero(s.temperature.values.data, s.temperature.values.size * sizeof(E));
        c.resource->zero(s.velocity.x.data, s.velocity.x.size * sizeof(E));
        c.resource->zero(s.velocity.y.data, s.velocity.y.size * sizeof(E));
        c.resource->zero(s.velocity.z.data, s.velocity.z.size * sizeof(E));
    }
    template <class S>
    static void copy(ExecutionContext& c, const S& s, S& d) {
        using E = std::remove_pointer_t<decltype(s.density.values.data)>;
        c.resource->copy_device(d.density.values.data, s.density.values.data, s.density.values.size * sizeof(E));
        c.resource->copy_device(d.temperature.values.data, s.temperature.values.data, s.temperature.values.size * sizeof(E));
        c.resource->copy_device(d.velocity.x.data, s.velocity.x.data, s.velocity.x.size * sizeof(E));
        c.resource->copy_device(d.velocity.y.data, s.velocity.y.data, s.velocity.y.size * sizeof(E));
        c.resource->copy_device(d.velocity.z.data, s.velocity.z.data, s.velocity.z.size * sizeof(E));
    }
    static void require_differentiable(const ExecutionContext& c) {
        if (c.mode_ != ExecutionMode::differentiable) throw std::logic_error("jvp_step / vjp_step need ExecutionMode::differentiable");
    }
    static XsVector view(const StaggeredVectorField& f) { return XsVector{f.x.data, f.y.data, f.z.data}; }
    static XsVector view(const CenteredVectorField& f) { return XsVector{f.x.values.data, f.y.values.data, f.z.values.data}; }
    static XsAdjointVector view(const StaggeredVectorAdjointField& f) { return XsAdjointVector{f.x.data, f.y.data, f.z.data}; }
    static XsAdjointVector view(const CenteredVectorAdjointField& f) { return XsAdjointVector{f.x.values.data, f.y.values.data, f.z.values.data}; }
    static XsState view(const State& s) { return XsState{s.density.values.data, s.temperature.values.data, view(s.velocity)}; }
    static XsControl view(const Control& u) { return XsControl{u.density_source.values.data, u.temperature_source.values.data, view(u.external_acceleration)}; }
    static XsParameters view(const Parameters& p) {
        return XsParameters{p.ambient_temperature.data, p.density_buoyancy.data, p.temperature_buoyancy.data, p.vorticity_confinement.data};
    }
    static XsStepCache view(const StepCache& k) {
        return XsStepCache{k.sourced_density.values.data, k.sourced_temperature.values.data, view(k.force), k.vorticity.storage.data,
                           view(k.forced_velocity), view(k.advected_velocity)};
    }
    static XsStateAdjoint view(const StateAdjoint& s) { return XsStateAdjoint{s.density.values.data, s.temperature.values.data, view(s.velocity)}; }
    static XsControlAdjoint view(const ControlAdjoint& u) {
        return XsControlAdjoint{u.density_source.values.data, u.temperature_source.values.data, view(u.external_acceleration)};
    }
    static XsParameterAdjoint view(const ParameterAdjoint& p) {
        return XsParameterAdjoint{p.ambient_temperature.data, p.density_buoyancy.data, p.temperature_buoyancy.data, p.vorticity_confinement.data};
    }
};

}  // namespace xayah::smoke
