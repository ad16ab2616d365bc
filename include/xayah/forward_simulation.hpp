// The forward example driver: C++ mirror of the reference's module
// xayah.examples.smoke.forward (examples/smoke/forward/simulation.ixx:8-66,
// simulation.cpp:15-120, simulation.h:8-13) over this library.
//
// A 128 x 192 x 128 thermal smoke scene driven by two pulsed Gaussian jets
// (xs_smoke_write_control) and stepped through Model::forward_step; after
// every step the metrics are reduced on the device (xs_smoke_reduce_metrics)
// and, with host_metrics, read back.  The reference solves the pressure with
// 160 red-black Gauss-Seidel sweeps; pressure_solver (an addition) selects the
// Jacobi-PCG solve to pressure_tolerance instead.
#pragma once

#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <utility>

#include "xayah/smoke.hpp"

namespace xayah::smoke::examples::forward {

// simulation.ixx:10-29
struct ForwardSimulationOptions {
    std::array<std::uint32_t, 3u> resolution{128u, 192u, 128u};
    float cell_size{1.0F / 128.0F};
    float time_step{1.0F / 120.0F};
    std::uint32_t pressure_iterations{160u};
    float density_source_rate{4.0F};
    float temperature_source_rate{8.0F};
    float ambient_temperature{};
    float density_buoyancy{-0.1F};
    float temperature_buoyancy{1.0F};
    float vorticity_confinement{2.0F};
    Vector3 left_source_center{0.25F, 0.10F, 0.36F};
    Vector3 right_source_center{0.75F, 0.10F, 0.64F};
    float source_radius{0.055F};
    Vector3 left_acceleration{3.5F, 5.0F, 1.8F};
    Vector3 right_acceleration{-3.5F, 5.0F, -1.8F};
    float pulse_period{0.9F};
    bool host_metrics{true};
    // additions
    PressureSolver pressure_solver{PressureSolver::red_black_gauss_seidel};
    double pressure_tolerance{1.0e-6};
};

// simulation.ixx:31-44
struct ForwardSimulationMetrics {
    std::uint64_t step{};
    double physical_time{};
    double density_mass{};
    double density_maximum{};
    double temperature_maximum{};
    double maximum_velocity{};
    double cfl{};
    double pre_projection_divergence_rms{};
    double post_projection_divergence_rms{};
    double divergence_ratio{};
    double step_milliseconds{};
    double average_step_milliseconds{};
};

// simulation.cpp:17-33
inline Configuration make_configuration(const ForwardSimulationOptions& o) {
    Configuration c{};
    c.resolution = o.resolution;
    c.cell_size = o.cell_size;
    c.time_step = o.time_step;
    c.pressure_iterations = o.pressure_iterations;
    c.velocity_boundary.x_min.mode = VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.x_max.mode = VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.y_min.mode = VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.y_max.mode = VelocityBoundaryMode::zero_gradient;
    c.velocity_boundary.z_min.mode = VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.z_max.mode = VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.pressure_boundary.y_max.mode = ScalarBoundaryMode::fixed_value;
    c.density_boundary.y_max.mode = ScalarBoundaryMode::fixed_value;
    c.temperature_boundary.y_max.mode = ScalarBoundaryMode::fixed_value;
    c.vorticity_confinement_enabled = true;
    c.pressure_solver = o.pressure_solver;
    c.pressure_tolerance = o.pressure_tolerance;
    c.pressure_max_iterations = 20000u;
    return c;
}

// simulation.ixx:46-64, simulation.cpp:72-120
struct ForwardSimulation {
    ForwardSimulationOptions options;
    Model model;
    ExecutionContext context;
    State current_state;
    ForwardSimulationMetrics metrics;
    cuda::Buffer<double> device_metrics;

    explicit ForwardSimulation(ForwardSimulationOptions next_options = {})
        : options(next_options), model(make_configuration(options)), context(model.allocate_context(ExecutionMode::forward)),
          current_state(model.allocate_state(context)), metrics{}, device_metrics(context.resource, 6u),
          next_state_(model.allocate_state(context)), control_(model.allocate_control(context)),
          parameters_(model.allocate_parameters(context)), step_cache_(model.allocate_step_cache(context)) {
        context.resource->copy_from_host(parameters_.ambient_temperature.data, &options.ambient_temperature, sizeof(float));
        context.resource->copy_from_host(parameters_.density_buoyancy.data, &options.density_buoyancy, sizeof(float));
        context.resource->copy_from_host(parameters_.temperature_buoyancy.data, &options.temperature_buoyancy, sizeof(float));
        context.resource->copy_from_host(parameters_.vorticity_confinement.data, &options.vorticity_confinement, sizeof(float));
        context.resource->synchronize();
        reset();
    }

    ForwardSimulation(const ForwardSimulation&) = delete;
    ForwardSimulation& operator=(const ForwardSimulation&) = delete;

    // simulation.cpp:80-92
    void reset() {
        for (State* s : {&current_state, &next_state_})
            for (auto [p, n] : {std::pair{s->density.values.data, s->density.values.size}, std::pair{s->temperature.values.data, s->temperature.values.size},
                                std::pair{s->velocity.x.data, s->velocity.x.size}, std::pair{s->velocity.y.data, s->velocity.y.size},
                                std::pair{s->velocity.z.data, s->velocity.z.size}})
                context.resource->zero(p, n * sizeof(float));
        context.resource->zero(device_metrics.data, 6u * sizeof(double));
        context.resource->synchronize();
        metrics = {};
    }

    // simulation.cpp:94-120
    void step() {
        const auto begin = options.host_metrics ? std::chrono::steady_clock::now() : std::chrono::steady_clock::time_point{};
        const cudaStream_t stream = context.resource->stream();
        const XsSmokeModel& m = context.native();
        check(xs_smoke_write_control(stream, m.grid, metrics.step, options.pulse_period, vec3(options.left_source_center),
                                     vec3(options.right_source_center), options.source_radius, options.density_source_rate,
                                     options.temperature_source_rate, vec3(options.left_acceleration), vec3(options.right_acceleration),
                                     control_.density_source.values.data, control_.temperature_source.values.data,
                                     XsVector{control_.external_acceleration.x.values.data, control_.external_acceleration.y.values.data,
                                              control_.external_acceleration.z.values.data}),
              "xs_smoke_write_control");
        model.forward_step(current_state, control_, parameters_, next_state_, step_cache_, context);
        const StaggeredVectorField& pre = step_cache_.advected_velocity;
        const StaggeredVectorField& post = next_state_.velocity;
        check(xs_smoke_reduce_metrics(stream, &m, next_state_.density.values.data, next_state_.temperature.values.data,
                                      XsVector{pre.x.data, pre.y.data, pre.z.data}, XsVector{post.x.data, post.y.data, post.z.data},
                                      device_metrics.data),
              "xs_smoke_reduce_metrics");
        std::array<double, 6u> values{};
        if (options.host_metrics) {
            context.resource->copy_to_host(values.data(), device_metrics.data, values.size() * sizeof(double));
            context.resource->synchronize();
        }
        std::swap(current_state, next_state_);
        ++metrics.step;
        metrics.physical_time = static_cast<double>(metrics.step) * options.time_step;
        if (!options.host_metrics) return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - begin).count();
        const double previous = static_cast<double>(metrics.step - 1u);
        const double cells = static_cast<double>(options.resolution[0]) * options.resolution[1] * options.resolution[2];
        metrics.density_mass = values[0] * static_cast<double>(options.cell_size) * options.cell_size * options.cell_size;
        metrics.density_maximum = values[1];
        metrics.temperature_maximum = values[2];
        metrics.maximum_velocity = values[3];
        metrics.cfl = values[3] * options.time_step / options.cell_size;
        metrics.pre_projection_divergence_rms = std::sqrt(values[4] / cells);
        metrics.post_projection_divergence_rms = std::sqrt(values[5] / cells);
        metrics.divergence_ratio = metrics.post_projection_divergence_rms / metrics.pre_projection_divergence_rms;
        metrics.step_milliseconds = ms;
        metrics.average_step_milliseconds = (previous * metrics.average_step_milliseconds + ms) / static_cast<double>(metrics.step);
    }

private:
    State next_state_;
    Control control_;
    Parameters parameters_;
    StepCache step_cache_;

    static XsVec3 vec3(const Vector3& v) { return XsVec3{v.x, v.y, v.z}; }
};

}  // namespace xayah::smoke::examples::forward
