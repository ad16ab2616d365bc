// C++ host API check: xayah::smoke::Model and xayah::solver::simulate / jvp /
// vjp (the drop-in headers) on the B200 kernels.  Prints one JSON line that
// tests/test_gpu_cpp.py checks.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "xayah/smoke.hpp"
#include "xayah/solver.hpp"
#include "xayah/warm_start.hpp"

using namespace xayah;

namespace {

smoke::Configuration plume() {
    smoke::Configuration c{};
    c.resolution = {20u, 18u, 16u};
    c.cell_size = 1.0F / 20.0F;
    c.time_step = 0.5F * c.cell_size;
    c.velocity_boundary.x_min.mode = smoke::VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.x_max.mode = smoke::VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.y_min.mode = smoke::VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.y_max.mode = smoke::VelocityBoundaryMode::zero_gradient;
    c.velocity_boundary.z_min.mode = smoke::VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.velocity_boundary.z_max.mode = smoke::VelocityBoundaryMode::normal_fixed_tangent_zero_gradient;
    c.pressure_boundary.y_max.mode = smoke::ScalarBoundaryMode::fixed_value;
    c.density_boundary.y_max.mode = smoke::ScalarBoundaryMode::fixed_value;
    c.temperature_boundary.y_max.mode = smoke::ScalarBoundaryMode::fixed_value;
    c.vorticity_confinement_enabled = true;
    c.inflows.push_back(smoke::Inflow{{0.5F, 0.15F, 0.5F}, 0.15F, 1.0F, 1.0F});
    c.pressure_tolerance = 1.0e-10;
    c.pressure_max_iterations = 20000u;
    return c;
}

template <class T>
std::vector<T> download(cuda::Resource& r, const T* p, std::size_t n) {
    std::vector<T> h(n);
    r.copy_to_host(h.data(), p, n * sizeof(T));
    r.synchronize();
    return h;
}

template <class T>
double max_rel(const std::vector<T>& a, const std::vector<T>& b) {
    double num = 0.0, den = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) {
        num = std::fmax(num, std::fabs(static_cast<double>(a[i]) - static_cast<double>(b[i])));
        den = std::fmax(den, std::fabs(static_cast<double>(b[i])));
    }
    return den > 0.0 ? num / den : num;
}

}  // namespace

int main() {
    try {
        const smoke::Model model{plume()};
        smoke::ExecutionContext ctx = model.allocate_context(smoke::ExecutionMode::differentiable);
        cuda::Resource& res = *ctx.resource;
        const std::size_t n = model.cell_count();
        const auto fc = model.face_counts();
        smoke::State initial = model.allocate_state(ctx);
        std::mt19937 rng(7);
        std::uniform_real_distribution<float> noise(-0.2F, 0.2F);
        std::vector<float> host;
        float* comps[3] = {initial.velocity.x.data, initial.velocity.y.data, initial.velocity.z.data};
        for (int a = 0; a < 3; ++a) {
            host.resize(fc[a]);
            for (float& v : host) v = noise(rng);
            res.copy_from_host(comps[a], host.data(), fc[a] * sizeof(float));
        }
        smoke::Parameters params = model.allocate_parameters(ctx);
        const float values[4] = {0.0F, -0.1F, 0.5F, 1.0F};
        res.copy_from_host(params.ambient_temperature.data, &values[0], 4);
        res.copy_from_host(params.density_buoyancy.data, &values[1], 4);
        res.copy_from_host(params.temperature_buoyancy.data, &values[2], 4);
        res.copy_from_host(params.vorticity_confinement.data, &values[3], 4);
        const std::size_t steps = 6;
        std::vector<smoke::Control> controls;
        for (std::size_t i = 0; i < steps; ++i) controls.push_back(model.allocate_control(ctx));
        const std::span<const smoke::Control> cs{controls};

        auto all = solver::simulate(model, ctx, initial, cs, params, solver::TapeMode::store_all);
        auto rec = solver::simulate(model, ctx, initial, cs, params, solver::TapeMode::recompute_step_cache);
        auto chk = solver::simulate(model, ctx, initial, cs, params, solver::TapeMode::checkpoint, 4);
        const auto final_all = download(res, all.states.back().density.values.data, n);
        const auto final_chk = download(res, chk.states.back().density.values.data, n);
        const double forward_diff = max_rel(final_chk, final_all);

        // seed: d(sum of final density) / d(everything)
        auto seeds_for = [&]() {
            std::vector<smoke::StateAdjoint> seeds;
            for (std::size_t i = 0; i <= steps; ++i) seeds.push_back(model.allocate_state_adjoint(ctx));
            std::vector<double> ones(n, 1.0);
            res.copy_from_host(seeds.back().density.values.data, ones.data(), n * sizeof(double));
            return seeds;
        };
        auto seeds = seeds_for();
        const std::span<const smoke::StateAdjoint> ss{seeds};
        auto g_all = solver::vjp(model, ctx, all, cs, params, ss);
        auto g_rec = solver::vjp(model, ctx, rec, cs, params, ss);
        auto g_chk = solver::vjp(model, ctx, chk, cs, params, ss);
        const auto gu_all = download(res, g_all.initial_state.velocity.y.data, fc[1]);
        const auto gu_rec = download(res, g_rec.initial_state.velocity.y.data, fc[1]);
        const auto gu_chk = download(res, g_chk.initial_state.velocity.y.data, fc[1]);

        // tangent along a random initial-velocity direction: <J v, seed> = <v, J^T seed>
        smoke::StateTangent v = model.allocate_state_tangent(ctx);
        std::vector<std::vector<float>> vhost(3);
        float* vcomps[3] = {v.velocity.x.data, v.velocity.y.data, v.velocity.z.data};
        for (int a = 0; a < 3; ++a) {
            vhost[a].resize(fc[a]);
            for (float& x : vhost[a]) x = noise(rng);
            res.copy_from_host(vcomps[a], vhost[a].data(), fc[a] * sizeof(float));
        }
        std::vector<smoke::ControlTangent> ct;
        for (std::size_t i = 0; i < steps; ++i) ct.push_back(model.allocate_control_tangent(ctx));
        smoke::ParameterTangent pt = model.allocate_parameter_tangent(ctx);
        auto tangents = solver::jvp(model, ctx, chk, cs, params, v, std::span<const smoke::ControlTangent>{ct}, pt);
        const auto jv = download(res, tangents.back().density.values.data, n);
        double lhs = 0.0;
        for (float x : jv) lhs += x;
        double rhs = 0.0;
        const double* gcomps[3] = {g_chk.initial_state.velocity.x.data, g_chk.initial_state.velocity.y.data, g_chk.initial_state.velocity.z.data};
        for (int a = 0; a < 3; ++a) {
            const auto g = download(res, gcomps[a], fc[a]);
            for (std::size_t i = 0; i < g.size(); ++i) rhs += g[i] * vhost[a][i];
        }
        const XsSolveStats st = ctx.solve_stats();

        // learned warm start on a grid the network tiles (128 x 64 x 32, network at factor 1)
        smoke::Configuration wc = plume();
        wc.resolution = {128u, 64u, 32u};
        wc.cell_size = 1.0F / 128.0F;
        wc.time_step = 0.5F * wc.cell_size;
        wc.vorticity_confinement_enabled = false;
        wc.pressure_tolerance = 1.0e-6;
        const smoke::Model wmodel{wc};
        smoke::ExecutionContext wctx = wmodel.allocate_context(smoke::ExecutionMode::forward);
        smoke::WarmStartNetwork net(128u, 64u, 32u, 1u, 1u, 3u, wctx.resource->stream());
        wctx.set_learned_warm_start(net.native());
        smoke::State w0 = wmodel.allocate_state(wctx);
        smoke::Parameters wp = wmodel.allocate_parameters(wctx);
        wctx.resource->copy_from_host(wp.density_buoyancy.data, &values[1], 4);
        wctx.resource->copy_from_host(wp.temperature_buoyancy.data, &values[2], 4);
        std::vector<smoke::Control> wcontrols;
        for (int i = 0; i < 3; ++i) wcontrols.push_back(wmodel.allocate_control(wctx));
        auto wtraj = solver::simulate(wmodel, wctx, w0, std::span<const smoke::Control>{wcontrols}, wp, solver::TapeMode::recompute_step_cache);
        net.check_status();
        const XsSolveStats wst = wctx.solve_stats();
        std::printf("{\"forward_checkpoint_vs_store_all\": %.3e, \"vjp_recompute_vs_store_all\": %.3e, "
                    "\"vjp_checkpoint_vs_store_all\": %.3e, \"dot_jvp\": %.12e, \"dot_vjp\": %.12e, \"checkpoints\": %zu, "
                    "\"last_solve_status\": %u, \"last_solve_residual\": %.3e, \"warm_solve_status\": %u, "
                    "\"warm_solve_residual\": %.3e, \"warm_states\": %zu}\n",
                    forward_diff, max_rel(gu_rec, gu_all), max_rel(gu_chk, gu_all), lhs, rhs, chk.states.size(), st.status,
                    st.final_residual, wst.status, wst.final_residual, wtraj.states.size());
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "test_solver failed: %s\n", e.what());
        return 1;
    }
}
