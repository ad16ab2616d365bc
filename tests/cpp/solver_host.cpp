// The model-agnostic C++ solver (include/xayah/solver.hpp) on a small CPU
// model, with no GPU: every tape mode must give the same rollout, the same
// tangents and the same gradients (bit for bit: the steps run the same
// arithmetic in the same order), the gradient must be the transpose of the
// tangent map, and it must match central differences of simulate.
//
// The toy step is x' = tanh(W x) + theta u.  The step cache holds W x, and
// the tangent and adjoint steps read the nonlinearity's derivative from the
// cache only, so a stale or misplaced cache changes the results.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <span>
#include <stdexcept>
#include <vector>

#include "xayah/solver.hpp"

namespace {

using Vec = std::vector<double>;
using xayah::solver::TapeMode;

struct Context {
    std::size_t forward_steps = 0;
};

struct Cache {
    Vec pre;
};

struct ToyModel {
    std::size_t n;
    Vec w;  // n x n, row-major

    Vec allocate_state(Context&) const { return Vec(n, 0.0); }
    Cache allocate_step_cache(Context&) const { return Cache{Vec(n, 0.0)}; }
    void copy_state(const Vec& a, Vec& b, Context&) const { b = a; }
    void forward_step(const Vec& x, const Vec& u, const Vec& theta, Vec& y, Cache& c, Context& ctx) const {
        ++ctx.forward_steps;
        for (std::size_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (std::size_t j = 0; j < n; ++j) s += w[i * n + j] * x[j];
            c.pre[i] = s;
            y[i] = std::tanh(s) + theta[0] * u[i];
        }
    }

    Vec allocate_state_tangent(Context&) const { return Vec(n, 0.0); }
    Vec allocate_control_tangent(Context&) const { return Vec(n, 0.0); }
    Vec allocate_parameter_tangent(Context&) const { return Vec(1, 0.0); }
    void copy_state_tangent(const Vec& a, Vec& b, Context&) const { b = a; }
    void jvp_step(const Vec&, const Vec& u, const Vec& theta, const Vec&, const Cache& c, const Vec& dx, const Vec& du, const Vec& dtheta,
                  Vec& dy, Context&) const {
        for (std::size_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (std::size_t j = 0; j < n; ++j) s += w[i * n + j] * dx[j];
            const double t = std::tanh(c.pre[i]);
            dy[i] = (1.0 - t * t) * s + dtheta[0] * u[i] + theta[0] * du[i];
        }
    }

    Vec allocate_state_adjoint(Context&) const { return Vec(n, 0.0); }
    Vec allocate_control_adjoint(Context&) const { return Vec(n, 0.0); }
    Vec allocate_parameter_adjoint(Context&) const { return Vec(1, 0.0); }
    void copy_state_adjoint(const Vec& a, Vec& b, Context&) const { b = a; }
    void accumulate_state_adjoint(const Vec& a, Vec& b, Context&) const {
        for (std::size_t i = 0; i < n; ++i) b[i] += a[i];
    }
    // accumulates into the three adjoint outputs, as the smoke model does
    void vjp_step(const Vec&, const Vec& u, const Vec& theta, const Vec&, const Cache& c, const Vec& next_adj, Vec& prev_adj, Vec& u_adj,
                  Vec& theta_adj, Context&) const {
        for (std::size_t i = 0; i < n; ++i) {
            const double t = std::tanh(c.pre[i]);
            const double g = next_adj[i] * (1.0 - t * t);
            for (std::size_t j = 0; j < n; ++j) prev_adj[j] += w[i * n + j] * g;
            u_adj[i] += theta[0] * next_adj[i];
            theta_adj[0] += next_adj[i] * u[i];
        }
    }
};

int failures = 0;

void expect(bool ok, const char* what, std::size_t k) {
    if (!ok) {
        std::fprintf(stderr, "FAILED: %s (checkpoint interval %zu)\n", what, k);
        ++failures;
    }
}

double dot(const Vec& a, const Vec& b) {
    double s = 0.0;
    for (std::size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

Vec random_vec(std::mt19937_64& rng, std::size_t n, double scale) {
    std::normal_distribution<double> d(0.0, scale);
    Vec v(n);
    for (double& x : v) x = d(rng);
    return v;
}

// L = sum_t <seed_t, x_t> over the rollout from x0 with controls u and theta
double objective(const ToyModel& m, const Vec& x0, const std::vector<Vec>& u, const Vec& theta, const std::vector<Vec>& seeds) {
    Context ctx;
    auto traj = xayah::solver::simulate(m, ctx, x0, std::span<const Vec>(u), theta, TapeMode::store_all);
    double s = 0.0;
    for (std::size_t t = 0; t < traj.states.size(); ++t) s += dot(seeds[t], traj.states[t]);
    return s;
}

}  // namespace

int main() {
    constexpr std::size_t n = 6, steps = 7;
    std::mt19937_64 rng(7);
    ToyModel m{n, random_vec(rng, n * n, 0.6)};
    const Vec x0 = random_vec(rng, n, 1.0);
    const Vec theta{0.7};
    std::vector<Vec> u, du, seeds;
    for (std::size_t t = 0; t < steps; ++t) {
        u.push_back(random_vec(rng, n, 0.5));
        du.push_back(random_vec(rng, n, 1.0));
    }
    for (std::size_t t = 0; t <= steps; ++t) seeds.push_back(random_vec(rng, n, 1.0));
    const Vec dx0 = random_vec(rng, n, 1.0), dtheta{0.3};
    const std::span<const Vec> controls(u);

    Context ref_ctx;
    const auto ref = xayah::solver::simulate(m, ref_ctx, x0, controls, theta, TapeMode::store_all);
    const auto ref_tan = xayah::solver::jvp(m, ref_ctx, ref, controls, theta, dx0, std::span<const Vec>(du), dtheta);
    const auto ref_grad = xayah::solver::vjp(m, ref_ctx, ref, controls, theta, std::span<const Vec>(seeds));
    expect(ref.states.size() == steps + 1 && ref.step_caches.size() == steps, "store_all keeps every state and cache", 0);

    // the gradient is the transpose of the tangent map
    double lhs = 0.0;
    for (std::size_t t = 0; t <= steps; ++t) lhs += dot(seeds[t], ref_tan[t]);
    double rhs = dot(ref_grad.initial_state, dx0) + ref_grad.parameters[0] * dtheta[0];
    for (std::size_t t = 0; t < steps; ++t) rhs += dot(ref_grad.controls[t], du[t]);
    expect(std::fabs(lhs - rhs) <= 1e-12 * std::fabs(lhs), "<seed, J v> == <J^T seed, v>", 0);

    // central differences of simulate along (dx0, du, dtheta)
    const double eps = 1e-6;
    auto shifted = [&](double s) {
        Vec x = x0, th{theta[0] + s * dtheta[0]};
        for (std::size_t i = 0; i < n; ++i) x[i] += s * dx0[i];
        std::vector<Vec> us = u;
        for (std::size_t t = 0; t < steps; ++t)
            for (std::size_t i = 0; i < n; ++i) us[t][i] += s * du[t][i];
        return objective(m, x, us, th, seeds);
    };
    const double fd = (shifted(eps) - shifted(-eps)) / (2.0 * eps);
    expect(std::fabs(fd - rhs) <= 1e-7 * std::fabs(rhs), "gradient matches central differences", 0);

    // the other tape modes reproduce store_all bit for bit
    struct Mode {
        TapeMode mode;
        std::size_t k;
    };
    const Mode modes[] = {{TapeMode::recompute_step_cache, 0}, {TapeMode::checkpoint, 1}, {TapeMode::checkpoint, 2},
                          {TapeMode::checkpoint, 3}, {TapeMode::checkpoint, steps}, {TapeMode::checkpoint, steps + 3}};
    for (const Mode& md : modes) {
        Context ctx;
        const auto tr = xayah::solver::simulate(m, ctx, x0, controls, theta, md.mode, md.k);
        expect(ctx.forward_steps == steps, "simulate runs each step once", md.k);
        if (md.mode == TapeMode::checkpoint) {
            std::vector<std::size_t> want;
            for (std::size_t s = 0; s < steps; s += md.k) want.push_back(s);
            want.push_back(steps);
            expect(tr.checkpoint_steps == want, "checkpoints at multiples of k and the last step", md.k);
            expect(tr.states.size() == want.size() && tr.step_caches.empty(), "checkpoint tape keeps only its checkpoints", md.k);
            expect(tr.states.back() == ref.states.back(), "final checkpoint equals the stored final state", md.k);
        } else {
            expect(tr.states == ref.states && tr.step_caches.empty(), "recompute tape keeps every state and no cache", md.k);
        }
        const auto tan = xayah::solver::jvp(m, ctx, tr, controls, theta, dx0, std::span<const Vec>(du), dtheta);
        bool same = tan.size() == ref_tan.size();
        for (std::size_t t = 0; same && t < tan.size(); ++t) same = tan[t] == ref_tan[t];
        expect(same, "tangents equal store_all's", md.k);
        ctx.forward_steps = 0;
        const auto grad = xayah::solver::vjp(m, ctx, tr, controls, theta, std::span<const Vec>(seeds));
        // every step is recomputed exactly once on the reverse pass
        expect(ctx.forward_steps == steps, "reverse pass recomputes each step once", md.k);
        same = grad.initial_state == ref_grad.initial_state && grad.parameters == ref_grad.parameters;
        for (std::size_t t = 0; same && t < steps; ++t) same = grad.controls[t] == ref_grad.controls[t];
        expect(same, "gradients equal store_all's", md.k);
    }

    // an empty rollout: the gradient of the initial state is its own seed
    {
        Context ctx;
        const std::vector<Vec> none;
        const auto tr = xayah::solver::simulate(m, ctx, x0, std::span<const Vec>(none), theta, TapeMode::checkpoint, 4);
        const std::vector<Vec> one_seed{seeds[0]};
        const auto grad = xayah::solver::vjp(m, ctx, tr, std::span<const Vec>(none), theta, std::span<const Vec>(one_seed));
        expect(tr.states.size() == 1 && grad.initial_state == seeds[0] && grad.controls.empty(), "empty rollout", 4);
    }

    // a checkpoint tape needs an interval
    {
        Context ctx;
        bool threw = false;
        try {
            (void)xayah::solver::simulate(m, ctx, x0, controls, theta, TapeMode::checkpoint, 0);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        expect(threw, "checkpoint interval 0 is rejected", 0);
    }

    if (failures) return 1;
    std::printf("solver host checks ok\n");
    return 0;
}
