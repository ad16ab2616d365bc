// xayah::solver -- model-agnostic rollout and differentiation for C++.
//
// Header-only counterpart of the reference module xayah.solver
// (solvers/solver.ixx:7-150): TapeMode, Trajectory, GradientResult, the
// ForwardModel / JvpModel / VjpModel concepts and simulate / jvp / vjp with
// the same signatures.  Addition: TapeMode::checkpoint keeps only every
// k-th state (plus the last); jvp and vjp recompute one segment of k steps
// (states and step caches) from its checkpoint and then run that segment.
#pragma once

#include <concepts>
#include <cstddef>
#include <optional>
#include <span>
#include <stdexcept>
#include <utility>
#include <vector>

namespace xayah::solver {

enum class TapeMode {
    store_all,
    recompute_step_cache,
    checkpoint,
};

template <typename State, typename StepCache>
struct Trajectory {
    TapeMode tape_mode;
    std::vector<State> states;  // checkpoint mode: states at checkpoint_steps
    std::vector<StepCache> step_caches;
    std::size_t checkpoint_interval{0};
    std::vector<std::size_t> checkpoint_steps{};
};

template <typename StateAdjoint, typename ControlAdjoint, typename ParameterAdjoint>
struct GradientResult {
    StateAdjoint initial_state;
    std::vector<ControlAdjoint> controls;
    ParameterAdjoint parameters;
};

template <typename Model, typename Context, typename State, typename Control, typename Parameters>
concept ForwardModel = requires(const Model& model, Context& context, const State& state, const Control& control, const Parameters& parameters,
                                decltype(std::declval<const Model&>().allocate_state(context))& next_state,
                                decltype(std::declval<const Model&>().allocate_step_cache(context))& step_cache) {
    { model.allocate_state(context) } -> std::same_as<State>;
    model.allocate_step_cache(context);
    { model.copy_state(state, next_state, context) } -> std::same_as<void>;
    { model.forward_step(state, control, parameters, next_state, step_cache, context) } -> std::same_as<void>;
};

template <typename Model, typename Context, typename State, typename Control, typename Parameters>
concept JvpModel = ForwardModel<Model, Context, State, Control, Parameters> &&
    requires(const Model& model, Context& context, const State& state, const Control& control, const Parameters& parameters,
             const State& next_state, const decltype(std::declval<const Model&>().allocate_step_cache(context))& step_cache,
             const decltype(std::declval<const Model&>().allocate_state_tangent(context))& state_tangent,
             const decltype(std::declval<const Model&>().allocate_control_tangent(context))& control_tangent,
             const decltype(std::declval<const Model&>().allocate_parameter_tangent(context))& parameter_tangent,
             decltype(std::declval<const Model&>().allocate_state_tangent(context))& next_state_tangent) {
        model.allocate_state_tangent(context);
        model.allocate_control_tangent(context);
        model.allocate_parameter_tangent(context);
        { model.copy_state_tangent(state_tangent, next_state_tangent, context) } -> std::same_as<void>;
        {
            model.jvp_step(state, control, parameters, next_state, step_cache, state_tangent, control_tangent, parameter_tangent,
                           next_state_tangent, context)
        } -> std::same_as<void>;
    };

template <typename Model, typename Context, typename State, typename Control, typename Parameters>
concept VjpModel = ForwardModel<Model, Context, State, Control, Parameters> &&
    requires(const Model& model, Context& context, const State& state, const Control& control, const Parameters& parameters,
             const State& next_state, const decltype(std::declval<const Model&>().allocate_step_cache(context))& step_cache,
             const decltype(std::declval<const Model&>().allocate_state_adjoint(context))& next_state_adjoint,
             decltype(std::declval<const Model&>().allocate_state_adjoint(context))& previous_state_adjoint,
             decltype(std::declval<const Model&>().allocate_control_adjoint(context))& control_adjoint,
             decltype(std::declval<const Model&>().allocate_parameter_adjoint(context))& parameter_adjoint) {
        model.allocate_state_adjoint(context);
        model.allocate_control_adjoint(context);
        model.allocate_parameter_adjoint(context);
        { model.copy_state_adjoint(next_state_adjoint, previous_state_adjoint, context) } -> std::same_as<void>;
        { model.accumulate_state_adjoint(next_state_adjoint, previous_state_adjoint, context) } -> std::same_as<void>;
        {
            model.vjp_step(state, control, parameters, next_state, step_cache, next_state_adjoint, previous_state_adjoint, control_adjoint,
                           parameter_adjoint, context)
        } -> std::same_as<void>;
    };

namespace detail {

// The states (start .. end) and step caches of the checkpoint segment
// beginning at `start`, recomputed from its checkpoint.
template <typename Model, typename Context, typename State, typename StepCache, typename Control, typename Parameters>
void recompute_segment(const Model& model, Context& context, const Trajectory<State, StepCache>& trajectory, std::span<const Control> controls,
                       const Parameters& parameters, std::size_t start, std::vector<State>& states, std::vector<StepCache>& caches) {
    const std::size_t end = std::min(start + trajectory.checkpoint_interval, controls.size());
    std::size_t slot = 0;
    while (slot < trajectory.checkpoint_steps.size() && trajectory.checkpoint_steps[slot] != start) ++slot;
    if (slot == trajectory.checkpoint_steps.size()) throw std::logic_error("checkpoint missing");
    while (states.size() < end - start + 1) states.push_back(model.allocate_state(context));
    while (caches.size() < end - start) caches.push_back(model.allocate_step_cache(context));
    model.copy_state(trajectory.states[slot], states[0], context);
    for (std::size_t step = start; step < end; ++step)
        model.forward_step(states[step - start], controls[step], parameters, states[step - start + 1], caches[step - start], context);
}

}  // namespace detail

// solver.ixx:53-81; checkpoint_interval is used by TapeMode::checkpoint.
template <typename Model, typename Context, typename State, typename Control, typename Parameters>
    requires ForwardModel<Model, Context, State, Control, Parameters>
[[nodiscard]] auto simulate(const Model& model, Context& context, const State& initial_state, std::span<const Control> controls,
                            const Parameters& parameters, TapeMode tape_mode, std::size_t checkpoint_interval = 0)
    -> Trajectory<State, decltype(model.allocate_step_cache(context))> {
    using StepCache = decltype(model.allocate_step_cache(context));
    Trajectory<State, StepCache> trajectory{.tape_mode = tape_mode, .states = {}, .step_caches = {}};
    State first = model.allocate_state(context);
    model.copy_state(initial_state, first, context);
    if (tape_mode == TapeMode::checkpoint) {
        if (checkpoint_interval == 0) throw std::invalid_argument("checkpoint tape mode needs checkpoint_interval >= 1");
        trajectory.checkpoint_interval = checkpoint_interval;
        trajectory.states.push_back(std::move(first));
        trajectory.checkpoint_steps.push_back(0);
        if (controls.empty()) return trajectory;
        StepCache cache = model.allocate_step_cache(context);
        State work[2] = {model.allocate_state(context), model.allocate_state(context)};
        int w = 0;
        const State* current = &trajectory.states.back();
        for (std::size_t step = 0; step < controls.size(); ++step) {
            State& out = work[w];
            model.forward_step(*current, controls[step], parameters, out, cache, context);
            const std::size_t done = step + 1;
            if (done % checkpoint_interval == 0 || done == controls.size()) {
                State kept = model.allocate_state(context);
                model.copy_state(out, kept, context);
                trajectory.states.push_back(std::move(kept));
                trajectory.checkpoint_steps.push_back(done);
                current = &trajectory.states.back();
            } else {
                current = &out;
                w ^= 1;
            }
        }
        return trajectory;
    }
    trajectory.states.reserve(controls.size() + 1);
    trajectory.states.push_back(std::move(first));
    if (tape_mode == TapeMode::store_all) trajectory.step_caches.reserve(controls.size());
    std::optional<StepCache> reusable;
    if (tape_mode == TapeMode::recompute_step_cache && !controls.empty()) reusable.emplace(model.allocate_step_cache(context));
    for (const Control& control : controls) {
        State next = model.allocate_state(context);
        if (tape_mode == TapeMode::store_all) {
            StepCache cache = model.allocate_step_cache(context);
            model.forward_step(trajectory.states.back(), control, parameters, next, cache, context);
            trajectory.step_caches.push_back(std::move(cache));
        } else {
            model.forward_step(trajectory.states.back(), control, parameters, next, *reusable, context);
        }
        trajectory.states.push_back(std::move(next));
    }
    return trajectory;
}

// solver.ixx:83-113
template <typename Model, typename Context, typename State, typename StepCache, typename Control, typename Parameters>
    requires JvpModel<Model, Context, State, Control, Parameters>
[[nodiscard]] auto jvp(const Model& model, Context& context, const Trajectory<State, StepCache>& trajectory, std::span<const Control> controls,
                       const Parameters& parameters, const decltype(model.allocate_state_tangent(context))& initial_state_tangent,
                       std::span<const decltype(model.allocate_control_tangent(context))> control_tangents,
                       const decltype(model.allocate_parameter_tangent(context))& parameter_tangent)
    -> std::vector<decltype(model.allocate_state_tangent(context))> {
    std::vector<decltype(model.allocate_state_tangent(context))> result;
    result.reserve(controls.size() + 1);
    auto first = model.allocate_state_tangent(context);
    model.copy_state_tangent(initial_state_tangent, first, context);
    result.push_back(std::move(first));
    std::optional<State> rstate;
    std::optional<StepCache> rcache;
    if (trajectory.tape_mode == TapeMode::recompute_step_cache && !controls.empty()) {
        rstate.emplace(model.allocate_state(context));
        rcache.emplace(model.allocate_step_cache(context));
    }
    std::vector<State> seg_states;
    std::vector<StepCache> seg_caches;
    std::size_t seg_start = static_cast<std::size_t>(-1);
    for (std::size_t step = 0; step < controls.size(); ++step) {
        const State* state;
        const State* next;
        const StepCache* cache;
        if (trajectory.tape_mode == TapeMode::store_all) {
            state = &trajectory.states[step];
            next = &trajectory.states[step + 1];
            cache = &trajectory.step_caches[step];
        } else if (trajectory.tape_mode == TapeMode::recompute_step_cache) {
            model.forward_step(trajectory.states[step], controls[step], parameters, *rstate, *rcache, context);
            state = &trajectory.states[step];
            next = &trajectory.states[step + 1];
            cache = &*rcache;
        } else {
            const std::size_t start = step - step % trajectory.checkpoint_interval;
            if (start != seg_start) {
                detail::recompute_segment(model, context, trajectory, controls, parameters, start, seg_states, seg_caches);
                seg_start = start;
            }
            state = &seg_states[step - start];
            next = &seg_states[step - start + 1];
            cache = &seg_caches[step - start];
        }
        auto nt = model.allocate_state_tangent(context);
        model.jvp_step(*state, controls[step], parameters, *next, *cache, result.back(), control_tangents[step], parameter_tangent, nt, context);
        result.push_back(std::move(nt));
    }
    return result;
}

// solver.ixx:115-150.  trajectory_adjoint holds T+1 state adjoints (seeds).
template <typename Model, typename Context, typename State, typename StepCache, typename Control, typename Parameters, typename StateAdjoint>
    requires VjpModel<Model, Context, State, Control, Parameters>
[[nodiscard]] auto vjp(const Model& model, Context& context, const Trajectory<State, StepCache>& trajectory, std::span<const Control> controls,
                       const Parameters& parameters, std::span<const StateAdjoint> trajectory_adjoint)
    -> GradientResult<StateAdjoint, decltype(model.allocate_control_adjoint(context)), decltype(model.allocate_parameter_adjoint(context))> {
    GradientResult<StateAdjoint, decltype(model.allocate_control_adjoint(context)), decltype(model.allocate_parameter_adjoint(context))> result{
        .initial_state = model.allocate_state_adjoint(context), .controls = {}, .parameters = model.allocate_parameter_adjoint(context)};
    result.controls.reserve(controls.size());
    for (std::size_t step = 0; step < controls.size(); ++step) result.controls.push_back(model.allocate_control_adjoint(context));
    StateAdjoint running = model.allocate_state_adjoint(context);
    model.copy_state_adjoint(trajectory_adjoint.back(), running, context);
    std::optional<State> rstate;
    std::optional<StepCache> rcache;
    if (trajectory.tape_mode == TapeMode::recompute_step_cache && !controls.empty()) {
        rstate.emplace(model.allocate_state(context));
        rcache.emplace(model.allocate_step_cache(context));
    }
    std::vector<State> seg_states;
    std::vector<StepCache> seg_caches;
    std::size_t seg_start = static_cast<std::size_t>(-1);
    for (std::size_t step = controls.size(); step-- > 0;) {
        const State* state;
        const State* next;
        const StepCache* cache;
        if (trajectory.tape_mode == TapeMode::store_all) {
            state = &trajectory.states[step];
            next = &trajectory.states[step + 1];
            cache = &trajectory.step_caches[step];
        } else if (trajectory.tape_mode == TapeMode::recompute_step_cache) {
            model.forward_step(trajectory.states[step], controls[step], parameters, *rstate, *rcache, context);
            state = &trajectory.states[step];
            next = &trajectory.states[step + 1];
            cache = &*rcache;
        } else {
            const std::size_t start = step - step % trajectory.checkpoint_interval;
            if (start != seg_start) {
                detail::recompute_segment(model, context, trajectory, controls, parameters, start, seg_states, seg_caches);
                seg_start = start;
            }
            state = &seg_states[step - start];
            next = &seg_states[step - start + 1];
            cache = &seg_caches[step - start];
        }
        StateAdjoint previous = model.allocate_state_adjoint(context);
        model.vjp_step(*state, controls[step], parameters, *next, *cache, running, previous, result.controls[step], result.parameters, context);
        model.accumulate_state_adjoint(trajectory_adjoint[step], previous, context);
        running = std::move(previous);
    }
    result.initial_state = std::move(running);
    return result;
}

}  // namespace xayah::solver
