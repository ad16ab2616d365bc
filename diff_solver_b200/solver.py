"""Model-agnostic rollout and differentiation: Python mirror of the
reference module ``xayah.solver`` (solvers/solver.ixx:7-150).

``simulate`` / ``jvp`` / ``vjp`` keep the reference's signatures and
semantics for the two reference tape modes (store every step cache, or
recompute each step's cache from the stored states).  The checkpoint tape
mode is an addition: only every k-th state is kept; the reverse pass
recomputes one segment of k steps forward (states and caches into a k-slot
buffer) and then runs that segment's VJP steps backwards.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Union


class TapeMode(enum.Enum):
    store_all = 0             # solver.ixx:8
    recompute_step_cache = 1  # solver.ixx:9
    checkpoint = 2            # addition: keep states at multiples of k


@dataclass
class Trajectory:
    """solver.ixx:12-17.  In checkpoint mode ``states`` holds the states at
    steps 0, k, 2k, ... and the final one; ``checkpoint_steps`` lists their
    step indices."""
    tape_mode: TapeMode
    states: list
    step_caches: list = field(default_factory=list)
    checkpoint_interval: int = 0
    checkpoint_steps: List[int] = field(default_factory=list)
    steps: int = 0

    def state_at(self, step: int):
        if self.tape_mode != TapeMode.checkpoint:
            return self.states[step]
        return self.states[self.checkpoint_steps.index(step)]


@dataclass
class GradientResult:
    """solver.ixx:19-24"""
    initial_state: object
    controls: list
    parameters: object


def simulate(model, context, initial_state, controls: Sequence, parameters, tape_mode: TapeMode = TapeMode.store_all,
             checkpoint_interval: int = 0) -> Trajectory:
    """solver.ixx:53-81"""
    traj = Trajectory(tape_mode=tape_mode, states=[], steps=len(controls))
    first = model.allocate_state(context)
    model.copy_state(initial_state, first, context)
    if tape_mode == TapeMode.checkpoint:
        if checkpoint_interval < 1:
            raise ValueError("checkpoint tape mode needs checkpoint_interval >= 1")
        traj.checkpoint_interval = checkpoint_interval
        traj.states.append(first)
        traj.checkpoint_steps.append(0)
        cache = model.allocate_step_cache(context) if controls else None
        work = [model.allocate_state(context), model.allocate_state(context)] if controls else []
        w = 0
        current = first
        for step, control in enumerate(controls):
            out = work[w]
            model.forward_step(current, control, parameters, out, cache, context)
            done = step + 1
            if done % checkpoint_interval == 0 or done == len(controls):
                kept = model.allocate_state(context)
                model.copy_state(out, kept, context)
                traj.states.append(kept)
                traj.checkpoint_steps.append(done)
                current = kept
            else:
                current = out
                w ^= 1
        return traj
    traj.states.append(first)
    reusable = model.allocate_step_cache(context) if (tape_mode == TapeMode.recompute_step_cache and controls) else None
    for control in controls:
        nxt = model.allocate_state(context)
        if tape_mode == TapeMode.store_all:
            cache = model.allocate_step_cache(context)
            model.forward_step(traj.states[-1], control, parameters, nxt, cache, context)
            traj.step_caches.append(cache)
        else:
            model.forward_step(traj.states[-1], control, parameters, nxt, reusable, context)
        traj.states.append(nxt)
    return traj


def _segment(model, context, traj: Trajectory, controls, parameters, start: int, pool=None):
    """Recompute the checkpoint segment beginning at ``start``: returns the
    states start..end and the caches of steps start..end-1.  ``pool`` (states,
    caches; at least one segment's worth) supplies the buffers, reused from
    segment to segment: every step overwrites its state and cache."""
    end = min(start + traj.checkpoint_interval, traj.steps)
    states = [traj.state_at(start)]
    caches = []
    for i, step in enumerate(range(start, end)):
        nxt = pool[0][i] if pool else model.allocate_state(context)
        cache = pool[1][i] if pool else model.allocate_step_cache(context)
        model.forward_step(states[-1], controls[step], parameters, nxt, cache, context)
        states.append(nxt)
        caches.append(cache)
    return states, caches


def jvp(model, context, trajectory: Trajectory, controls: Sequence, parameters, initial_state_tangent, control_tangents: Sequence,
        parameter_tangent) -> list:
    """solver.ixx:83-113.  Returns the T+1 state tangents."""
    result = []
    first = model.allocate_state_tangent(context)
    model.copy_state_tangent(initial_state_tangent, first, context)
    result.append(first)
    mode = trajectory.tape_mode
    rstate = model.allocate_state(context) if (mode == TapeMode.recompute_step_cache and controls) else None
    rcache = model.allocate_step_cache(context) if (mode == TapeMode.recompute_step_cache and controls) else None
    seg_states, seg_caches, seg_start = None, None, -1
    for step in range(len(controls)):
        if mode == TapeMode.store_all:
            state, nxt, cache = trajectory.states[step], trajectory.states[step + 1], trajectory.step_caches[step]
        elif mode == TapeMode.recompute_step_cache:
            model.forward_step(trajectory.states[step], controls[step], parameters, rstate, rcache, context)
            state, nxt, cache = trajectory.states[step], trajectory.states[step + 1], rcache
        else:
            start = step - step % trajectory.checkpoint_interval
            if start != seg_start:
                seg_states, seg_caches = _segment(model, context, trajectory, controls, parameters, start)
                seg_start = start
            state, nxt, cache = seg_states[step - start], seg_states[step - start + 1], seg_caches[step - start]
        nt = model.allocate_state_tangent(context)
        model.jvp_step(state, controls[step], parameters, nxt, cache, result[-1], control_tangents[step], parameter_tangent, nt, context)
        result.append(nt)
    return result


def _seed(trajectory_adjoint, step):
    if isinstance(trajectory_adjoint, dict):
        return trajectory_adjoint.get(step)
    return trajectory_adjoint[step]


def vjp(model, context, trajectory: Trajectory, controls: Sequence, parameters,
        trajectory_adjoint: Union[Sequence, Dict[int, object]], after_step=None) -> GradientResult:
    """solver.ixx:115-150.  ``trajectory_adjoint`` holds one state adjoint per
    state (T+1 entries, as in the reference); it may also be a dict
    {step: adjoint} or contain None for steps without a seed.  ``after_step``
    (an addition, optional) is called with the step index right after that
    step's vjp_step has been enqueued (for instance to copy the adjoint
    solve's statistics without synchronising)."""
    T = len(controls)
    result = GradientResult(initial_state=model.allocate_state_adjoint(context),
                            controls=[model.allocate_control_adjoint(context) for _ in range(T)],
                            parameters=model.allocate_parameter_adjoint(context))
    running = model.allocate_state_adjoint(context)
    last = _seed(trajectory_adjoint, T)
    if last is not None:
        model.copy_state_adjoint(last, running, context)
    mode = trajectory.tape_mode
    rstate = model.allocate_state(context) if (mode == TapeMode.recompute_step_cache and controls) else None
    rcache = model.allocate_step_cache(context) if (mode == TapeMode.recompute_step_cache and controls) else None
    spare = model.allocate_state_adjoint(context)
    seg_states, seg_caches, seg_start = None, None, -1
    pool = None
    if mode == TapeMode.checkpoint and controls:
        k = min(trajectory.checkpoint_interval, T)
        pool = ([model.allocate_state(context) for _ in range(k)], [model.allocate_step_cache(context) for _ in range(k)])
    for step in range(T - 1, -1, -1):
        if mode == TapeMode.store_all:
            state, nxt, cache = trajectory.states[step], trajectory.states[step + 1], trajectory.step_caches[step]
        elif mode == TapeMode.recompute_step_cache:
            model.forward_step(trajectory.states[step], controls[step], parameters, rstate, rcache, context)
            state, nxt, cache = trajectory.states[step], trajectory.states[step + 1], rcache
        else:
            start = step - step % trajectory.checkpoint_interval
            if start != seg_start:
                seg_states, seg_caches = _segment(model, context, trajectory, controls, parameters, start, pool)
                seg_start = start
            state, nxt, cache = seg_states[step - start], seg_states[step - start + 1], seg_caches[step - start]
        model.zero_state_adjoint(spare, context)
        model.vjp_step(state, controls[step], parameters, nxt, cache, running, spare, result.controls[step], result.parameters, context)
        if after_step is not None:
            after_step(step)
        seed = _seed(trajectory_adjoint, step)
        if seed is not None:
            model.accumulate_state_adjoint(seed, spare, context)
        running, spare = spare, running
    model.copy_state_adjoint(running, result.initial_state, context)
    return result
