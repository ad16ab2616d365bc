"""The model-agnostic rollout and differentiation drivers on the CPU (no
GPU): the C++ templates of include/xayah/solver.hpp and their Python mirror
diff_solver_b200/solver.py, each driven by a small differentiable toy model.

Every tape mode (store every cache, recompute each cache, checkpoint every k
steps) must reproduce the store-all rollout, tangents and gradients bit for
bit, recompute each step once on the reverse pass, and give the transpose of
the tangent map; the gradient must match central differences."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from diff_solver_b200.solver import TapeMode, jvp, simulate, vjp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_solver_templates_on_a_cpu_model():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    out_dir = os.path.join(ROOT, "tests", "cpp", "_build")
    os.makedirs(out_dir, exist_ok=True)
    exe = os.path.join(out_dir, "solver_host")
    src = os.path.join(ROOT, "tests", "cpp", "solver_host.cpp")
    build = subprocess.run([gxx, "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    assert "ok" in run.stdout


class ToyModel:
    """x' = tanh(W x) + theta u; the step cache holds W x, and the tangent
    and adjoint steps read the nonlinearity's derivative from it only."""

    def __init__(self, n, rng):
        self.n = n
        self.w = rng.normal(0.0, 0.6, (n, n))
        self.forward_steps = 0

    def allocate_state(self, ctx):
        return np.zeros(self.n)

    allocate_state_tangent = allocate_control_tangent = allocate_state_adjoint = allocate_control_adjoint = allocate_state

    def allocate_parameter_adjoint(self, ctx):
        return np.zeros(1)

    allocate_parameter_tangent = allocate_parameter_adjoint

    def allocate_step_cache(self, ctx):
        return np.zeros(self.n)

    def copy_state(self, a, b, ctx):
        b[:] = a

    copy_state_tangent = copy_state_adjoint = copy_state

    def zero_state_adjoint(self, a, ctx):
        a[:] = 0.0

    def accumulate_state_adjoint(self, a, b, ctx):
        b += a

    def forward_step(self, x, u, theta, y, cache, ctx):
        self.forward_steps += 1
        cache[:] = self.w @ x
        y[:] = np.tanh(cache) + theta[0] * u

    def jvp_step(self, x, u, theta, y, cache, dx, du, dtheta, dy, ctx):
        dy[:] = (1.0 - np.tanh(cache) ** 2) * (self.w @ dx) + dtheta[0] * u + theta[0] * du

    def vjp_step(self, x, u, theta, y, cache, next_adj, prev_adj, u_adj, theta_adj, ctx):
        prev_adj += self.w.T @ (next_adj * (1.0 - np.tanh(cache) ** 2))
        u_adj += theta[0] * next_adj
        theta_adj[0] += next_adj @ u


def _problem(n=6, steps=7):
    rng = np.random.default_rng(7)
    m = ToyModel(n, rng)
    x0 = rng.normal(size=n)
    theta = np.array([0.7])
    u = [rng.normal(0.0, 0.5, n) for _ in range(steps)]
    du = [rng.normal(size=n) for _ in range(steps)]
    seeds = [rng.normal(size=n) for _ in range(steps + 1)]
    return m, x0, theta, u, du, seeds, rng.normal(size=n), np.array([0.3])


MODES = [(TapeMode.recompute_step_cache, 0)] + [(TapeMode.checkpoint, k) for k in (1, 2, 3, 7, 10)]


@pytest.mark.parametrize("mode,k", MODES)
def test_python_tape_modes_reproduce_store_all(mode, k):
    m, x0, theta, u, du, seeds, dx0, dth = _problem()
    ref = simulate(m, None, x0, u, theta, TapeMode.store_all)
    ref_tan = jvp(m, None, ref, u, theta, dx0, du, dth)
    ref_grad = vjp(m, None, ref, u, theta, seeds)
    m.forward_steps = 0
    tr = simulate(m, None, x0, u, theta, mode, k)
    assert m.forward_steps == len(u)
    if mode == TapeMode.checkpoint:
        assert tr.checkpoint_steps == list(range(0, len(u), k)) + [len(u)]
        assert len(tr.states) == len(tr.checkpoint_steps) and not tr.step_caches
        assert np.array_equal(tr.states[-1], ref.states[-1])
    else:
        assert all(np.array_equal(a, b) for a, b in zip(tr.states, ref.states))
    tan = jvp(m, None, tr, u, theta, dx0, du, dth)
    assert all(np.array_equal(a, b) for a, b in zip(tan, ref_tan))
    m.forward_steps = 0
    grad = vjp(m, None, tr, u, theta, seeds)
    assert m.forward_steps == len(u)  # each step recomputed once on the reverse pass
    assert np.array_equal(grad.initial_state, ref_grad.initial_state)
    assert np.array_equal(grad.parameters, ref_grad.parameters)
    assert all(np.array_equal(a, b) for a, b in zip(grad.controls, ref_grad.controls))


def test_python_gradient_is_the_transpose_of_the_tangent_map_and_matches_differences():
    m, x0, theta, u, du, seeds, dx0, dth = _problem()
    tr = simulate(m, None, x0, u, theta, TapeMode.checkpoint, 3)
    tan = jvp(m, None, tr, u, theta, dx0, du, dth)
    grad = vjp(m, None, tr, u, theta, seeds)
    lhs = sum(s @ t for s, t in zip(seeds, tan))
    rhs = grad.initial_state @ dx0 + grad.parameters[0] * dth[0] + sum(g @ d for g, d in zip(grad.controls, du))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)

    def objective(s):
        t = simulate(m, None, x0 + s * dx0, [a + s * b for a, b in zip(u, du)], theta + s * dth, TapeMode.store_all)
        return sum(w @ x for w, x in zip(seeds, t.states))
    eps = 1e-6
    fd = (objective(eps) - objective(-eps)) / (2 * eps)
    assert abs(fd - rhs) <= 1e-7 * abs(rhs)


def test_python_sparse_seeds_and_step_callback():
    m, x0, theta, u, du, seeds, dx0, dth = _problem()
    T = len(u)
    tr = simulate(m, None, x0, u, theta, TapeMode.checkpoint, 2)
    dense = [np.zeros_like(s) for s in seeds]
    dense[T], dense[3] = seeds[T], seeds[3]
    calls = []
    sparse = vjp(m, None, tr, u, theta, {T: seeds[T], 3: seeds[3]}, after_step=calls.append)
    full = vjp(m, None, tr, u, theta, dense)
    assert calls == list(range(T - 1, -1, -1))
    assert np.array_equal(sparse.initial_state, full.initial_state)
    assert all(np.array_equal(a, b) for a, b in zip(sparse.controls, full.controls))
    with pytest.raises(ValueError):
        simulate(m, None, x0, u, theta, TapeMode.checkpoint, 0)
