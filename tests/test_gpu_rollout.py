"""Per-step parity of whole rollouts at the benchmark's sizes.

* The 64^3 plume (100 steps from rest with seeded velocity noise, pressure by
  Jacobi-PCG to a 1e-6 relative residual) and a 30-step 128^3 rollout of the
  learned pipeline: every 10th step of the product's own rollout is
  recomputed from the same input state by the FP64 CPU oracle (pressure
  converged to 1e-12) and by the reference's own kernels
  (solvers/smoke/operators.cu through oracle/_ref, model.cpp:341-349 order,
  red-black Gauss-Seidel iterated until the FP32 sweeps stop lowering the
  residual: about 3e-6 relative at 64^3, 1e-5 at 128^3).  Density, temperature and
  velocity must agree to 1e-5 relative L2.
  Run with the plain zero start, the classical warm start (ring of previous
  solutions, coarse-grid step) and the benchmark's learned pipeline.
* The 256^3 headline pipeline (float4 fast paths, three-level coarse start,
  network step, smoothed PCG): one step after a 30-step rollout against the
  FP64 oracle's step from the same state.

Measured errors are appended to $XS_PARITY_REPORT when it is set.
"""
import os

import numpy as np
import pytest

from common import (PLUME_PARAMS, ROOT, field_errors, from_model_state, product_domain, reference_step, report,  # noqa: F401
                    seeded_control, to_model_state)

from oracle import binding as ob

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(ROOT, "diff_solver_b200", "weights", "warm_start_128.npz")


def plume(n, history=0, coarsening=0, tolerance=1e-6):
    from diff_solver_b200.data import plume_configuration
    cfg = plume_configuration((n, n, n), inflow_center=(0.5, 0.1, 0.5), inflow_radius=0.08)
    cfg.pressure_tolerance = tolerance
    cfg.pressure_max_iterations = 20000
    cfg.warm_start_history = history
    cfg.warm_start_coarsening = coarsening
    return cfg


def rollout_context(cfg, learned, factor=2):
    import torch
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.forward)
    network = None
    if learned:
        from diff_solver_b200.warm_start import WarmStartNetwork
        network = WarmStartNetwork(tuple(int(v) // factor for v in cfg.resolution), factor=factor)
        network.load(WEIGHTS)
        ctx.set_learned_warm_start(network)
    params = fill_parameters(model.allocate_parameters(ctx), **PLUME_PARAMS)
    control = model.allocate_control(ctx)
    n = int(np.prod(cfg.resolution))
    rng = np.random.default_rng(0)
    f = [(cfg.resolution[0] + 1) * cfg.resolution[1] * cfg.resolution[2], cfg.resolution[0] * (cfg.resolution[1] + 1) * cfg.resolution[2],
         cfg.resolution[0] * cfg.resolution[1] * (cfg.resolution[2] + 1)]
    start = {"density": np.zeros(n), "temperature": np.zeros(n), "velocity": [rng.uniform(-0.01, 0.01, k) for k in f]}
    state = to_model_state(model, ctx, start)
    torch.cuda.synchronize()
    return model, ctx, network, params, control, state


# (grid, start, steps, check every): the plain zero start; the classical
# warm start (ring of previous solutions + coarse-grid step); the full
# learned pipeline (the network runs at factor 1 on 128^3: on a 32^3 network
# grid its coarsest level is smaller than one convolution tile).
ROLLOUTS = [(64, "plain", 100, 10), (64, "history+coarse", 100, 10), (128, "learned+history+coarse", 30, 10)]


@pytest.mark.parametrize("n,start,steps,every", ROLLOUTS)
def test_plume_rollout_matches_oracle_and_reference_kernels(cuda, n, start, steps, every):
    import torch
    warm = start != "plain"
    learned = start.startswith("learned")
    cfg = plume(n, history=5 if warm else 0, coarsening=2 if warm else 0)
    model, ctx, network, params, control, cur = rollout_context(cfg, learned=learned, factor=1 if n <= 128 else 4)
    nxt = model.allocate_state(ctx)
    cache = model.allocate_step_cache(ctx)
    zero_control = ob.zeros_control(tuple(cfg.resolution), np.float64)
    ob.set_threads(os.cpu_count() or 1)
    P = ob.Problem(plume(n), "f64", solver="pcg", iterations=50000, tolerance=1e-12)
    worst = {"oracle": 0.0, "reference": 0.0}
    for step in range(steps):
        check = step % every == every - 1
        if check:
            before = from_model_state(model, cur)
        model.forward_step(cur, control, params, nxt, cache, ctx)
        if check:
            torch.cuda.synchronize()
            stats = ctx.read_solve_stats()
            assert stats["status"] == 0 and stats["final_residual"] <= 1e-6, stats
            got = from_model_state(model, nxt)
            want, _, ost, _ = P.forward_step(before, zero_control, PLUME_PARAMS, guess=ctx.pressure_fields()[0].double().cpu().numpy())
            assert ost.converged == 1
            ref, sweeps, residual = reference_step(plume(n), product_domain(ctx), before, zero_control, PLUME_PARAMS, tolerance=1e-9)
            e_oracle, e_ref = field_errors(got, want), field_errors(got, ref)
            report(f"rollout{n}_{start}", step=step + 1, oracle=e_oracle, reference=e_ref, reference_sweeps=sweeps,
                   reference_residual=residual, product_iterations=stats["iterations"], product_residual=stats["final_residual"],
                   warm_start_used=stats["warm_start_used"])
            # the reference's FP32 sweeps stop at their rounding floor (the
            # stall test of the harness: ~3e-6 relative at 64^3, ~1e-5 at
            # 128^3); that they got there and not stuck early is checked here,
            # the fields below
            assert residual < 3e-5, (step, sweeps, residual)
            for name, e in (("oracle", e_oracle), ("reference", e_ref)):
                for field, v in e.items():
                    assert v < 1e-5, (start, step + 1, name, field, v)
                worst[name] = max(worst[name], *e.values())
        cur, nxt = nxt, cur
    if network is not None:
        network.check()
    report(f"rollout{n}_{start}_worst", **worst)


def test_headline_pipeline_step_at_256_matches_fp64_oracle(cuda):
    import torch
    cfg = plume(256, history=5, coarsening=2)
    # the benchmark's network: trained at 128^3, run on the grid restricted x4
    model, ctx, network, params, control, cur = rollout_context(cfg, learned=True, factor=4)
    nxt = model.allocate_state(ctx)
    cache = model.allocate_step_cache(ctx)
    for _ in range(30):
        model.forward_step(cur, control, params, nxt, cache, ctx)
        cur, nxt = nxt, cur
    before = from_model_state(model, cur)
    model.forward_step(cur, control, params, nxt, cache, ctx)
    torch.cuda.synchronize()
    stats = ctx.read_solve_stats()
    assert stats["status"] == 0 and stats["final_residual"] <= 1e-6 and stats["warm_start_used"] == 1, stats
    got = from_model_state(model, nxt)
    pressure = ctx.pressure_fields()[0].double().cpu().numpy()
    network.check()
    ob.set_threads(os.cpu_count() or 1)
    P = ob.Problem(plume(256), "f64", solver="pcg", iterations=50000, tolerance=1e-10)
    want, _, ost, _ = P.forward_step(before, ob.zeros_control(tuple(cfg.resolution), np.float64), PLUME_PARAMS, guess=pressure)
    assert ost.converged == 1
    e = field_errors(got, want)
    report("headline256_step", step=31, oracle=e, product_iterations=stats["iterations"], coarse_iterations=stats["coarse_iterations"],
           product_residual=stats["final_residual"], oracle_iterations=ost.iterations)
    for field, v in e.items():
        assert v < 1e-5, (field, v)
