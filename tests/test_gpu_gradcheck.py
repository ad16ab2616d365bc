"""The checkpointed multi-step VJP on the GPU against central finite
differences of the FP64 CPU oracle (the differentiable-plume check at a size
the oracle rolls out in seconds): gradient of sum (rho_T - target)^2 with
respect to the initial velocity along seeded smooth unit directions."""
import numpy as np
import pytest

from common import ROOT  # noqa: F401

pytestmark = pytest.mark.gpu

PARAMS = dict(ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=0.5, vorticity_confinement=0.0)


@pytest.mark.parametrize("steps,interval,directions", [(24, 5, 6), (50, 10, 8)])
def test_checkpointed_vjp_matches_fp64_finite_differences(cuda, steps, interval, directions):
    import torch
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.gradcheck import smooth_direction
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    from diff_solver_b200.solver import TapeMode, simulate, vjp
    from oracle import binding as ob

    # FP64 finite differences allow a step small enough that few trilinear
    # interpolation weights cross a cell boundary between the two rollouts
    # (each crossing is a kink of the discrete map)
    n, eps = 32, 1e-4
    cfg = plume_configuration((n, n, n), inflow_center=(0.5, 0.15, 0.5), inflow_radius=0.15)
    cfg.pressure_tolerance = 1e-11
    cfg.pressure_max_iterations = 20000
    rng = np.random.default_rng(7)
    u0 = [rng.uniform(-0.05, 0.05, s) for s in ((n + 1) * n * n, n * (n + 1) * n, n * n * (n + 1))]
    c = (np.arange(n) + 0.5) / n
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    centre = rng.uniform(0.3, 0.7, 3)
    target = np.exp(-((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2) / (2 * 0.1 ** 2)).reshape(-1)

    # GPU: checkpointed rollout and VJP
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.differentiable)
    params = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    controls = [model.allocate_control(ctx) for _ in range(steps)]
    s0 = model.allocate_state(ctx)
    for t, v in zip(s0.velocity.components(), u0):
        t.copy_(torch.from_numpy(v).float())
    traj = simulate(model, ctx, s0, controls, params, TapeMode.checkpoint, interval)
    seed = model.allocate_state_adjoint(ctx)
    target_d = torch.from_numpy(target).cuda()
    seed.density.values.copy_(2.0 * (traj.states[-1].density.values.double() - target_d))
    grad = vjp(model, ctx, traj, controls, params, {steps: seed})
    g = [t.cpu().numpy() for t in grad.initial_state.velocity.components()]

    # FP64 oracle: central differences
    P = ob.Problem(cfg, "f64", solver="pcg", iterations=20000, tolerance=1e-12)
    ctl = ob.zeros_control(P.res, np.float64)

    def loss(u):
        st = ob.zeros_state(P.res, np.float64)
        for a in range(3):
            st["velocity"][a][:] = u[a]
        for _ in range(steps):
            st, _, stats, _ = P.forward_step(st, ctl, PARAMS)
            assert stats.converged == 1
        d = st["density"] - target
        return float(d @ d)

    shapes = [(n, n, n + 1), (n, n + 1, n), (n + 1, n, n)]
    rels = []
    for _ in range(directions):
        d = [x.reshape(-1) for x in smooth_direction(rng, shapes, n)]
        gd = sum(float(gi @ di) for gi, di in zip(g, d))
        fd = (loss([u + eps * di for u, di in zip(u0, d)]) - loss([u - eps * di for u, di in zip(u0, d)])) / (2 * eps)
        rels.append(abs(fd - gd) / max(abs(fd), 1e-30))
    assert max(rels) < 1e-3, rels
