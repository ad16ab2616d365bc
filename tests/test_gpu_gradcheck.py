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


def test_plume_vjp_matches_oracle_finite_differences(cuda):
    """The differentiable plume as specified (tests/common.py:
    differentiable_plume): 128^3, 50 steps, loss = ||rho_50 - target||_2, the
    gradient with respect to the initial velocity from the checkpointed VJP
    (every 10 steps, recompute in between), against FP64 central finite
    differences (eps = 1e-3) of the CPU oracle along the first seeded unit
    directions, precomputed by tests/golden/make_fd.py (pressure converged
    to 1e-12 in every oracle step).  Agreement to 1e-3 relative."""
    import os

    import torch
    from common import differentiable_plume, plume_directions
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    from diff_solver_b200.solver import TapeMode, simulate, vjp
    path = os.path.join(ROOT, "tests", "golden", "fd_plume_128.npz")
    if not os.path.exists(path):
        pytest.skip("finite-difference fixture not generated (tests/golden/make_fd.py)")
    z = np.load(path)
    fd = np.asarray(z["finite_differences"], np.float64)
    n, steps = int(z["grid"]), int(z["steps"])
    if fd.size < 4:  # make_fd.py keeps partial results in the same file while it runs
        pytest.skip(f"finite-difference fixture incomplete ({fd.size} of 4 directions)")
    cfg, u0, target = differentiable_plume(n)
    cfg.pressure_tolerance = 1e-10
    cfg.pressure_max_iterations = 50000
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.differentiable)
    params = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    controls = [model.allocate_control(ctx) for _ in range(steps)]
    s0 = model.allocate_state(ctx)
    for t, v in zip(s0.velocity.components(), u0):
        t.copy_(torch.from_numpy(v).float())
    traj = simulate(model, ctx, s0, controls, params, TapeMode.checkpoint, 10)
    final = traj.states[-1].density.values.double()
    target_d = torch.from_numpy(target).cuda()
    diff = final - target_d
    loss = float(torch.sqrt((diff * diff).sum()))
    assert abs(loss - float(z["loss"])) <= 1e-5 * float(z["loss"]), (loss, float(z["loss"]))
    seed = model.allocate_state_adjoint(ctx)
    seed.density.values.copy_(diff / loss)
    grad = vjp(model, ctx, traj, controls, params, {steps: seed})
    g = [t.cpu().numpy() for t in grad.initial_state.velocity.components()]
    rels = []
    for d, want in zip(plume_directions(n, fd.size), fd):
        got = sum(float(gi @ di) for gi, di in zip(g, d))
        rels.append(abs(got - want) / abs(want))
    from common import report
    report("fd_plume_128", loss=loss, finite_differences=fd.tolist(), relative_errors=rels)
    assert max(rels) < 1e-3, rels
