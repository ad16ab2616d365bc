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
    to 1e-12 in every oracle step).  Agreement to 1e-3 relative (see the
    assertions for directions with small derivatives)."""
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
    got = np.array([sum(float(gi @ di) for gi, di in zip(g, d)) for d in plume_directions(n, fd.size)])
    rels = np.abs(got - fd) / np.abs(fd)
    projected = float(np.linalg.norm(got - fd) / np.linalg.norm(fd))
    from common import report
    report("fd_plume_128", loss=loss, finite_differences=fd.tolist(), vjp=got.tolist(), relative_errors=rels.tolist(),
           projected_relative_error=projected)
    # the gradient projected on the directions agrees to 1e-3 relative L2, and
    # so does each directional derivative of comparable size; a direction
    # whose derivative is far smaller than the largest (the fourth: 11x) is
    # held to the others' absolute error, the FP32 model's noise floor
    # (~5e-7 here against FP64 differences)
    assert projected < 1e-3, (projected, rels)
    large = np.abs(fd) >= 0.25 * np.abs(fd).max()
    assert np.all(rels[large] < 1e-3), rels
    assert np.all(np.abs(got - fd) < 1e-3 * np.abs(fd).max()), (got, fd)


def test_rollout_vjp_matches_the_reference_kernels(cuda):
    """The differentiable plume's rollout differentiated by the reference's
    own kernels (solvers/smoke/operators.cu through oracle/_ref): 128^3, 50
    steps, the reference's solver (red-black sweeps, a fixed count), loss =
    ||rho_50 - target||_2.  The reference side runs its forward steps keeping
    every state and step cache, then chains its vjp_step kernels back to step
    0 (model.cpp:362-389 per step); the product runs its checkpointed VJP
    (every 10 steps, segments recomputed).  The inflow sphere has no
    reference primitive, so density and temperature start as a blob instead
    and the controls are zero.  Gradients with respect to the initial
    velocity and density agree to 1e-4 relative L2."""
    import torch
    from common import differentiable_plume
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    from diff_solver_b200.solver import TapeMode, simulate, vjp
    from oracle import ref_binding as rb
    if not rb.available():
        pytest.skip("reference harness not built")
    n, steps, sweeps = 128, 50, 40
    cfg, u0, target = differentiable_plume(n)
    cfg.inflows = []
    cfg = with_solver_rbgs(cfg, sweeps)
    c = (np.arange(n) + 0.5) / n
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    blob = np.exp(-((X - 0.5) ** 2 + (Y - 0.15) ** 2 + (Z - 0.5) ** 2) / (2 * 0.06 ** 2)).reshape(-1).astype(np.float32)
    dev = torch.device("cuda")
    # product: checkpointed rollout and VJP
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.differentiable)
    params = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    controls = [model.allocate_control(ctx) for _ in range(steps)]
    s0 = model.allocate_state(ctx)
    s0.density.values.copy_(torch.from_numpy(blob))
    s0.temperature.values.copy_(torch.from_numpy(blob))
    for t, v in zip(s0.velocity.components(), u0):
        t.copy_(torch.from_numpy(v).float())
    traj = simulate(model, ctx, s0, controls, params, TapeMode.checkpoint, 10)
    target_d = torch.from_numpy(target).to(dev)
    diff = traj.states[-1].density.values.double() - target_d
    seed = model.allocate_state_adjoint(ctx)
    seed.density.values.copy_(diff / torch.sqrt((diff * diff).sum()))
    grad = vjp(model, ctx, traj, controls, params, {steps: seed})
    got = [t.double() for t in (grad.initial_state.density.values, *grad.initial_state.velocity.components())]
    del traj
    # reference: every state and cache kept, its vjp_step chained backwards
    d = ctx.domain
    ref = rb.Reference(cfg, {"mask": d.cell_mask, "cv": list(d.collider_velocity.components()), "cd": d.collider_density.values,
                             "ct": d.collider_temperature.values, "anchor": d.pressure_anchor}, iterations=sweeps)
    N = n ** 3
    faces = [t.numel() for t in s0.velocity.components()]
    states = [[t.clone() for t in model._state_tensors(s0)]]
    caches = []
    zeros_n = lambda: torch.zeros(N, dtype=torch.float32, device=dev)
    control = [zeros_n() for _ in range(5)]
    rparams = [params.ambient_temperature, params.density_buoyancy, params.temperature_buoyancy, params.vorticity_confinement]
    for _ in range(steps):
        nxt = [torch.empty_like(t) for t in states[-1]]
        cache = [zeros_n(), zeros_n(), zeros_n(), zeros_n(), zeros_n(), torch.zeros((11, N), dtype=torch.float32, device=dev),
                 *[torch.zeros(f, dtype=torch.float32, device=dev) for f in faces], *[torch.zeros(f, dtype=torch.float32, device=dev) for f in faces]]
        ref.forward_step(states[-1], control, rparams, nxt, cache)
        states.append(nxt)
        caches.append(cache)
    rdiff = states[-1][0].double() - target_d
    na = [rdiff / torch.sqrt((rdiff * rdiff).sum())] + [torch.zeros(t.numel(), dtype=torch.float64, device=dev) for t in states[0][1:]]
    for k in range(steps - 1, -1, -1):
        pa = [torch.zeros_like(x) for x in na]
        ca = [torch.zeros(N, dtype=torch.float64, device=dev) for _ in range(5)]
        qa = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(4)]
        ref.vjp_step(states[k], rparams, states[k + 1], caches[k], na, pa, ca, qa)
        na = pa
    torch.cuda.synchronize()
    want = [na[0], na[2], na[3], na[4]]
    errors = [float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) for a, b in zip(got, want)]
    from common import report
    report("rollout_vjp_vs_reference_128", steps=steps, sweeps=sweeps, relative_errors=errors)
    assert max(errors) < 1e-4, errors


def with_solver_rbgs(cfg, sweeps):
    from common import with_solver
    return with_solver(cfg, "rbgs", iterations=sweeps)
