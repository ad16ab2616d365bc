"""Learned pressure warm start on the GPU: the native network's forward pass,
loss and parameter gradient against the CPU reference network (PyTorch FP32
autograd with the GPU's BF16 storage points), restriction / prolongation,
Adam training, the energy-scaled PCG start with its zero-guess fallback, and
the network inside a model step."""
import os

import numpy as np
import pytest

from common import ROOT  # noqa: F401  (puts the repository on sys.path)

pytestmark = pytest.mark.gpu

SHAPE = (128, 64, 16)  # smallest grid whose coarsest level still tiles by 128 voxels


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def smooth_field(rng, shape, batch):
    """Random fields with large-scale structure (a sum of a few Gaussians plus noise)."""
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.linspace(0, 1, nz), np.linspace(0, 1, ny), np.linspace(0, 1, nx), indexing="ij")
    out = np.zeros((batch, nz, ny, nx), np.float32)
    for b in range(batch):
        for _ in range(4):
            c = rng.uniform(0.2, 0.8, 3)
            s = rng.uniform(0.05, 0.2)
            out[b] += rng.normal() * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
        out[b] += 0.05 * rng.normal(size=(nz, ny, nx))
    return out


@pytest.fixture(scope="module")
def net_and_data(cuda):
    import torch
    from diff_solver_b200.warm_start import WarmStartNetwork
    rng = np.random.default_rng(3)
    rhs = smooth_field(rng, SHAPE, 2)
    p = smooth_field(rng, SHAPE, 2)
    net = WarmStartNetwork(SHAPE, max_batch=2, factor=2, seed=11)
    return net, rhs, p, torch.from_numpy(rhs).cuda().reshape(-1), torch.from_numpy(p).cuda().reshape(-1)


def test_parameter_layout_matches_reference(net_and_data):
    from oracle import unet_reference as R
    net = net_and_data[0]
    assert net.parameter_count() == R.parameter_count()
    params = net.parameters()
    w = R.split_parameters(params)
    # initialisation: unused input channels of the first layer and unused
    # output channels of the last one start (and stay) at zero
    assert np.all(w[0][:, :, 2:] == 0) and np.all(w[11][:, 1:, :] == 0)
    assert all(np.std(x) > 0 for x in w)


def test_forward_matches_reference(net_and_data):
    import torch
    from oracle import unet_reference as R
    net, rhs, _, rhs_d, _ = net_and_data
    got = net.predict(rhs_d).cpu().numpy().reshape(rhs.shape)
    torch.cuda.synchronize()
    net.check()
    want = R.predict(net.parameters(), rhs)
    assert rel(got, want) < 2e-2


def test_loss_and_gradient_match_reference(net_and_data):
    from oracle import unet_reference as R
    net, rhs, p, rhs_d, p_d = net_and_data
    loss, grad = net.gradient(rhs_d, p_d)
    net.check()
    want_loss, want_grad = R.loss_and_gradient(net.parameters(), rhs, p)
    assert abs(float(loss.item()) - want_loss) / want_loss < 1e-2
    got = grad.cpu().numpy()
    assert rel(got, want_grad) < 3e-2
    off = 0
    for i, (ci, co, _) in enumerate(R.LAYERS):
        n = 27 * ci * co
        g, w = got[off:off + n], want_grad[off:off + n]
        if i == 0:  # only input channels 0 and 1 carry data
            g, w = g.reshape(27, co, ci)[:, :, :2], w.reshape(27, co, ci)[:, :, :2]
        if i == len(R.LAYERS) - 1:  # only output channel 0 is in the loss
            g, w = g.reshape(27, co, ci)[:, :1], w.reshape(27, co, ci)[:, :1]
        assert rel(g, w) < 5e-2, (i, rel(g, w))
        off += n


@pytest.mark.parametrize("modes", [(1, 1, 1, 0, 1, 1), (2, 2, 0, 1, 2, 2)])
def test_energy_loss_and_gradient_match_reference(cuda, modes):
    """The energy (A-norm) loss: plume boundaries (open top) and a periodic
    variant, against autograd through the reference operator."""
    import torch
    from diff_solver_b200 import _native as N
    from diff_solver_b200.warm_start import WarmStartNetwork
    from oracle import unet_reference as R
    rng = np.random.default_rng(21)
    rhs = smooth_field(rng, SHAPE, 2)
    p = smooth_field(rng, SHAPE, 2)
    net = WarmStartNetwork(SHAPE, max_batch=2, seed=5)
    pb = N.XsScalarBoundary()
    pb.modes[:] = list(modes)
    net.set_loss("energy", pb)
    loss, grad = net.gradient(torch.from_numpy(rhs).cuda().reshape(-1), torch.from_numpy(p).cuda().reshape(-1))
    net.check()
    want_loss, want_grad = R.loss_and_gradient(net.parameters(), rhs, p, kind="energy", modes=modes)
    assert 0.0 <= want_loss <= 1.0
    assert abs(float(loss.item()) - want_loss) < 1e-2 * max(want_loss, 1e-3)
    assert rel(grad.cpu().numpy(), want_grad) < 3e-2


def test_guess_restricts_and_prolongs(net_and_data):
    import torch
    from diff_solver_b200 import _native as N
    from oracle import unet_reference as R
    net = net_and_data[0]
    rng = np.random.default_rng(5)
    fine_shape = tuple(2 * s for s in SHAPE)
    fine = smooth_field(rng, fine_shape, 1)[0]
    grid = N.XsGrid(*fine_shape, 1.0 / fine_shape[0], 0.5 / fine_shape[0])
    got = net.guess(grid, torch.from_numpy(fine).cuda().reshape(-1)).cpu().numpy().reshape(fine.shape)
    coarse = R.restrict(fine.astype(np.float64), 2).astype(np.float32)
    want = R.prolong(R.predict(net.parameters(), coarse[None])[0], 2)
    assert rel(got, want) < 2e-2


def test_adam_reduces_the_loss(cuda):
    import torch
    from diff_solver_b200.warm_start import WarmStartNetwork
    rng = np.random.default_rng(9)
    rhs = torch.from_numpy(smooth_field(rng, SHAPE, 2)).cuda().reshape(-1)
    p = torch.from_numpy(smooth_field(rng, SHAPE, 2)).cuda().reshape(-1)
    net = WarmStartNetwork(SHAPE, max_batch=2, seed=1)
    losses = [float(net.train_step(rhs, p, 1e-3).item()) for _ in range(40)]
    net.check()
    assert all(np.isfinite(losses))
    assert losses[-1] < 0.6 * losses[0], losses[::8]


def _plume_problem(res=(32, 32, 32), steps=12):
    """A developed plume's pressure problem: the model, its context and the
    right-hand side of its last solve."""
    import torch
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    cfg = plume_configuration(res)
    m = Model(cfg)
    ctx = m.allocate_context(ExecutionMode.forward)
    s, n = m.allocate_state(ctx), m.allocate_state(ctx)
    c, k = m.allocate_control(ctx), m.allocate_step_cache(ctx)
    q = fill_parameters(m.allocate_parameters(ctx), 0.0, -0.1, 0.5)
    g = torch.Generator().manual_seed(0)
    for t in s.velocity.components():
        t.copy_((torch.rand(t.shape, generator=g) * 0.02 - 0.01).cuda())
    for _ in range(steps):
        m.forward_step(s, c, q, n, k, ctx)
        s, n = n, s
    p, b = ctx.pressure_fields()
    return m, ctx, p.clone(), b.clone()


def test_energy_scaled_guess_and_fallback(cuda):
    import torch
    from diff_solver_b200.warm_start import solve_iterations
    m, ctx, p, b = _plume_problem()
    plain = solve_iterations(m, ctx, b, None)
    assert plain["status"] == 0 and plain["iterations"] > 10
    # a multiple of the solution: alpha undoes the factor, nothing left to do
    st = solve_iterations(m, ctx, b, 2.5 * p)
    assert st["warm_start_used"] == 1 and abs(st["guess_scale"] - 0.4) < 1e-3
    assert st["iterations"] <= 0.25 * plain["iterations"] and st["final_residual"] <= 1e-6
    # unscaled, the same guess is worse than zero and is dropped
    st = solve_iterations(m, ctx, b, 2.5 * p, scale=False)
    assert st["warm_start_used"] == 0 and st["guess_scale"] == 0.0 and st["final_residual"] <= 1e-6
    # noise: scaled towards zero, never worse than the zero guess in the A-norm
    noise = torch.randn(b.numel(), device=b.device, generator=torch.Generator(device=b.device).manual_seed(2))
    st = solve_iterations(m, ctx, b, noise)
    assert st["status"] == 0 and st["final_residual"] <= 1e-6 and abs(st["guess_scale"]) < 0.1


def _rollout(cfg, steps, network=None, seed=0):
    import torch
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    m = Model(cfg)
    ctx = m.allocate_context(ExecutionMode.forward)
    if network is not None:
        ctx.set_learned_warm_start(network)
    s, n = m.allocate_state(ctx), m.allocate_state(ctx)
    c, k = m.allocate_control(ctx), m.allocate_step_cache(ctx)
    q = fill_parameters(m.allocate_parameters(ctx), 0.0, -0.1, 0.5)
    g = torch.Generator().manual_seed(seed)
    for t in s.velocity.components():
        t.copy_((torch.rand(t.shape, generator=g) * 0.02 - 0.01).cuda())
    stats = []
    for _ in range(steps):
        m.forward_step(s, c, q, n, k, ctx)
        s, n = n, s
        stats.append(ctx.read_solve_stats())
    vel = torch.cat([t.reshape(-1) for t in s.velocity.components()]).cpu().numpy()
    return vel, stats, ctx


def test_galerkin_history_start(cuda):
    """Previous solutions as a Galerkin start: same steps within the solver
    tolerance, far fewer iterations once the ring holds solutions, and a
    reset ring starts from zero again."""
    from diff_solver_b200.data import plume_configuration
    cfg = plume_configuration((64, 64, 64))
    plain, plain_stats, _ = _rollout(cfg, 24)
    cfg.warm_start_history = 4
    warm, warm_stats, ctx = _rollout(cfg, 24)
    assert all(s["status"] == 0 and s["final_residual"] <= 1e-6 for s in warm_stats)
    assert warm_stats[0]["iterations"] == plain_stats[0]["iterations"]  # empty ring: zero start
    late_plain = np.mean([s["iterations"] for s in plain_stats[8:]])
    late_warm = np.mean([s["iterations"] for s in warm_stats[8:]])
    assert late_warm < 0.6 * late_plain, (late_warm, late_plain)
    assert rel(warm, plain) < 1e-4
    ctx.reset_warm_start()


def test_adjoint_solves_start_from_their_own_history(cuda):
    """A differentiable context with a ring also starts the adjoint pressure
    solves of a reverse pass from previous adjoint solutions (and, with
    coarsening, from their coarse-grid correction): the gradient agrees with
    the zero-start one within the solver tolerance and the last adjoint solve
    needs fewer iterations."""
    import torch
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    from diff_solver_b200.solver import TapeMode, simulate, vjp
    out = {}
    for history, coarsening in ((0, 0), (4, 0), (4, 4)):
        cfg = plume_configuration((64, 64, 64))
        cfg.warm_start_history = history
        cfg.warm_start_coarsening = coarsening
        m = Model(cfg)
        ctx = m.allocate_context(ExecutionMode.differentiable)
        q = fill_parameters(m.allocate_parameters(ctx), 0.0, -0.1, 0.5)
        controls = [m.allocate_control(ctx) for _ in range(12)]
        s0 = m.allocate_state(ctx)
        g = torch.Generator().manual_seed(0)
        for t in s0.velocity.components():
            t.copy_((torch.rand(t.shape, generator=g) * 0.02 - 0.01).cuda())
        traj = simulate(m, ctx, s0, controls, q, TapeMode.store_all)
        seed = m.allocate_state_adjoint(ctx)
        seed.density.values.copy_(traj.states[-1].density.values.double())
        grad = vjp(m, ctx, traj, controls, q, {12: seed})
        last = ctx.read_solve_stats()
        assert last["status"] == 0 and last["final_residual"] <= 1e-6
        out[(history, coarsening)] = (torch.cat([t.reshape(-1) for t in grad.initial_state.velocity.components()]).cpu().numpy(),
                                      last["iterations"], last["coarse_iterations"])
    assert rel(out[(4, 0)][0], out[(0, 0)][0]) < 1e-3
    assert out[(4, 0)][1] < out[(0, 0)][1], (out[(4, 0)][1], out[(0, 0)][1])
    # with the coarse-grid step the adjoint solves start from the ring's start
    # corrected on the 16^3 grid (solved exactly: the plume's operator
    # separates, no coarse CG iterations): the same gradient, fewer
    # iterations than the ring alone
    assert rel(out[(4, 4)][0], out[(0, 0)][0]) < 1e-3
    assert out[(4, 4)][2] == 0 and out[(4, 4)][1] < out[(4, 0)][1], (out[(4, 4)][1:], out[(4, 0)][1:])


def test_coarse_grid_correction(cuda):
    """The coarse-grid correction of the history start: the same steps within
    the solver tolerance and far fewer fine iterations than the history start
    alone once the plume has developed (the smooth error the correction
    removes is what keeps CG on its residual plateau).  The plume's operator
    separates (open top, no anchor): its coarse grid is solved exactly and
    reports no coarse CG iterations."""
    from diff_solver_b200.data import plume_configuration
    cfg = plume_configuration((128, 128, 128))
    cfg.warm_start_history = 5
    hist, hist_stats, _ = _rollout(cfg, 50)
    cfg.warm_start_coarsening = 4
    coarse, coarse_stats, _ = _rollout(cfg, 50)
    assert all(s["status"] == 0 and s["final_residual"] <= 1e-6 for s in coarse_stats)
    assert rel(coarse, hist) < 1e-4
    assert all(s["coarse_iterations"] == 0 for s in hist_stats + coarse_stats)
    late_hist = np.mean([s["iterations"] for s in hist_stats[30:]])
    late_coarse = np.mean([s["iterations"] for s in coarse_stats[30:]])
    print(late_hist, late_coarse)
    assert late_coarse < 0.7 * late_hist, (late_coarse, late_hist)


def test_coarse_grid_correction_on_axes_past_128(cuda):
    """A coarse axis of 129-256 cells (the case of the 512x512x256 plume,
    here 320 x 96 x 64 coarsened x2 to 160 x 48 x 32) is solved exactly as
    well, by the transforms that take the basis in two halves: converged
    steps, the history start's steps within the tolerance, no coarse CG
    iterations, fewer fine iterations."""
    from diff_solver_b200.data import plume_configuration
    cfg = plume_configuration((320, 96, 64), inflow_center=(0.5, 0.05, 0.1), inflow_radius=0.04)
    cfg.warm_start_history = 5
    hist, hist_stats, _ = _rollout(cfg, 30)
    cfg.warm_start_coarsening = 2
    coarse, coarse_stats, _ = _rollout(cfg, 30)
    assert all(s["status"] == 0 and s["final_residual"] <= 1e-6 for s in coarse_stats)
    assert rel(coarse, hist) < 1e-4
    assert all(s["coarse_iterations"] == 0 for s in coarse_stats)
    late_hist = np.mean([s["iterations"] for s in hist_stats[15:]])
    late_coarse = np.mean([s["iterations"] for s in coarse_stats[15:]])
    print(late_hist, late_coarse)
    assert late_coarse < 0.7 * late_hist, (late_coarse, late_hist)


def test_coarse_grid_correction_by_coarse_cg(cuda):
    """A closed box (zero-gradient pressure on every face: an anchor cell) does
    not separate: its coarse grid is solved by Jacobi-PCG from the
    three-level start, with the iterations reported; converged, the same
    steps, fewer fine iterations than the history start alone."""
    from diff_solver_b200.data import ScalarBoundaryMode, VelocityBoundaryMode, plume_configuration
    cfg = plume_configuration((64, 64, 64))
    cfg.velocity_boundary.y_max.mode = VelocityBoundaryMode.normal_fixed_tangent_zero_gradient
    cfg.pressure_boundary.y_max.mode = ScalarBoundaryMode.zero_gradient
    cfg.warm_start_history = 5
    hist, hist_stats, _ = _rollout(cfg, 30)
    cfg.warm_start_coarsening = 2
    coarse, coarse_stats, _ = _rollout(cfg, 30)
    assert all(s["status"] == 0 and s["final_residual"] <= 1e-6 for s in coarse_stats)
    assert rel(coarse, hist) < 1e-4
    assert all(s["coarse_iterations"] > 0 for s in coarse_stats[1:])
    late_hist = np.mean([s["iterations"] for s in hist_stats[15:]])
    late_coarse = np.mean([s["iterations"] for s in coarse_stats[15:]])
    print(late_hist, late_coarse)
    assert late_coarse < late_hist, (late_coarse, late_hist)


def test_coarse_correction_with_learned_guess(cuda):
    """Ring start, coarse-grid step, then the network's step on the residual
    left by that: converged, same steps."""
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.warm_start import WarmStartNetwork
    res = (128, 64, 32)
    cfg = plume_configuration(res)
    plain, _, _ = _rollout(cfg, 8)
    cfg.warm_start_history = 5
    cfg.warm_start_coarsening = 2
    net = WarmStartNetwork(res, factor=1, seed=4)
    warm, warm_stats, _ = _rollout(cfg, 8, network=net)
    net.check()
    assert all(s["status"] == 0 and s["final_residual"] <= 1e-6 for s in warm_stats)
    assert rel(warm, plain) < 1e-4


def test_galerkin_history_with_learned_guess(cuda):
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.warm_start import WarmStartNetwork
    res = (128, 64, 32)
    cfg = plume_configuration(res)
    plain, plain_stats, _ = _rollout(cfg, 8)
    cfg.warm_start_history = 3
    net = WarmStartNetwork(res, factor=1, seed=4)
    warm, warm_stats, _ = _rollout(cfg, 8, network=net)
    net.check()
    assert all(s["status"] == 0 and s["final_residual"] <= 1e-6 for s in warm_stats)
    assert rel(warm, plain) < 1e-4
    assert sum(s["iterations"] for s in warm_stats) < sum(s["iterations"] for s in plain_stats)


def test_trained_network_gain(cuda):
    """What the committed network (trained at 128^3 on 20k plume pairs) gains
    in the benchmark's own pipeline and window: the 256^3 plume spun up 180
    steps from rest, then from that state 5 + 20 steps with each forward
    solve started from the ring of the last 5 solutions and one round of
    sweeps and coarse-grid correction, with and without the network's
    correction step on top (network on the grid restricted x4, as the
    benchmark runs it).  The network's step removes fine PCG iterations there
    (measured: 9 -> 7 per step); on the young plume (steps 20-60) the x4
    network removes none.  A second round of sweeps and coarse correction,
    the start without the network uses by default, removes more (4 per
    step) for less time; the network's restriction, inference and line step
    cost more time than the iterations it saves (bench.py's history+coarse
    and learned+history+coarse arms report both).  This test asserts the
    iteration gain over the same start, the part the network is
    responsible for, and records the two-round start beside it."""
    import torch
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters, tensors_of
    from diff_solver_b200.warm_start import WarmStartNetwork
    weights = os.path.join(ROOT, "diff_solver_b200", "weights", "warm_start_128.npz")
    res = (256, 256, 256)
    net = WarmStartNetwork((64, 64, 64), factor=4)
    net.load(weights)

    def model(rounds=1):
        cfg = plume_configuration(res)
        cfg.pressure_max_iterations = 20000
        cfg.warm_start_history = 5
        cfg.warm_start_coarsening = 2
        cfg.warm_start_rounds = rounds
        m = Model(cfg)
        ctx = m.allocate_context(ExecutionMode.forward)
        return m, ctx, m.allocate_state(ctx), m.allocate_state(ctx), m.allocate_control(ctx), m.allocate_step_cache(ctx), \
            fill_parameters(m.allocate_parameters(ctx), 0.0, -0.1, 0.5)

    m, ctx, s, n, c, k, q = model()
    g = torch.Generator(device="cuda").manual_seed(0)
    for t in s.velocity.components():
        t.uniform_(-0.01, 0.01, generator=g)
    for _ in range(180):
        m.forward_step(s, c, q, n, k, ctx)
        s, n = n, s
    spun = [t.clone() for t in tensors_of(s)]
    del m, ctx, s, n, c, k, q
    iterations = {}
    for name, rounds in (("classical", 1), ("learned", 1), ("classical, two rounds", 2)):
        m, ctx, s, n, c, k, q = model(rounds)
        if name == "learned":
            ctx.set_learned_warm_start(net)
        for d, src in zip(tensors_of(s), spun):
            d.copy_(src)
        its = []
        for step in range(25):
            m.forward_step(s, c, q, n, k, ctx)
            s, n = n, s
            st = ctx.read_solve_stats()
            assert st["status"] == 0 and st["final_residual"] <= 1e-6, st
            if step >= 5:
                its.append(st["iterations"])
        iterations[name] = float(np.mean(its))
        del m, ctx, s, n, c, k, q
        torch.cuda.empty_cache()
    net.check()
    print(iterations)
    from common import report
    report("trained_network_gain_256", **iterations)
    assert iterations["learned"] <= 0.9 * iterations["classical"], iterations


def test_learned_warm_start_inside_a_model_step(cuda):
    """A model carrying the network solves to the same tolerance and gives the
    same step as the plain solver (both within the 1e-6 residual)."""
    import torch
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    from diff_solver_b200.warm_start import WarmStartNetwork
    res = (128, 64, 32)
    cfg = plume_configuration(res)
    m = Model(cfg)
    out = {}
    net = WarmStartNetwork(res, factor=1, seed=4)
    for name in ("plain", "learned"):
        ctx = m.allocate_context(ExecutionMode.forward)
        if name == "learned":
            ctx.set_learned_warm_start(net)
        s, n = m.allocate_state(ctx), m.allocate_state(ctx)
        c, k = m.allocate_control(ctx), m.allocate_step_cache(ctx)
        q = fill_parameters(m.allocate_parameters(ctx), 0.0, -0.1, 0.5)
        g = torch.Generator().manual_seed(0)
        for t in s.velocity.components():
            t.copy_((torch.rand(t.shape, generator=g) * 0.02 - 0.01).cuda())
        stats = []
        for _ in range(6):
            m.forward_step(s, c, q, n, k, ctx)
            s, n = n, s
            stats.append(ctx.read_solve_stats())
        out[name] = (torch.cat([t.reshape(-1) for t in s.velocity.components()]).cpu().numpy(), stats)
    net.check()
    for st in out["learned"][1]:
        assert st["status"] == 0 and st["final_residual"] <= 1e-6
    assert rel(out["learned"][0], out["plain"][0]) < 1e-4
