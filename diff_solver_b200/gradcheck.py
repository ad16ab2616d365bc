"""Gradient checks and adjoint timing of the differentiable plume.

    python -m diff_solver_b200.gradcheck fd     [--grid 128 --steps 50 --checkpoint 10 --directions 16 --eps 1e-3]
    python -m diff_solver_b200.gradcheck adjoint [--grid 256 --forward 200 --window 40 --checkpoint 8]

``fd``: the plume of the benchmark physics (inflow r = 0.08 at (0.5, 0.1,
0.5), buoyancy 0.5 T - 0.1 rho) from rest with seeded velocity noise; loss
L = sum over cells of (rho_T - target)^2 with target a Gaussian blob
(sigma = 0.1) at a seeded uniform centre in [0.3, 0.7]^3.  The gradient with
respect to the initial velocity comes from the checkpointed VJP (every
``checkpoint`` steps, recompute in between) and is compared with central
finite differences of the loss along seeded unit directions (smooth random
fields: a few Gaussian bumps per velocity component, scaled to unit L2
norm over all faces).  The pressure solves use a tight tolerance so that the
finite differences resolve the derivative (the PCG result then is a smooth
function of its input to the working precision).  The state is FP32: the
rounding of every cell's density in the two perturbed rollouts makes the
loss difference noisy at about 1e-7 of each cell's contribution, so a
direction whose derivative is small is resolved only at larger step sizes
(--eps takes a list; each direction is reported at each).  The test suite
checks the same VJP against FP64 finite differences of the CPU oracle.

``adjoint``: ``forward`` steps forward (with the warm start the benchmark
uses when --learned is given), then a VJP over the last ``window`` steps
with checkpoints every ``checkpoint`` steps; reports the wall times of the
forward rollout, the checkpointed re-simulation and the reverse pass,
measured with CUDA events.

Each prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

PARAMS = dict(ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=0.5, vorticity_confinement=0.0)


def _setup(grid, tolerance, history=0, mode=None, coarsening=0):
    import torch

    from .data import plume_configuration
    from .model import ExecutionMode, Model, fill_parameters
    cfg = plume_configuration((grid, grid, grid), inflow_center=(0.5, 0.1, 0.5), inflow_radius=0.08)
    cfg.pressure_tolerance = tolerance
    cfg.pressure_max_iterations = 50000
    cfg.warm_start_history = history
    cfg.warm_start_coarsening = coarsening
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.differentiable if mode is None else mode)
    params = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    return torch, model, ctx, params


def _cell_centres(grid):
    c = (np.arange(grid) + 0.5) / grid
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return x, y, z


def smooth_direction(rng, shapes, grid, bumps=3):
    """Unit-norm velocity direction: per face component a sum of Gaussian bumps
    (sigma 0.08, centres uniform in [0.2, 0.8]^3, normal amplitudes)."""
    out = []
    for a, shape in enumerate(shapes):  # shape (nz, ny, nx) of face component a
        nz, ny, nx = shape
        off = [0.5, 0.5, 0.5]
        off[a] = 0.0
        x = (np.arange(nx) + off[0]) / grid
        y = (np.arange(ny) + off[1]) / grid
        z = (np.arange(nz) + off[2]) / grid
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        f = np.zeros(shape)
        for _ in range(bumps):
            c = rng.uniform(0.2, 0.8, 3)
            f += rng.normal() * np.exp(-((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) / (2 * 0.08 ** 2))
        out.append(f)
    norm = np.sqrt(sum(float((f * f).sum()) for f in out))
    return [f / norm for f in out]


def finite_difference_check(grid=128, steps=50, checkpoint=10, directions=16, eps=1e-3, tolerance=1e-10, seed=0):
    from .model import tensors_of
    from .solver import TapeMode, simulate, vjp
    torch, model, ctx, params = _setup(grid, tolerance)
    rng = np.random.default_rng(seed)
    controls = [model.allocate_control(ctx) for _ in range(steps)]
    u0 = model.allocate_state(ctx)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    for t in u0.velocity.components():
        t.copy_((torch.rand(t.shape, generator=gen, dtype=torch.float64) * 0.02 - 0.01).float().cuda())
    centre = rng.uniform(0.3, 0.7, 3)
    x, y, z = _cell_centres(grid)
    target = torch.from_numpy(np.exp(-((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2) / (2 * 0.1 ** 2)).reshape(-1)).cuda()

    def loss(state):
        d = state.density.values.double() - target
        return float((d * d).sum())

    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    traj = simulate(model, ctx, u0, controls, params, TapeMode.checkpoint, checkpoint)
    b.record()
    torch.cuda.synchronize()
    forward_ms = a.elapsed_time(b)
    final = traj.states[-1]
    L0 = loss(final)
    seed_adj = model.allocate_state_adjoint(ctx)
    seed_adj.density.values.copy_(2.0 * (final.density.values.double() - target))
    a.record()
    grad = vjp(model, ctx, traj, controls, params, {steps: seed_adj})
    b.record()
    torch.cuda.synchronize()
    vjp_ms = a.elapsed_time(b)
    g = [t.cpu().numpy().astype(np.float64) for t in grad.initial_state.velocity.components()]
    n = grid
    shapes = [(n, n, n + 1), (n, n + 1, n), (n + 1, n, n)]  # (z, y, x) extents of the face components

    work = model.allocate_state(ctx)
    nxt = model.allocate_state(ctx)
    cache = model.allocate_step_cache(ctx)

    base = [t.double().cpu().numpy() for t in u0.velocity.components()]

    def rollout(perturbation, scale):
        """Loss from u0 + scale * perturbation (rounded to FP32) and the
        perturbation actually applied (the FP32 state minus u0, in FP64)."""
        for dst, src in zip(tensors_of(work), tensors_of(u0)):
            dst.copy_(src)
        applied = []
        for t, d, b0 in zip(work.velocity.components(), perturbation, base):
            t.copy_(torch.from_numpy(b0 + scale * d.reshape(-1)).float().cuda())
            applied.append(t.double().cpu().numpy() - b0)
        cur, other = work, nxt
        for k in range(steps):
            model.forward_step(cur, controls[k], params, other, cache, ctx)
            cur, other = other, cur
        return loss(cur), applied

    epsilons = [eps] if np.isscalar(eps) else list(eps)
    rows = []
    for k in range(directions):
        d = smooth_direction(rng, shapes, grid)
        row = {"direction": k, "vjp": sum(float((gi * di.reshape(-1)).sum()) for gi, di in zip(g, d))}
        for e in epsilons:
            (lp, ap), (lm, am) = rollout(d, e), rollout(d, -e)
            # the directional derivative along the perturbation the FP32 state received
            gd = sum(float(gi @ (a - b)) for gi, a, b in zip(g, ap, am)) / (2 * e)
            fd = (lp - lm) / (2 * e)
            row[f"fd@{e:g}"] = fd
            row[f"vjp@{e:g}"] = gd
            row[f"rel@{e:g}"] = abs(fd - gd) / max(abs(fd), abs(gd), 1e-300)
        rows.append(row)
    summary = {}
    for e in epsilons:
        rels = [r[f"rel@{e:g}"] for r in rows]
        summary[f"{e:g}"] = {"max_rel": max(rels), "median_rel": float(np.median(rels)),
                             "below_1e-3": int(sum(r < 1e-3 for r in rels))}
    return {"check": "fd", "grid": grid, "steps": steps, "checkpoint": checkpoint, "epsilons": epsilons, "tolerance": tolerance,
            "loss": L0, "summary": summary, "directions": rows, "forward_ms": forward_ms, "vjp_ms": vjp_ms,
            "checkpoints": len(traj.states)}


def adjoint_timing(grid=256, forward=200, window=40, checkpoint=8, tolerance=1e-6, learned=False, history=5, seed=0, coarsening=2):
    from .model import ExecutionMode, tensors_of
    from .solver import TapeMode, simulate, vjp
    torch, model, ctx, params = _setup(grid, tolerance, history=history, coarsening=coarsening if history else 0)
    network = None
    if learned:
        from .warm_start import WarmStartNetwork
        weights = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", f"warm_start_{grid // 2}.npz")
        network = WarmStartNetwork((grid // 2,) * 3, factor=2)
        network.load(weights)
        ctx.set_learned_warm_start(network)
    gen = torch.Generator(device="cpu").manual_seed(seed)
    state = model.allocate_state(ctx)
    for t in state.velocity.components():
        t.copy_((torch.rand(t.shape, generator=gen) * 0.02 - 0.01).cuda())
    controls = [model.allocate_control(ctx) for _ in range(forward)]
    nxt = model.allocate_state(ctx)
    cache = model.allocate_step_cache(ctx)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    cur, other = state, nxt
    iterations = []
    for k in range(forward - window):
        model.forward_step(cur, controls[k], params, other, cache, ctx)
        cur, other = other, cur
    ev[1].record()
    traj = simulate(model, ctx, cur, controls[forward - window:], params, TapeMode.checkpoint, checkpoint)
    ev[2].record()
    seed_adj = model.allocate_state_adjoint(ctx)
    seed_adj.density.values.copy_(traj.states[-1].density.values.double())
    grad = vjp(model, ctx, traj, controls[forward - window:], params, {window: seed_adj})
    ev[3].record()
    torch.cuda.synchronize()
    gnorm = float(sum((t.double() ** 2).sum() for t in grad.initial_state.velocity.components()) ** 0.5)
    if network is not None:
        network.check()
    return {"check": "adjoint", "grid": grid, "forward_steps": forward, "window": window, "checkpoint": checkpoint,
            "learned": learned, "history": history, "coarsening": coarsening if history else 0, "lead_in_ms": ev[0].elapsed_time(ev[1]),
            "window_forward_ms": ev[1].elapsed_time(ev[2]), "vjp_ms": ev[2].elapsed_time(ev[3]),
            "vjp_ms_per_step": ev[2].elapsed_time(ev[3]) / window, "gradient_norm": gnorm, "checkpoints": len(traj.states)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    f = sub.add_parser("fd")
    f.add_argument("--grid", type=int, default=128)
    f.add_argument("--steps", type=int, default=50)
    f.add_argument("--checkpoint", type=int, default=10)
    f.add_argument("--directions", type=int, default=16)
    f.add_argument("--eps", type=lambda s: [float(v) for v in s.split(",")], default=[1e-3],
                   help="comma-separated step sizes (each direction is checked at every one)")
    f.add_argument("--tolerance", type=float, default=1e-10)
    f.add_argument("--seed", type=int, default=0)
    a = sub.add_parser("adjoint")
    a.add_argument("--grid", type=int, default=256)
    a.add_argument("--forward", type=int, default=200)
    a.add_argument("--window", type=int, default=40)
    a.add_argument("--checkpoint", type=int, default=8)
    a.add_argument("--tolerance", type=float, default=1e-6)
    a.add_argument("--history", type=int, default=5)
    a.add_argument("--learned", action="store_true")
    a.add_argument("--coarsening", type=int, default=2, help="coarse-grid correction of the forward and adjoint starts (0: off)")
    args = ap.parse_args(argv)
    if args.cmd == "fd":
        out = finite_difference_check(args.grid, args.steps, args.checkpoint, args.directions, args.eps, args.tolerance, args.seed)
    else:
        out = adjoint_timing(args.grid, args.forward, args.window, args.checkpoint, args.tolerance, args.learned, args.history,
                             coarsening=args.coarsening)
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
