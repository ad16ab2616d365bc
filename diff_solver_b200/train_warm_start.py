"""Trains the learned pressure warm start on plume pairs and evaluates it.

    python -m diff_solver_b200.train_warm_start --grid 128 --pairs 20000 --batch 8 \
        --lr 1e-3 --out diff_solver_b200/weights/warm_start_128.npz

Training pairs are (right-hand side, pressure) of the plain PCG solver
(relative residual 1e-6) on plumes whose inflow centre, radius (0.05-0.12)
and buoyancy (0.2-1.0) are drawn from a seeded uniform distribution.  The
evaluation counts PCG iterations to 1e-6 from the learned guess against the
zero guess on a held-out plume (the benchmark's: centre (0.5, 0.1, 0.5),
radius 0.08, buoyancy 0.5) at the training grid and, with --eval-factor 2, on
a grid twice as fine through restriction and prolongation.  Progress is
printed as JSON lines.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--grid", type=int, default=128, help="network grid (cubic)")
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--loss", choices=["energy", "l2"], default="energy")
    ap.add_argument("--buffer", type=int, default=256, help="replay buffer size (pairs)")
    ap.add_argument("--episode", type=int, default=200, help="steps per plume before it restarts")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--init", default=None, help="start from these weights (.npz)")
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval-steps", type=int, default=100)
    ap.add_argument("--eval-every", type=int, default=10)
    ap.add_argument("--eval-factor", type=int, default=0, help="also evaluate on a grid this many times finer (0: no)")
    ap.add_argument("--eval-fine-steps", type=int, default=40)
    ap.add_argument("--eval-arms-steps", type=int, default=0,
                    help="steps of the side-by-side run of the plain, history, learned and learned+history starts (0: skip)")
    ap.add_argument("--history", type=int, default=4, help="previous solutions in the Galerkin start of that run")
    ap.add_argument("--fine-factor", type=int, default=1,
                    help="generate the pairs on a grid this many times finer and restrict them to the network grid")
    ap.add_argument("--train-history", type=int, default=0,
                    help="train on (residual, correction) pairs of a ring of this many previous solutions (0: (rhs, pressure))")
    ap.add_argument("--time-inference", action="store_true",
                    help="only time the network: guess on a grid twice as fine, then predict on its own grid (3 warm-up + 10 timed each)")
    args = ap.parse_args(argv)

    import torch

    from .warm_start import WarmStartNetwork, evaluate_arms, evaluate_on_plume, train_on_plumes

    def emit(rec):
        print(json.dumps(rec), flush=True)

    if args.time_inference:
        from . import _native as N
        shape = (args.grid,) * 3
        net = WarmStartNetwork(shape, factor=2)
        if args.init:
            net.load(args.init)
        fine = tuple(2 * s for s in shape)
        rhs = torch.randn(fine[0] * fine[1] * fine[2], device="cuda")
        small = torch.randn(shape[0] * shape[1] * shape[2], device="cuda")
        grid = N.XsGrid(*fine, 1.0 / fine[0], 0.5 / fine[0])
        for _ in range(3):
            net.guess(grid, rhs)
            net.predict(small)
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record()
        for _ in range(10):
            net.guess(grid, rhs)
        ev[1].record()
        for _ in range(10):
            net.predict(small)
        ev[2].record()
        torch.cuda.synchronize()
        net.check()
        emit({"network_grid": shape, "guess_ms": ev[0].elapsed_time(ev[1]) / 10, "predict_ms": ev[1].elapsed_time(ev[2]) / 10})
        return 0

    shape = (args.grid,) * 3
    net = WarmStartNetwork(shape, max_batch=args.batch, factor=1, seed=args.seed)
    if args.init:
        net.load(args.init)
    t0 = time.perf_counter()
    records = []
    if args.pairs > 0:
        records = train_on_plumes(net, pairs=args.pairs, batch=args.batch, learning_rate=args.lr, buffer_size=args.buffer,
                                  episode_steps=args.episode, seed=args.seed, log=emit, loss=args.loss, history=args.train_history,
                                  fine_factor=args.fine_factor)
    train_s = time.perf_counter() - t0
    emit({"trained_pairs": args.pairs, "seconds": train_s})
    summary = {"pairs": args.pairs, "train_seconds": train_s, "final_loss": records[-1]["loss"] if records else None}
    if args.eval_steps > 0:
        ev = evaluate_on_plume(net, shape, steps=args.eval_steps, every=args.eval_every)
        for r in ev:
            emit({"eval_grid": args.grid, **r})
        plain = float(np.mean([r["plain_iterations"] for r in ev]))
        learned = float(np.mean([r["learned_iterations"] for r in ev]))
        summary.update(eval_plain_iterations=plain, eval_learned_iterations=learned)
        emit({"eval_grid": args.grid, "mean_plain_iterations": plain, "mean_learned_iterations": learned, "ratio": plain / learned})
    if args.eval_factor > 1:
        f = args.eval_factor
        params = net.parameters()
        fine_net = WarmStartNetwork(shape, max_batch=1, factor=f)
        fine_net.set_parameters(params)
        ev = evaluate_on_plume(fine_net, tuple(f * s for s in shape), steps=args.eval_fine_steps, every=max(1, args.eval_fine_steps // 8))
        for r in ev:
            emit({"eval_grid": f * args.grid, **r})
        plain = float(np.mean([r["plain_iterations"] for r in ev]))
        learned = float(np.mean([r["learned_iterations"] for r in ev]))
        summary.update(fine_plain_iterations=plain, fine_learned_iterations=learned)
        emit({"eval_grid": f * args.grid, "mean_plain_iterations": plain, "mean_learned_iterations": learned, "ratio": plain / learned})
    if args.eval_arms_steps > 0:
        arms = evaluate_arms(net, shape, steps=args.eval_arms_steps, history=args.history)
        for name, its in arms.items():
            late = its[len(its) // 4:]
            emit({"arm": name, "grid": args.grid, "mean_iterations": float(np.mean(its)), "mean_late_iterations": float(np.mean(late)),
                  "iterations": its})
            summary[f"arm_{name}_iterations"] = float(np.mean(its))
    if args.out:
        net.save(args.out, **{k: v for k, v in summary.items() if v is not None})
        emit({"saved": args.out})
    torch.cuda.synchronize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
