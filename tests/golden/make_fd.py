"""Generates tests/golden/fd_plume_<n>.npz: FP64 central finite differences of
the differentiable plume's loss (tests/common.py: differentiable_plume) along
its first seeded unit directions, from the CPU oracle (oracle/smoke_oracle.c,
FP64 build).  TEST INFRASTRUCTURE: the GPU test
tests/test_gpu_gradcheck.py::test_plume_vjp_matches_oracle_finite_differences
compares the product's checkpointed VJP with these numbers.

Each rollout runs `steps` FP64 oracle steps with the pressure solved by
Jacobi-PCG to `tolerance` (started from the previous step's pressure: the
converged result does not depend on the start).  Partial results are kept in
the output file after every rollout, and a rerun resumes from them.

    python tests/golden/make_fd.py [--grid 128] [--steps 50] [--directions 4] [--eps 1e-3] [--tolerance 1e-12] [--threads N]
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from common import PLUME_PARAMS, density_distance, differentiable_plume, plume_directions  # noqa: E402

from oracle import binding as ob  # noqa: E402


def rollout(P, u0, target, steps):
    st = ob.zeros_state(P.res, np.float64)
    for a in range(3):
        st["velocity"][a][:] = u0[a]
    ctl = ob.zeros_control(P.res, np.float64)
    guess = None
    iterations = 0
    for _ in range(steps):
        st, _, stats, w = P.forward_step(st, ctl, PLUME_PARAMS, guess=guess)
        if stats.converged != 1:
            raise RuntimeError(f"oracle solve did not converge (residual {stats.final_residual:.3e})")
        iterations += stats.iterations
        guess = w["p"].copy()
    return density_distance(st["density"], target), iterations


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--directions", type=int, default=4)
    ap.add_argument("--eps", type=float, default=1e-3)
    ap.add_argument("--tolerance", type=float, default=1e-12)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    out = a.out or os.path.join(HERE, f"fd_plume_{a.grid}.npz")
    ob.set_threads(a.threads)
    cfg, u0, target = differentiable_plume(a.grid)
    P = ob.Problem(cfg, "f64", solver="pcg", iterations=100000, tolerance=a.tolerance)
    dirs = plume_directions(a.grid, a.directions)
    done = {}
    if os.path.exists(out):
        z = np.load(out)
        if int(z["grid"]) == a.grid and int(z["steps"]) == a.steps and float(z["eps"]) == a.eps and float(z["tolerance"]) == a.tolerance:
            done = {"base": float(z["loss"]), "plus": list(z["loss_plus"]), "minus": list(z["loss_minus"])}
    base = done.get("base")
    plus, minus = list(done.get("plus", [])), list(done.get("minus", []))

    def save():
        k = min(len(plus), len(minus))
        fd = [(plus[i] - minus[i]) / (2 * a.eps) for i in range(k)]
        np.savez(out, grid=a.grid, steps=a.steps, eps=a.eps, tolerance=a.tolerance, loss=base if base is not None else np.nan,
                 loss_plus=np.array(plus[:k]), loss_minus=np.array(minus[:k]), finite_differences=np.array(fd),
                 direction_seed=2, velocity_seed=0, target_seed=1)

    t0 = time.time()
    if base is None:
        base, its = rollout(P, u0, target, a.steps)
        print(f"base loss {base:.15e} ({its} PCG iterations, {time.time() - t0:.0f} s)", flush=True)
        save()
    for k in range(len(plus), a.directions):
        d = dirs[k]
        lp, _ = rollout(P, [u + a.eps * di for u, di in zip(u0, d)], target, a.steps)
        lm, _ = rollout(P, [u - a.eps * di for u, di in zip(u0, d)], target, a.steps)
        plus.append(lp)
        minus.append(lm)
        save()
        print(f"direction {k}: fd {(lp - lm) / (2 * a.eps):.10e} ({time.time() - t0:.0f} s)", flush=True)
    save()


if __name__ == "__main__":
    main()
