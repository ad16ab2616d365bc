"""Timing of the reference's own smoke kernels on the GPU (test infrastructure).

The reference (solvers/smoke/operators.cu, compiled unmodified for sm_100a
into oracle/_ref by oracle/build_ref.sh) stepped in the reference's order
(model.cpp:341-349) through the harness: its default 80 red-black
Gauss-Seidel sweeps per step (data.ixx:76, not converged), and its sweeps
iterated until the FP64 relative residual of the pressure system reaches a
tolerance (what a 1e-6 solve costs the reference's method).  The controls
are zero (the benchmark's inflow is not emulated: timing only), the
velocity starts as the benchmark's seeded noise.  Prints one JSON line per
case.  Needs oracle/_ref (built in the development container).

    python oracle/time_reference.py [--grids 64,256] [--converged 64] [--steps 3]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def setup(n):
    import torch
    from common import reference_control  # noqa: F401  (tests helper, inflow emulation)
    from diff_solver_b200.data import plume_configuration
    from diff_solver_b200.model import ExecutionMode, Model
    from oracle import ref_binding as rb
    cfg = plume_configuration((n, n, n), inflow_center=(0.5, 0.1, 0.5), inflow_radius=0.08)
    m = Model(cfg)
    ctx = m.allocate_context(ExecutionMode.forward)
    d = ctx.domain
    dom = {"mask": d.cell_mask, "cv": list(d.collider_velocity.components()), "cd": d.collider_density.values,
           "ct": d.collider_temperature.values, "anchor": d.pressure_anchor}
    N = n ** 3
    faces = [(n + 1) * n * n, n * (n + 1) * n, n * n * (n + 1)]
    dev = "cuda"
    g = torch.Generator(device="cuda").manual_seed(0)
    state = [torch.zeros(N, device=dev), torch.zeros(N, device=dev)] + [torch.empty(f, device=dev).uniform_(-0.01, 0.01, generator=g)
                                                                        for f in faces]
    nxt = [torch.zeros(N, device=dev), torch.zeros(N, device=dev)] + [torch.zeros(f, device=dev) for f in faces]
    control = [torch.zeros(N, device=dev) for _ in range(5)]
    params = [torch.tensor([v], dtype=torch.float32, device=dev) for v in (0.0, -0.1, 0.5, 0.0)]
    cache = [torch.zeros(N, device=dev), torch.zeros(N, device=dev)] + [torch.zeros(N, device=dev) for _ in range(3)] + \
            [torch.zeros(11 * N, device=dev)] + [torch.zeros(f, device=dev) for f in faces] + [torch.zeros(f, device=dev) for f in faces]
    return cfg, dom, state, nxt, control, params, cache


def time_case(n, steps, tolerance, sweeps):
    import torch
    from oracle import ref_binding as rb
    cfg, dom, state, nxt, control, params, cache = setup(n)
    ref = rb.Reference(cfg, dom, iterations=sweeps)
    ref.forward_step(state, control, params, nxt, cache, tolerance=tolerance)  # warm-up
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total_sweeps = 0
    a.record()
    for _ in range(steps):
        s, res = ref.forward_step(state, control, params, nxt, cache, tolerance=tolerance)
        total_sweeps += s
        state, nxt = nxt, state
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    return {"grid": n, "rbgs": "to tolerance" if tolerance > 0 else f"{sweeps} sweeps", "tolerance": tolerance,
            "ms_per_step": ms, "steps_per_s": 1e3 / ms, "sweeps_per_step": total_sweeps / steps, "final_residual": res}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grids", default="64,256")
    ap.add_argument("--converged", default="64")
    ap.add_argument("--steps", type=int, default=3)
    args = ap.parse_args()
    for n in [int(v) for v in args.grids.split(",") if v]:
        print(json.dumps(time_case(n, args.steps, 0.0, 80)), flush=True)
    for n in [int(v) for v in args.converged.split(",") if v]:
        print(json.dumps(time_case(n, 1, 1e-6, 80)), flush=True)


if __name__ == "__main__":
    main()
