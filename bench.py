#!/usr/bin/env python
"""Benchmark of the smoke step on B200.

Metric: smoke steps per second on the 256^3 plume (dx = 1/256, dt = dx/2,
inflow sphere r = 0.08 at (0.5, 0.1, 0.5) setting density = temperature = 1,
buoyancy +0.5 T - 0.1 rho on v, no confinement, walls with a fixed normal
velocity on the sides and bottom, open top), pressure by Jacobi-PCG to a
1e-6 relative residual from a zero guess (plain) or from the learned warm
start.  One step is Model.forward_step through the C ABI; the rollout starts
from rest with seeded uniform velocity noise in +-0.01.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs an independent
replica of the workload (the path does not shard: replicas only), timing is
max over ranks and ``value`` is the steps of all ranks per second.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256^3 smoke steps/s: learned-warm-start vs plain PCG at rel. residual 1e-6"
UNIT = "steps/s"
GRID = 256


def workload_configuration(n=GRID):
    from diff_solver_b200.data import plume_configuration
    cfg = plume_configuration((n, n, n), inflow_center=(0.5, 0.1, 0.5), inflow_radius=0.08)
    cfg.pressure_tolerance = 1e-6
    cfg.pressure_max_iterations = 20000
    return cfg


PARAMS = dict(ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=0.5, vorticity_confinement=0.0)


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


# --------------------------------------------------------------------- helpers
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def pcg_algorithmic_bytes(n_cells, iterations, refinements):
    """Unique bytes the persistent PCG kernel must move: per CG iteration
    36 B/cell (spmv phase: read z, p_old, e; write p_new, q, e -- 24 B;
    update phase: read z, q; write z -- 12 B); per true-residual pass 36 B
    (read rhs 4 + x64 8, write z, p0, e, pressure 16, x64 8) plus 24 B for
    each fold (read e, p, x64; write x64)."""
    return n_cells * (36.0 * iterations + 36.0 * (refinements + 1) + 24.0 * refinements)


def init_distributed():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=None)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------- CPU
def cpu_sample(n=GRID, sample_iterations=8, gpu_iterations=None):
    """The FP64 oracle step on the host cores: one step with the PCG capped at
    0 and at `sample_iterations` iterations; the step time at the GPU's
    iteration count is t0 + k * (t_k - t0) / sample_iterations."""
    import numpy as np
    from oracle import binding as ob
    threads = os.cpu_count() or 1
    ob.set_threads(threads)
    cfg = workload_configuration(n)
    rng = np.random.default_rng(0)
    P0 = ob.Problem(cfg, "f64", solver="pcg", iterations=0, tolerance=1e-6)
    st = ob.zeros_state(P0.res, np.float64)
    for a in range(3):
        st["velocity"][a][:] = rng.uniform(-0.01, 0.01, st["velocity"][a].shape)
    ctl = ob.zeros_control(P0.res, np.float64)
    t = time.perf_counter()
    P0.forward_step(st, ctl, PARAMS)
    t0 = time.perf_counter() - t
    Pk = ob.Problem(cfg, "f64", solver="pcg", iterations=sample_iterations, tolerance=1e-30)
    t = time.perf_counter()
    _, _, stats, _ = Pk.forward_step(st, ctl, PARAMS)
    tk = time.perf_counter() - t
    per_iteration = max(tk - t0, 0.0) / max(stats.iterations, 1)
    k = gpu_iterations if gpu_iterations is not None else 1400
    seconds = t0 + k * per_iteration
    return {"value": 1.0 / seconds, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"FP64 oracle forward step at {n}^3 on {threads} threads: one step with 0 and one with {sample_iterations} "
                      f"PCG iterations ({t0:.2f} s, {tk:.2f} s), projected to {k} iterations per step "
                      f"({per_iteration * 1e3:.1f} ms per iteration)",
            "seconds_per_step": seconds}


# --------------------------------------------------------------------- product
def product_arm(args, world, rank, local):
    import torch

    from diff_solver_b200 import _native as N
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters

    torch.cuda.set_device(local)
    L = N.lib()
    cfg = workload_configuration(args.grid)
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.forward)
    stream = ctx.stream
    n = model.cell_count
    gen = torch.Generator(device="cuda").manual_seed(0)
    state = model.allocate_state(ctx)
    for t in (state.velocity.x, state.velocity.y, state.velocity.z):
        t.uniform_(-0.01, 0.01, generator=gen)
    nxt = model.allocate_state(ctx)
    control = model.allocate_control(ctx)
    params = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    cache = model.allocate_step_cache(ctx)
    stats_off = L.xs_solve_stats_offset()
    stats_dev = ctx.workspace[stats_off:stats_off + C.sizeof(N.XsSolveStats)]

    def step(s, o):
        model.forward_step(s, control, params, o, cache, ctx)

    # warm-up rollout
    cur, other = state, nxt
    for _ in range(args.warmup):
        step(cur, other)
        cur, other = other, cur
    torch.cuda.synchronize()

    # timed region: K steps, solve kernel timed per step with events
    k_steps = args.steps
    stats_host = torch.zeros((k_steps, C.sizeof(N.XsSolveStats)), dtype=torch.uint8).pin_memory()
    solve_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k_steps)]
    for a, b in solve_events:  # create the handles
        a.record(stream)
        b.record(stream)
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    launches0 = L.xs_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    with torch.cuda.stream(stream):
        for i in range(k_steps):
            ctx.native.solve_begin = solve_events[i][0].cuda_event
            ctx.native.solve_end = solve_events[i][1].cuda_event
            step(cur, other)
            stats_host[i].copy_(stats_dev, non_blocking=True)
            cur, other = other, cur
    end.record(stream)
    torch.cuda.synchronize()
    launches = L.xs_launch_count() - launches0
    barrier(world)
    clocks = sampler.stop()
    elapsed_ms = start.elapsed_time(end)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    per_step = [N.XsSolveStats.from_buffer_copy(bytes(stats_host[i].numpy())) for i in range(k_steps)]
    iterations = [s.iterations for s in per_step]
    refinements = [s.refinements for s in per_step]
    residuals = [s.final_residual for s in per_step]

    # the dominant kernel (persistent PCG), one launch per step, timed by the
    # events the step recorded around it inside the timed region
    kernel_ms = [a.elapsed_time(b) for a, b in solve_events]
    ctx.native.solve_begin = None
    ctx.native.solve_end = None

    # end to end through the public API with host buffers: every step copies
    # its control fields from pinned host memory and reads back the metrics
    host_ctl = [torch.zeros(n, dtype=torch.float32).pin_memory() for _ in range(5)]
    dev_ctl = [control.density_source.values, control.temperature_source.values, control.external_acceleration.x.values,
               control.external_acceleration.y.values, control.external_acceleration.z.values]
    metrics_dev = torch.zeros(6, dtype=torch.float64, device="cuda")
    metrics_host = torch.zeros((k_steps, 6), dtype=torch.float64).pin_memory()
    barrier(world)
    torch.cuda.synchronize()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    with torch.cuda.stream(stream):
        for i in range(k_steps):
            for h, d in zip(host_ctl, dev_ctl):
                d.copy_(h, non_blocking=True)
            model.forward_step(cur, control, params, other, cache, ctx)
            N.check("metrics", L.xs_smoke_reduce_metrics(ctx.stream_handle, C.byref(ctx.native), other.density.values.data_ptr(),
                                                         other.temperature.values.data_ptr(), N.vec(cache.advected_velocity.components()),
                                                         N.vec(other.velocity.components()), metrics_dev.data_ptr()))
            metrics_host[i].copy_(metrics_dev, non_blocking=True)
            cur, other = other, cur
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e_start.elapsed_time(e_end), world)
    m_last = metrics_host[-1].numpy()
    return dict(model=model, elapsed_ms=elapsed_ms, iterations=iterations, refinements=refinements, residuals=residuals,
                kernel_ms=kernel_ms, launches=launches, clocks=clocks, e2e_ms=e2e_ms,
                h2d=5 * n * 4, d2h=6 * 8 + 0, metrics=m_last, n=n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["product", "reference"], default="product")
    ap.add_argument("--grid", type=int, default=GRID)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = init_distributed()
    config = {"workload": f"smoke plume {args.grid}^3, Jacobi-PCG to rel. residual 1e-6, zero guess",
              "grid": [args.grid] * 3, "cells": args.grid ** 3, "dt": "0.5 dx", "steps_per_replica": args.steps,
              "l2": "inputs larger than L2 (state 336 MB at 256^3)", "parallelism": f"replicas{world}"}
    if args.impl == "reference":
        if rank == 0:
            cpu = cpu_sample(args.grid, gpu_iterations=None)
            line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": 1e3 * cpu["seconds_per_step"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                    "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                    "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return
    r = product_arm(args, world, rank, local)
    if rank != 0:
        return
    steps_total = args.steps * world
    value = steps_total / (r["elapsed_ms"] / 1e3)
    peak, peak_kind = measured_peaks()
    kbytes_each = [pcg_algorithmic_bytes(r["n"], it, rf) for it, rf in zip(r["iterations"], r["refinements"])]
    kbytes = statistics.mean(kbytes_each)
    kms = statistics.mean(r["kernel_ms"])
    achieved = sum(kbytes_each) / (sum(r["kernel_ms"]) / 1e3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["elapsed_ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 CG reductions and iterate)", "data": "synthetic", "config": config,
            "method": "plain", "pcg_iterations_per_step": r["iterations"], "final_residuals": r["residuals"],
            "roofline": {"bound": "hbm", "kernel": "pcg_kernel", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": kbytes, "launch_ms": kms,
                         "iterations_per_launch": statistics.mean(r["iterations"])},
            "gpu_launches": r["launches"], "clocks": r["clocks"],
            "e2e": {"value": steps_total / (r["e2e_ms"] / 1e3), "unit": UNIT, "h2d_bytes_per_step": r["h2d"],
                    "d2h_bytes_per_step": r["d2h"]},
            "example_metrics_last_step": [float(v) for v in r["metrics"]]}
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(args.grid, gpu_iterations=int(statistics.mean(r["iterations"])))
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
