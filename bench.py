#!/usr/bin/env python
"""Benchmark of the smoke step on B200.

Metric: smoke steps per second on the 256^3 plume (dx = 1/256, dt = dx/2,
inflow sphere r = 0.08 at (0.5, 0.1, 0.5) setting density = temperature = 1,
buoyancy +0.5 T - 0.1 rho on v, no confinement, walls with a fixed normal
velocity on the sides and bottom, open top), pressure by Jacobi-PCG to a
1e-6 relative residual.  One step is Model.forward_step through the C ABI.

The plume first spins up from rest (seeded uniform velocity noise in
+-0.01) for --spinup steps; every arm then starts from that state:

  plain                   zero start (the reference's zero-initialised solve)
  history                 Galerkin start from the last 5 forward solutions
  history+coarse          ... then a step along the coarse-grid correction
  learned                 the warm-start network's guess alone, energy-scaled
  learned+history         the ring start, then a step along the network's
                          correction of its residual
  learned+history+coarse  the ring start, the coarse-grid step, then the
                          network's step (headline)

Each arm runs W warm-up steps (which also refill its ring) and K timed steps.
``value`` is the headline arm's steps/s; every arm's steps/s and PCG
iterations are in ``arms``.

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
HISTORY = 5
COARSENING = 2  # coarse-grid correction of the start on the grid coarsened x2 per axis
WEIGHTS = os.path.join(ROOT, "diff_solver_b200", "weights", "warm_start_128.npz")


def grid_shape(spec):
    """'256' -> (256, 256, 256); '512,512,256' -> (512, 512, 256)."""
    v = [int(s) for s in str(spec).split(",")]
    return tuple(v * 3) if len(v) == 1 else tuple(v)


def workload_configuration(shape=(GRID,) * 3, history=0, coarsening=0):
    """dx = 1 / nx; the inflow sits at x = 0.5, y = 0.1 and the middle of z."""
    from diff_solver_b200.data import plume_configuration
    nx, ny, nz = shape
    cfg = plume_configuration((nx, ny, nz), inflow_center=(0.5, 0.1, 0.5 * nz / nx), inflow_radius=0.08)
    cfg.pressure_tolerance = 1e-6
    cfg.pressure_max_iterations = 20000
    cfg.warm_start_history = history
    cfg.warm_start_coarsening = coarsening
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


# DRAM traffic of the plain solve's persistent PCG launch per algorithmic byte,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of this
# workload's plain solve at 256^3: 800.5 GB for 1323 CG iterations and 2
# refinement passes, whose algorithmic count below is 801.7 GB.
PCG_TRAFFIC_PER_ALGORITHMIC_BYTE_256 = 800.5 / 801.7


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
    """The slowest rank's figure (NCCL groups reduce on the device, gloo on
    the host)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------- CPU
def cpu_sample(shape=(GRID,) * 3, sample_iterations=40, gpu_iterations=None):
    """The FP64 oracle step on the host cores: one step with the PCG capped at
    0 and at `sample_iterations` iterations; the step time at the GPU's
    iteration count is t0 + k * (t_k - t0) / sample_iterations."""
    import numpy as np
    from oracle import binding as ob
    threads = os.cpu_count() or 1
    ob.set_threads(threads)
    cfg = workload_configuration(shape)
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
            "sample": f"FP64 oracle forward step at {'x'.join(map(str, shape))} on {threads} threads: one step with 0 and one with {sample_iterations} "
                      f"PCG iterations ({t0:.2f} s, {tk:.2f} s), projected to {k} iterations per step "
                      f"({per_iteration * 1e3:.1f} ms per iteration)",
            "seconds_per_step": seconds}


# --------------------------------------------------------------------- product
class Rollout:
    """One execution context of the workload with its own state buffers."""

    def __init__(self, grid, history, network, coarsening=0):
        from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
        self.model = Model(workload_configuration(grid, history, coarsening))
        self.ctx = self.model.allocate_context(ExecutionMode.forward)
        if network is not None:
            self.ctx.set_learned_warm_start(network)
        m = self.model
        self.cur, self.other = m.allocate_state(self.ctx), m.allocate_state(self.ctx)
        self.control = m.allocate_control(self.ctx)
        self.params = fill_parameters(m.allocate_parameters(self.ctx), **PARAMS)
        self.cache = m.allocate_step_cache(self.ctx)

    def load(self, state):
        from diff_solver_b200.model import tensors_of
        for d, s in zip(tensors_of(self.cur), tensors_of(state)):
            d.copy_(s)
        self.ctx.reset_warm_start()

    def step(self):
        self.model.forward_step(self.cur, self.control, self.params, self.other, self.cache, self.ctx)
        self.cur, self.other = self.other, self.cur


def timed_arm(args, world, ro, initial, e2e=False):
    """W warm-up and K timed steps of one arm from `initial`; per-step solve
    windows (warm start + PCG) timed by events the step records."""
    import torch

    from diff_solver_b200 import _native as N
    L = N.lib()
    ro.load(initial)
    stream = ro.ctx.stream
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            ro.step()
    torch.cuda.synchronize()
    k_steps = args.steps
    stats_off = L.xs_solve_stats_offset()
    stats_dev = ro.ctx.workspace[stats_off:stats_off + C.sizeof(N.XsSolveStats)]
    stats_host = torch.zeros((k_steps, C.sizeof(N.XsSolveStats)), dtype=torch.uint8).pin_memory()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k_steps)]
    for a, b in events:
        a.record(stream)
        b.record(stream)
    barrier(world)
    torch.cuda.synchronize()
    launches0 = L.xs_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    with torch.cuda.stream(stream):
        for i in range(k_steps):
            ro.ctx.native.solve_begin = events[i][0].cuda_event
            ro.ctx.native.solve_end = events[i][1].cuda_event
            ro.step()
            stats_host[i].copy_(stats_dev, non_blocking=True)
    end.record(stream)
    torch.cuda.synchronize()
    launches = L.xs_launch_count() - launches0
    barrier(world)
    ro.ctx.native.solve_begin = None
    ro.ctx.native.solve_end = None
    per_step = [N.XsSolveStats.from_buffer_copy(bytes(stats_host[i].numpy())) for i in range(k_steps)]
    out = dict(elapsed_ms=max_over_ranks(start.elapsed_time(end), world), launches=launches,
               iterations=[s.iterations for s in per_step], refinements=[s.refinements for s in per_step],
               coarse_iterations=[s.coarse_iterations for s in per_step],
               residuals=[s.final_residual for s in per_step], initial_residuals=[s.initial_residual for s in per_step],
               solve_ms=[a.elapsed_time(b) for a, b in events])
    if e2e:
        # the same K steps again, from the same state after the same warm-up
        ro.load(initial)
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                ro.step()
        torch.cuda.synchronize()
        out.update(end_to_end(args, world, ro))
    return out


def end_to_end(args, world, ro):
    """K steps through the public API with host buffers: every step copies
    its control fields from pinned host memory and reads back the example
    metrics.  The controls are double-buffered: step k+1's upload runs on a
    copy stream while step k computes (it waits for step k-1, the last user
    of its buffer); the first upload and every step's wait on its upload lie
    inside the timed region."""
    import torch

    from diff_solver_b200 import _native as N
    L = N.lib()
    n = ro.model.cell_count
    host_ctl = [torch.zeros(n, dtype=torch.float32).pin_memory() for _ in range(5)]
    ctls = [ro.control, ro.model.allocate_control(ro.ctx)]

    def fields(c):
        return [c.density_source.values, c.temperature_source.values, c.external_acceleration.x.values, c.external_acceleration.y.values,
                c.external_acceleration.z.values]

    metrics_dev = torch.zeros(6, dtype=torch.float64, device="cuda")
    metrics_host = torch.zeros((args.steps, 6), dtype=torch.float64).pin_memory()
    stream = ro.ctx.stream
    copy_stream = torch.cuda.Stream()
    uploaded = [torch.cuda.Event(), torch.cuda.Event()]
    released = [torch.cuda.Event(), torch.cuda.Event()]

    def upload(j):
        with torch.cuda.stream(copy_stream):
            for h, d in zip(host_ctl, fields(ctls[j])):
                d.copy_(h, non_blocking=True)
            uploaded[j].record(copy_stream)

    barrier(world)
    torch.cuda.synchronize()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    copy_stream.wait_event(e_start)
    upload(0)
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            j = i % 2
            if i + 1 < args.steps:
                if i >= 1:
                    copy_stream.wait_event(released[1 - j])
                upload(1 - j)
            stream.wait_event(uploaded[j])
            ro.model.forward_step(ro.cur, ctls[j], ro.params, ro.other, ro.cache, ro.ctx)
            released[j].record(stream)
            N.check("metrics", L.xs_smoke_reduce_metrics(ro.ctx.stream_handle, C.byref(ro.ctx.native), ro.other.density.values.data_ptr(),
                                                         ro.other.temperature.values.data_ptr(), N.vec(ro.cache.advected_velocity.components()),
                                                         N.vec(ro.other.velocity.components()), metrics_dev.data_ptr()))
            metrics_host[i].copy_(metrics_dev, non_blocking=True)
            ro.cur, ro.other = ro.other, ro.cur
    e_end.record(stream)
    torch.cuda.synchronize()
    return dict(e2e_ms=max_over_ranks(e_start.elapsed_time(e_end), world), h2d=5 * n * 4, d2h=6 * 8, metrics=metrics_host[-1].numpy())


def product_run(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    network = None
    if not args.no_learned:
        from diff_solver_b200.warm_start import WarmStartNetwork
        if not os.path.exists(args.weights):
            raise FileNotFoundError(f"{args.weights} is missing: train it with python -m diff_solver_b200.train_warm_start")
        # trained at 128^3, applied fully convolutionally on the grid restricted
        # x network_factor (2 by default)
        f = args.network_factor
        network = WarmStartNetwork(tuple(s // f for s in args.shape), factor=f)
        network.load(args.weights)
    # spin-up from rest with the fastest start; its final state opens every arm
    spin = Rollout(args.shape, HISTORY, network, args.coarsening)
    gen = torch.Generator(device="cuda").manual_seed(0)
    for t in spin.cur.velocity.components():
        t.uniform_(-0.01, 0.01, generator=gen)
    with torch.cuda.stream(spin.ctx.stream):
        for _ in range(args.spinup):
            spin.step()
    torch.cuda.synchronize()
    from diff_solver_b200.model import tensors_of
    initial = spin.model.allocate_state(spin.ctx)
    for d, s in zip(tensors_of(initial), tensors_of(spin.cur)):
        d.copy_(s)
    del spin
    arms = [("plain", 0, None, 0), ("history", HISTORY, None, 0)]
    if args.coarsening:
        arms += [("history+coarse", HISTORY, None, args.coarsening)]
    if network is not None:
        arms += [("learned", 0, network, 0), ("learned+history", HISTORY, network, 0)]
        if args.coarsening:
            arms += [("learned+history+coarse", HISTORY, network, args.coarsening)]
    if args.arms:  # a subset (profiling runs); the last one named is the headline
        keep = args.arms.split(",")
        unknown = [k for k in keep if k not in {a[0] for a in arms}]
        if unknown:
            raise ValueError(f"unknown arms {unknown}: choose from {[a[0] for a in arms]}")
        arms = [a for k in keep for a in arms if a[0] == k]
    headline = arms[-1][0]
    sampler = ClockSampler(local)
    sampler.start()
    results = {}
    for name, history, net, coarsening in arms:
        ro = Rollout(args.shape, history, net, coarsening)
        results[name] = timed_arm(args, world, ro, initial, e2e=(name == headline))
        del ro
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    if network is not None:
        network.check()
    return results, headline, clocks


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # the warm-started arms' iteration counts vary from step to step (120-550 at
    # 256^3): 20 timed steps per arm keep the mean within a few per cent
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--spinup", type=int, default=40, help="steps from rest before the arms start")
    ap.add_argument("--impl", choices=["product", "reference"], default="product")
    ap.add_argument("--grid", default=str(GRID), help="N for N^3, or nx,ny,nz")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="plain and history arms only")
    ap.add_argument("--weights", default=WEIGHTS, help="warm-start network parameters (.npz)")
    ap.add_argument("--coarsening", type=int, default=COARSENING, help="coarse-grid correction factor (0: off)")
    ap.add_argument("--network-factor", type=int, default=2, help="restriction from the grid to the network's grid (1, 2 or 4)")
    ap.add_argument("--arms", default="", help="comma-separated subset of the arms, headline last (profiling; no roofline "
                                               "or CPU baseline without the plain arm)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    args.shape = grid_shape(args.grid)
    world, rank, local = init_distributed()
    n = args.shape[0] * args.shape[1] * args.shape[2]
    name = "x".join(map(str, args.shape))
    config = {"workload": f"smoke plume {name} after a {args.spinup}-step spin-up from rest, Jacobi-PCG to rel. residual 1e-6",
              "grid": list(args.shape), "cells": n, "dt": "0.5 dx", "steps_per_replica": args.steps, "spinup_steps": args.spinup,
              "warm_start": f"Galerkin start over the last {HISTORY} solutions"
                            + (f", 6 Jacobi sweeps and a step along the coarse-grid correction (grid coarsened x{args.coarsening}, "
                               f"Jacobi-PCG to 1e-2 from its own two-level start)"
                               if args.coarsening else "")
                            + ("" if args.no_learned else
                               f", step along the U-Net correction (network trained at 128^3, applied on the grid restricted "
                               f"x{args.network_factor})"),
              "l2": f"inputs larger than L2 (state {n * 21 * 4 / 1e6:.0f} MB)", "parallelism": f"replicas{world}"}
    if args.impl == "reference":
        if rank == 0:
            cpu = cpu_sample(args.shape, gpu_iterations=None)
            line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": 1e3 * cpu["seconds_per_step"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                    "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                    "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return
    results, headline, clocks = product_run(args, world, rank, local)
    if rank != 0:
        return
    steps_total = args.steps * world
    arms = {}
    for name, r in results.items():
        arms[name] = {"steps_per_s": steps_total / (r["elapsed_ms"] / 1e3), "ms_per_step": r["elapsed_ms"] / args.steps,
                      "pcg_iterations_per_step": r["iterations"], "mean_pcg_iterations": statistics.mean(r["iterations"]),
                      "coarse_iterations_per_step": r["coarse_iterations"],
                      "refinement_passes_per_step": r["refinements"],
                      "solve_ms_per_step": statistics.mean(r["solve_ms"]), "initial_residuals": r["initial_residuals"],
                      "final_residuals": r["residuals"], "gpu_launches": r["launches"]}
    # whole-step roofline: B_step = 4 (8 N + 8 F) + 40 N k bytes per step (the
    # scope table's count: fused stages once, 10 floats per cell per CG iteration)
    nx, ny, nz = args.shape
    faces = (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)
    peak_gbs, _ = measured_peaks()
    for name, a in arms.items():
        b_step = 4.0 * (8 * n + 8 * faces) + 40.0 * n * a["mean_pcg_iterations"]
        a["step_roofline"] = {"bytes_per_step": b_step, "achieved_gbs": b_step / (a["ms_per_step"] / 1e3) / 1e9,
                              "frac": b_step / (a["ms_per_step"] / 1e3) / 1e9 / peak_gbs}
    h = results[headline]
    value = arms[headline]["steps_per_s"]
    # roofline of the dominant kernel (the persistent PCG), from the plain arm
    # where the solve window holds that kernel alone
    roofline = None
    if "plain" in results:
        p = results["plain"]
        peak, peak_kind = measured_peaks()
        kbytes_each = [pcg_algorithmic_bytes(n, it, rf) for it, rf in zip(p["iterations"], p["refinements"])]
        achieved = sum(kbytes_each) / (sum(p["solve_ms"]) / 1e3) / 1e9
        traffic = None
        if tuple(args.shape) == (GRID,) * 3:  # the captured workload: its measured traffic per algorithmic byte
            traffic = PCG_TRAFFIC_PER_ALGORITHMIC_BYTE_256 * statistics.mean(kbytes_each)
        roofline = {"bound": "hbm", "kernel": "pcg_kernel", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "traffic_unit": "bytes per launch", "peak_kind": peak_kind,
                    "algorithmic_bytes_per_launch": statistics.mean(kbytes_each),
                    "launch_ms": statistics.mean(p["solve_ms"]), "iterations_per_launch": statistics.mean(p["iterations"]), "arm": "plain"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": h["elapsed_ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 CG reductions and iterate)", "data": "synthetic", "config": config,
            "method": headline, "speedup_vs_plain": value / arms["plain"]["steps_per_s"] if "plain" in arms else None, "arms": arms,
            "roofline": roofline,
            "gpu_launches": h["launches"], "clocks": clocks,
            "e2e": {"value": steps_total / (h["e2e_ms"] / 1e3), "unit": UNIT, "h2d_bytes_per_step": h["h2d"],
                    "d2h_bytes_per_step": h["d2h"]},
            "example_metrics_last_step": [float(v) for v in h["metrics"]]}
    if world == 1 and not args.no_cpu_baseline and "plain" in arms:
        cpu = cpu_sample(args.shape, gpu_iterations=int(arms["plain"]["mean_pcg_iterations"]))
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
