#!/usr/bin/env python
"""Benchmark of the smoke step on B200.

Metric: smoke steps per second on the 256^3 plume (dx = 1/256, dt = dx/2,
inflow sphere r = 0.08 at (0.5, 0.1, 0.5) setting density = temperature = 1,
buoyancy +0.5 T - 0.1 rho on v, no confinement, walls with a fixed normal
velocity on the sides and bottom, open top), pressure by Jacobi-PCG to a
1e-6 relative residual.  One step is Model.forward_step through the C ABI.

The plume first spins up from rest (seeded uniform velocity noise in
+-0.01) for --spinup steps (180: the timed window is steps 185-205 of the
200-step plume); every arm then starts from that state:

  plain                   zero start (the reference's zero-initialised solve)
  history                 Galerkin start from the last 5 forward solutions
  history+coarse          ... then two rounds of Jacobi sweeps and a step along
                          the coarse-grid correction (coarse grid solved exactly
                          when its operator separates)
  learned                 the warm-start network's guess alone, energy-scaled
  learned+history         the ring start, then a step along the network's
                          correction of its residual
  learned+history+coarse  the ring start, one round of sweeps and coarse-grid
                          step, then the network's step (headline)

Each arm runs W warm-up steps (which also refill its ring) and K timed steps,
every timed step with per-stage CUDA events (XsSmokeModel.stage_events).
``value`` is the headline arm's steps/s; every arm's steps/s, PCG iterations
and per-stage times are in ``arms``.  Further records of the same run:

  roofline            the headline arm's dominant kernel, the fine PCG launch
                      (stage events around it), against the measured copy peak
  roofline_plain      the same kernel in the plain arm
  adjoint             the 40-step VJP (checkpoints every 8) ending at step 200,
                      with the reverse step's algorithmic bytes
  reference_kernels   the reference's own kernels (oracle/_ref) timed per kernel
                      on the same box and state, next to this library's
  large_grid          512x512x256 (steps 89-98 of its 100-step plume): plain,
                      two-round classical and headline arms, per-stage GB/s
  network             the warm-start network alone on its grid (predict and
                      guess), its convolution FLOPs against the bf16 peak
  config0             the 64^3 plume's full 100 steps from rest: plain and
                      headline arms on the GPU, the FP64 oracle on the host
  cpu_baseline        full FP64 oracle steps from the spun-up state on the
                      host's cores

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs an independent
replica of the workload (the path does not shard: replicas only), timing is
max over ranks and ``value`` is the steps of all ranks per second.  The
reference arm (--impl reference) times the FP64 oracle's full steps from the
same spun-up state on rank 0 (the other ranks exit).
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
HEADLINE = "learned+history+coarse"
LARGE_GRID = (512, 512, 256)


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


def counts(shape):
    nx, ny, nz = shape
    return nx * ny * nz, (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)


# DRAM traffic of the plain solve's persistent PCG launch per algorithmic byte,
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of this
# workload's plain solve at 256^3: 800.5 GB for 1323 CG iterations and 2
# refinement passes, whose algorithmic count below is 801.7 GB.
PCG_TRAFFIC_PER_ALGORITHMIC_BYTE_256 = 800.5 / 801.7
# The same for the warm-started solve with minimal-residual smoothing
# (pcg_kernel<1, 1>) in the benchmark window: 7.223 GB per launch over three
# captured launches of 7 CG iterations (5 smoothed) and 1 refinement pass,
# whose algorithmic count below is 7.181 GB.
PCG_SMOOTH_TRAFFIC_PER_ALGORITHMIC_BYTE_256 = 7.223 / 7.181


def pcg_algorithmic_bytes(n_cells, iterations, refinements, smoothed=0):
    """Unique bytes the persistent PCG kernel must move: per CG iteration
    36 B/cell (spmv phase: read z, p_old, e; write p_new, q, e -- 24 B;
    update phase: read z, q; write z -- 12 B), 16 B/cell more for each
    iteration that also carries the minimal-residual smoothed sequence (read
    and write s and y); per true-residual pass 36 B (read rhs 4 + x64 8,
    write z, p0, e, pressure 16, x64 8) plus 24 B for each fold (read e, p,
    x64; write x64)."""
    return n_cells * (36.0 * iterations + 16.0 * smoothed + 36.0 * (refinements + 1) + 24.0 * refinements)


# Algorithmic bytes of the step's stages (stage k runs between events k and
# k + 1), as functions of the cell count N and the face count F: unique reads
# plus writes of every array the stage's kernels must touch.
def stage_bytes(n, f):
    return {
        "sources_forces": 48.0 * n,             # read rho, T, 2 sources, 3 accelerations; write 2 sourced fields, 3 forces
        "integrate": 8.0 * f + 12.0 * n,        # read u, write u*; read the 3 force fields
        "advect_constrain": 8.0 * f,            # read u* (staged), write the advected velocity
        "pressure_rhs": 4.0 * f + 4.0 * n,      # read u, write the right-hand side
        "warm_start": None,                     # ring Galerkin pass, sweeps, coarse solves, network, line steps
        "fine_pcg": None,                       # pcg_algorithmic_bytes of the launch
        "ring_update": None,
        "projection": 8.0 * f + 8.0 * n,        # read u and the FP64 pressure, write u
        "scalar_advection": 4.0 * f + 16.0 * n,  # read u (staged), 2 sourced fields; write density, temperature
    }


STAGES = ["sources_forces", "integrate", "advect_constrain", "pressure_rhs", "warm_start", "fine_pcg", "ring_update", "projection",
          "scalar_advection"]


def reverse_step_bytes(n, f, forward_iterations, adjoint_iterations):
    """Algorithmic bytes of one checkpointed reverse step: the recomputed
    forward step (each state of a segment is recomputed once) plus the VJP
    step's transposes and its adjoint solve.  FP64 adjoints (8 B), FP32
    state (4 B), accumulated targets counted read + write:
      zeroing the scratch adjoints 8 (5N + 9F); copy of the incoming velocity
      adjoint 16F; scalar advection adjoint (density and temperature) 20F +
      56N; projection adjoint 40F + 16N (+ 36 B/cell per adjoint CG
      iteration); constraint 24F; velocity advection adjoint 28F; integration
      24F + 48N; buoyancy 112N; sources 80N: 352N + 224F in all."""
    forward = 4.0 * (8 * n + 8 * f) + 36.0 * n * forward_iterations
    return forward + 352.0 * n + 224.0 * f + 36.0 * n * adjoint_iterations


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
def cpu_steps(state_arrays, shape, budget_s=60.0, max_steps=3, min_steps=1):
    """Full forward steps of the FP64 CPU oracle (the same step, pressure by
    Jacobi-PCG to 1e-6 from a zero start as the plain arm) from the given
    host state, on all host cores, in sequence; stops after max_steps or once
    budget_s is spent (at least min_steps).  Returns the timing record."""
    import numpy as np

    from oracle import binding as ob
    threads = ob.set_threads(os.cpu_count() or 1)
    cfg = workload_configuration(shape)
    P = ob.Problem(cfg, "f64", solver="pcg", iterations=20000, tolerance=1e-6)
    ctl = ob.zeros_control(P.res, np.float64)
    st = state_arrays
    times, iterations = [], []
    t_all = time.perf_counter()
    while len(times) < max_steps and (len(times) < min_steps or time.perf_counter() - t_all < budget_s):
        t = time.perf_counter()
        st, _, stats, _ = P.forward_step(st, ctl, PARAMS)
        times.append(time.perf_counter() - t)
        iterations.append(int(stats.iterations))
    seconds = statistics.mean(times)
    return {"value": 1.0 / seconds, "unit": UNIT, "cores": threads, "kind": "port", "steps": len(times),
            "sample": f"{len(times)} full FP64 oracle forward step(s) at {'x'.join(map(str, shape))} from the spun-up plume state, "
                      f"pressure by Jacobi-PCG to 1e-6 from zero ({', '.join(map(str, iterations))} iterations; "
                      f"{', '.join(f'{t:.1f}' for t in times)} s) on {threads} host threads",
            "seconds_per_step": seconds, "iterations": iterations}


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


def make_events(count):
    import torch
    return [torch.cuda.Event(enable_timing=True) for _ in range(count)]


def timed_arm(args, world, ro, initial, e2e=False):
    """W warm-up and K timed steps of one arm from `initial`; each timed step
    records the stage events of the step (XsSmokeModel.stage_events) and the
    solve statistics."""
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
    stages = [make_events(N.XS_STEP_STAGES + 1) for _ in range(k_steps)]
    arrays = []
    for evs in stages:
        for e in evs:
            e.record(stream)  # creates the CUDA events
        arrays.append((C.c_void_p * len(evs))(*[e.cuda_event for e in evs]))
    barrier(world)
    torch.cuda.synchronize()
    launches0 = L.xs_launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    # an NVTX range around the timed steps lets a profiler select them
    with torch.cuda.stream(stream), torch.cuda.nvtx.range("timed"):
        for i in range(k_steps):
            ro.ctx.native.stage_events = C.cast(arrays[i], C.c_void_p)
            ro.step()
            stats_host[i].copy_(stats_dev, non_blocking=True)
    end.record(stream)
    torch.cuda.synchronize()
    launches = L.xs_launch_count() - launches0
    barrier(world)
    ro.ctx.native.stage_events = None
    per_step = [N.XsSolveStats.from_buffer_copy(bytes(stats_host[i].numpy())) for i in range(k_steps)]
    stage_ms = {name: [evs[k].elapsed_time(evs[k + 1]) for evs in stages] for k, name in enumerate(STAGES)}
    out = dict(elapsed_ms=max_over_ranks(start.elapsed_time(end), world), launches=launches,
               iterations=[s.iterations for s in per_step], refinements=[s.refinements for s in per_step],
               smoothed=[s.smoothed_iterations for s in per_step], coarse_iterations=[s.coarse_iterations for s in per_step],
               residuals=[s.final_residual for s in per_step], initial_residuals=[s.initial_residual for s in per_step],
               stage_ms=stage_ms, solve_ms=[w + p for w, p in zip(stage_ms["warm_start"], stage_ms["fine_pcg"])])
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


def load_network(args, shape):
    from diff_solver_b200.warm_start import WarmStartNetwork
    if not os.path.exists(args.weights):
        raise FileNotFoundError(f"{args.weights} is missing: train it with python -m diff_solver_b200.train_warm_start")
    # trained at 128^3, applied fully convolutionally on the grid restricted
    # x network_factor (4 by default; halved while that grid would be
    # smaller than 64 cells on an axis, the smallest the U-Net's four levels
    # are run on here)
    f = args.network_factor
    while f > 1 and min(shape) // f < 64:
        f //= 2
    args.network_factor = f
    network = WarmStartNetwork(tuple(s // f for s in shape), factor=f)
    network.load(args.weights)
    return network


# The U-Net's twelve 3x3x3 convolutions as (C_in, C_out, level), level l on
# the network grid coarsened 2^l per axis; channel counts as the tensor cores
# run them (padded to 16: the first layer reads 2 real channels, the output
# layer writes 1).
UNET_CONVOLUTIONS = [(16, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2), (64, 64, 3), (64, 64, 3),
                     (64, 32, 2), (32, 16, 1), (16, 16, 0), (16, 16, 0)]


def unet_flops(voxels, padded=True):
    """Multiply-add FLOPs (2 per MAC) of one network forward on `voxels` cells
    of the network grid; padded=False counts only the real input channels of
    the first layer (2) and the real output channel of the last (1)."""
    total = 0.0
    for i, (cin, cout, level) in enumerate(UNET_CONVOLUTIONS):
        if not padded:
            cin = 2 if i == 0 else cin
            cout = 1 if i == len(UNET_CONVOLUTIONS) - 1 else cout
        total += 2.0 * 27 * cin * cout * voxels / 8 ** level
    return total


def network_record(network, shape, repeats=10):
    """The learned step's network alone, timed with CUDA events on the
    launching stream after 3 warm-up calls: `predict` (the twelve tcgen05
    convolutions, pooling and upsampling on the network grid) and `guess`
    (restriction of a fine-grid right-hand side, normalisation, predict and
    prolongation).  Achieved TFLOP/s counts the algorithmic convolution
    FLOPs (real channels) against the measured burst bf16 peak (the network
    is timed alone)."""
    import torch

    from diff_solver_b200 import _native as N
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak, kind = (float(peaks["bf16_tflops"]), "measured burst") if "bf16_tflops" in peaks else (1590.0, "fallback burst")
    cells = network.cells
    gen = torch.Generator(device="cuda").manual_seed(3)
    small = torch.randn(cells, device="cuda", generator=gen)
    fine_shape = tuple(s * network.factor for s in network.shape)
    fine = torch.randn(fine_shape[0] * fine_shape[1] * fine_shape[2], device="cuda", generator=gen)
    grid = N.XsGrid(*fine_shape, 1.0 / fine_shape[0], 0.5 / fine_shape[0])
    stream = network.stream
    for _ in range(3):
        network.predict(small)
        network.guess(grid, fine)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    for _ in range(repeats):
        network.predict(small)
    ev[1].record(stream)
    for _ in range(repeats):
        network.guess(grid, fine)
    ev[2].record(stream)
    torch.cuda.synchronize()
    network.check()
    predict_ms = ev[0].elapsed_time(ev[1]) / repeats
    guess_ms = ev[1].elapsed_time(ev[2]) / repeats
    flops = unet_flops(cells, padded=False)
    achieved = flops / (predict_ms / 1e3) / 1e12
    return {"network_grid": list(network.shape), "fluid_grid": list(fine_shape), "predict_ms": predict_ms, "guess_ms": guess_ms,
            "flops_per_predict": flops, "flops_per_predict_padded": unet_flops(cells, padded=True),
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_kind": kind}}


def config0_record(args, shape=(64, 64, 64), steps=100, cpu=True, cpu_budget_s=90.0):
    """The 64^3 plume rolled from rest for its full 100 steps: on the GPU by
    the plain arm and the headline arm (network on the 64^3 grid itself),
    each timed with CUDA events on its stream after a 3-step warm-up and a
    reload of the start; and, with `cpu`, by the FP64 CPU oracle from the
    same start (the plain solve: Jacobi-PCG to 1e-6 from zero, all host
    cores) until all steps are done or `cpu_budget_s` is spent."""
    import torch

    from diff_solver_b200.model import tensors_of
    from diff_solver_b200.warm_start import WarmStartNetwork
    net = WarmStartNetwork(shape, factor=1)
    net.load(args.weights)
    rec = {"grid": list(shape), "steps": steps, "start": "rest; velocity noise U(-0.01, 0.01) on every face (CUDA generator, seed 0)",
           "arms": {}}
    initial = None
    for name, history, network, coarsening in (("plain", 0, None, 0), (HEADLINE, HISTORY, net, COARSENING)):
        ro = Rollout(shape, history, network, coarsening)
        gen = torch.Generator(device="cuda").manual_seed(0)
        for t in ro.cur.velocity.components():
            t.uniform_(-0.01, 0.01, generator=gen)
        start = ro.model.allocate_state(ro.ctx)
        for d, s in zip(tensors_of(start), tensors_of(ro.cur)):
            d.copy_(s)
        if initial is None:
            initial = [x.double().cpu().numpy() for x in tensors_of(start)]
        with torch.cuda.stream(ro.ctx.stream):
            for _ in range(3):
                ro.step()
        torch.cuda.synchronize()
        ro.load(start)
        torch.cuda.synchronize()
        ev = make_events(2)
        ev[0].record(ro.ctx.stream)
        with torch.cuda.stream(ro.ctx.stream):
            for _ in range(steps):
                ro.step()
        ev[1].record(ro.ctx.stream)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        last = ro.ctx.read_solve_stats()
        rec["arms"][name] = {"steps_per_s": steps / (ms / 1e3), "ms_per_step": ms / steps,
                             "last_solve": {k: last[k] for k in ("iterations", "final_residual")}}
        del ro, start
    net.check()
    del net
    torch.cuda.empty_cache()
    if cpu:
        rec["cpu"] = cpu_rollout({"density": initial[0], "temperature": initial[1], "velocity": initial[2:5]}, shape, steps, cpu_budget_s)
    return rec


def cpu_rollout(state_arrays, shape, steps, budget_s):
    """Consecutive FP64 CPU oracle steps of the workload from `state_arrays`
    (pressure by Jacobi-PCG to 1e-6 from zero, all host cores) until `steps`
    are done or `budget_s` is spent; returns the timing record."""
    import numpy as np

    from oracle import binding as ob
    threads = ob.set_threads(os.cpu_count() or 1)
    P = ob.Problem(workload_configuration(shape), "f64", solver="pcg", iterations=20000, tolerance=1e-6)
    ctl = ob.zeros_control(P.res, np.float64)
    st = state_arrays
    done, iterations, t0 = 0, 0, time.perf_counter()
    while done < steps and time.perf_counter() - t0 < budget_s:
        st, _, stats, _ = P.forward_step(st, ctl, PARAMS)
        done += 1
        iterations += int(stats.iterations)
    seconds = time.perf_counter() - t0
    return {"steps_per_s": done / seconds, "steps": done, "seconds": seconds, "pcg_iterations": iterations, "cores": threads,
            "kind": "port", "sample": f"{done} of the {steps} steps by the FP64 CPU oracle from the same start, pressure by "
                                      f"Jacobi-PCG to 1e-6 from zero ({iterations} iterations in all), on {threads} host threads"}


def spin_up(shape, network, steps, keep=()):
    """The plume from rest (seeded velocity noise) with the headline start;
    returns {step: state copy} for the steps in `keep` and the last."""
    import torch

    from diff_solver_b200.model import tensors_of
    spin = Rollout(shape, HISTORY, network, COARSENING)
    gen = torch.Generator(device="cuda").manual_seed(0)
    for t in spin.cur.velocity.components():
        t.uniform_(-0.01, 0.01, generator=gen)
    saved = {}

    def save(step):
        s = spin.model.allocate_state(spin.ctx)
        for d, src in zip(tensors_of(s), tensors_of(spin.cur)):
            d.copy_(src)
        saved[step] = s

    with torch.cuda.stream(spin.ctx.stream):
        for k in range(steps):
            if k in keep:
                save(k)
            spin.step()
        save(steps)
    torch.cuda.synchronize()
    return saved, spin


def summarize(results, args, shape, world, headline):
    n, faces = counts(shape)
    peak, peak_kind = measured_peaks()
    sb = stage_bytes(n, faces)
    steps_total = args.steps * world
    arms = {}
    for name, r in results.items():
        stage = {}
        for s in STAGES:
            ms = statistics.mean(r["stage_ms"][s])
            rec = {"ms": ms}
            if sb[s] is not None:
                rec["bytes"] = sb[s]
                rec["gbs"] = sb[s] / (ms / 1e3) / 1e9
            stage[s] = rec
        pcg_bytes = [pcg_algorithmic_bytes(n, it, rf, sm) for it, rf, sm in zip(r["iterations"], r["refinements"], r["smoothed"])]
        stage["fine_pcg"]["bytes"] = statistics.mean(pcg_bytes)
        stage["fine_pcg"]["gbs"] = sum(pcg_bytes) / (sum(r["stage_ms"]["fine_pcg"]) / 1e3) / 1e9
        b_step = 4.0 * (8 * n + 8 * faces) + 40.0 * n * statistics.mean(r["iterations"])
        arms[name] = {"steps_per_s": steps_total / (r["elapsed_ms"] / 1e3), "ms_per_step": r["elapsed_ms"] / args.steps,
                      "pcg_iterations_per_step": r["iterations"], "mean_pcg_iterations": statistics.mean(r["iterations"]),
                      "smoothed_iterations_per_step": r["smoothed"], "coarse_iterations_per_step": r["coarse_iterations"],
                      "refinement_passes_per_step": r["refinements"], "solve_ms_per_step": statistics.mean(r["solve_ms"]),
                      "initial_residuals": r["initial_residuals"], "final_residuals": r["residuals"], "gpu_launches": r["launches"],
                      "stages": stage,
                      "step_roofline": {"bytes_per_step": b_step, "achieved_gbs": b_step / (r["elapsed_ms"] / args.steps / 1e3) / 1e9,
                                        "frac": b_step / (r["elapsed_ms"] / args.steps / 1e3) / 1e9 / peak}}

    def pcg_roofline(arm):
        r = results[arm]
        pcg_bytes = [pcg_algorithmic_bytes(n, it, rf, sm) for it, rf, sm in zip(r["iterations"], r["refinements"], r["smoothed"])]
        achieved = sum(pcg_bytes) / (sum(r["stage_ms"]["fine_pcg"]) / 1e3) / 1e9
        kernel = "pcg_kernel<1, 1>" if arm != "plain" else "pcg_kernel<1, 0>"
        return {"bound": "hbm", "kernel": kernel, "arm": arm, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": statistics.mean(pcg_bytes),
                "launch_ms": statistics.mean(r["stage_ms"]["fine_pcg"]), "iterations_per_launch": statistics.mean(r["iterations"]),
                "smoothed_iterations_per_launch": statistics.mean(r["smoothed"])}
    return arms, pcg_roofline


def adjoint_record(args, shape, network, start_state, window=40, checkpoint=8):
    """Config 3's reverse pass: from the state at step 200 - window, the
    window's steps with checkpoints every `checkpoint`, then the VJP of the
    final density's L2 distance to a Gaussian target (sigma 0.1 at a seeded
    centre) back to the window's start.  Forward and adjoint solves use the
    headline starts (the network only in the forward solves)."""
    import numpy as np
    import torch

    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    from diff_solver_b200.solver import TapeMode, simulate, vjp
    cfg = workload_configuration(shape, HISTORY, COARSENING)
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.differentiable)
    if network is not None:
        ctx.set_learned_warm_start(network)
    ctx.reset_warm_start()
    params = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    controls = [model.allocate_control(ctx) for _ in range(window)]
    nx, ny, nz = shape
    centre = np.random.default_rng(1).uniform(0.3, 0.7, 3) * np.array([1.0, ny / nx, nz / nx])
    x = (torch.arange(nx, device="cuda", dtype=torch.float64) + 0.5) / nx
    y = (torch.arange(ny, device="cuda", dtype=torch.float64) + 0.5) / nx
    z = (torch.arange(nz, device="cuda", dtype=torch.float64) + 0.5) / nx
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    target = torch.exp(-((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2) / (2 * 0.1 ** 2)).reshape(-1)
    del X, Y, Z
    ev = make_events(4)
    torch.cuda.synchronize()
    ev[0].record()
    traj = simulate(model, ctx, start_state, controls, params, TapeMode.checkpoint, checkpoint)
    ev[1].record()
    final = traj.states[-1].density.values.double()
    d = final - target
    loss = torch.sqrt((d * d).sum())
    seed = model.allocate_state_adjoint(ctx)
    seed.density.values.copy_(d / loss)
    # The reverse pass allocates its gradient (one control adjoint per step),
    # its running adjoints and the checkpoint segment's states and caches.
    # Allocated and released once here, they are served from PyTorch's cached
    # blocks inside the timed pass, as in every call after a process' first:
    # the first cudaMalloc of ~30 GB measured 3 ms more per reverse step.
    warm = ([model.allocate_control_adjoint(ctx) for _ in range(window)], [model.allocate_state_adjoint(ctx) for _ in range(3)],
            [model.allocate_state(ctx) for _ in range(checkpoint)], [model.allocate_step_cache(ctx) for _ in range(checkpoint)],
            model.allocate_parameter_adjoint(ctx))
    del warm
    torch.cuda.synchronize()
    # every reverse step's adjoint-solve statistics, copied without a sync
    from diff_solver_b200 import _native as N
    off = N.lib().xs_solve_stats_offset()
    stats_dev = ctx.workspace[off:off + C.sizeof(N.XsSolveStats)]
    stats_host = torch.zeros((window, C.sizeof(N.XsSolveStats)), dtype=torch.uint8).pin_memory()
    torch.cuda.nvtx.range_push("reverse")  # the reverse pass, for profilers
    ev[2].record()
    grad = vjp(model, ctx, traj, controls, params, {window: seed},
               after_step=lambda step: stats_host[step].copy_(stats_dev, non_blocking=True))
    ev[3].record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    per_step = [N.XsSolveStats.from_buffer_copy(bytes(stats_host[i].numpy())) for i in range(window)]
    stats = ctx.read_solve_stats()
    gnorm = float(sum((t.double() ** 2).sum() for t in grad.initial_state.velocity.components()) ** 0.5)
    n, faces = counts(shape)
    reverse_ms = ev[2].elapsed_time(ev[3]) / window
    return {"window": window, "checkpoint": checkpoint, "steps": f"{200 - window}-200", "loss": float(loss),
            "forward_ms": ev[0].elapsed_time(ev[1]), "vjp_ms": ev[2].elapsed_time(ev[3]), "ms_per_reverse_step": reverse_ms,
            "gradient_norm": gnorm, "last_adjoint_solve": {"iterations": stats["iterations"], "residual": stats["final_residual"]},
            "adjoint_iterations_per_step": [s.iterations for s in per_step],
            "adjoint_coarse_iterations_per_step": [s.coarse_iterations for s in per_step],
            "adjoint_start_used_per_step": [s.warm_start_used for s in per_step],
            "adjoint_initial_residual_per_step": [s.initial_residual for s in per_step],
            "bytes_rule": "reverse_step_bytes(N, F, forward PCG iterations, adjoint PCG iterations)", "_n": n, "_f": faces}


def reference_kernels_record(args, ro, shape, repeats=5):
    """The reference's own kernels (solvers/smoke/operators.cu through
    oracle/_ref) timed one by one with CUDA events on the state of the last
    headline step, next to this library's kernels for the same operation.
    Algorithmic bytes as stage_bytes (the reference's advection + constraint
    and scalar advection count the same arrays)."""
    import torch

    from diff_solver_b200 import _native as N
    from oracle import ref_binding as rb
    if not rb.available():
        return {"unavailable": "oracle/_ref is not built"}
    n, faces = counts(shape)
    ctx = ro.ctx
    d = ctx.domain
    dom = {"mask": d.cell_mask, "cv": list(d.collider_velocity.components()), "cd": d.collider_density.values,
           "ct": d.collider_temperature.values, "anchor": d.pressure_anchor}
    ref = rb.Reference(ro.model.configuration, dom, iterations=1)
    dev = torch.device("cuda")
    forced = list(ro.cache.forced_velocity.components())
    u_next = list(ro.cur.velocity.components())
    out = [torch.empty_like(t) for t in forced]
    raw = [torch.empty_like(t) for t in forced]
    src = ro.cache.sourced_density.values
    sout = torch.empty_like(src)
    rhs = torch.empty(n, device=dev)
    pressure = ctx.pressure_fields()[0].clone()
    gen = torch.Generator(device="cuda").manual_seed(3)
    oa = [torch.randn(t.numel(), generator=gen, device=dev, dtype=torch.float64) for t in forced]
    ua = [torch.zeros(t.numel(), device=dev, dtype=torch.float64) for t in forced]
    soa = torch.randn(n, generator=gen, device=dev, dtype=torch.float64)
    sa = torch.zeros(n, device=dev, dtype=torch.float64)
    L = N.lib()
    g = ctx.native.grid
    vb = ctx.native.velocity_boundary

    def time_it(fn):
        fn()
        torch.cuda.synchronize()
        a, b = make_events(2)
        a.record()
        for _ in range(repeats):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / repeats

    R = rb
    rec = {}
    rec["advect_constrain"] = {"reference_ms": time_it(lambda: (ref.launch(R.ADVECT_VELOCITY, u=forced, out=raw),
                                                                ref.launch(R.CONSTRAIN_VELOCITY, u=raw, out=out)))}
    rec["scalar_advection"] = {"reference_ms": time_it(lambda: (ref.launch(R.ADVECT_SCALAR, src=src, u=u_next, sout=sout),
                                                                ref.launch(R.ADVECT_SCALAR, src=ro.cache.sourced_temperature.values,
                                                                           u=u_next, sout=sout)))}
    rec["pressure_rhs"] = {"reference_ms": time_it(lambda: ref.launch(R.PRESSURE_RHS, u=forced, rhs=rhs))}
    rec["projection"] = {"reference_ms": time_it(lambda: ref.launch(R.PROJECT_VELOCITY, u=forced, pressure=pressure, out=out))}
    sweep_ms = time_it(lambda: ref.launch(R.RBGS_SWEEPS, rhs=rhs, pressure=pressure))
    rec["pressure_iteration"] = {"reference_ms": sweep_ms, "reference": "one red-black Gauss-Seidel sweep pair (rbgs_kernel x2)",
                                 "reference_bytes": 2 * 4.0 * n * 2, "reference_gbs": 16.0 * n / (sweep_ms / 1e3) / 1e9}
    rec["advect_velocity_vjp"] = {"reference_ms": time_it(lambda: ref.launch(R.ADVECT_VELOCITY_VJP, u=forced, oa=oa, ua=ua)),
                                  "product_ms": time_it(lambda: N.check("vjp", L.xs_advect_velocity_vjp(ctx.stream_handle, g, None,
                                                                                                        N.vec(forced), vb, N.vec(oa),
                                                                                                        N.vec(ua)))),
                                  "bytes": 4.0 * faces + 8.0 * faces + 16.0 * faces}
    rec["advect_scalar_vjp"] = {"reference_ms": time_it(lambda: ref.launch(R.ADVECT_SCALAR_VJP, src=src, u=u_next, soa=soa, sa=sa, ua=ua)),
                                "product_ms": time_it(lambda: N.check("svjp", L.xs_advect_scalar_vjp(
                                    ctx.stream_handle, g, None, C.c_void_p(src.data_ptr()), N.vec(u_next), ctx.native.density_boundary, vb,
                                    C.c_void_p(soa.data_ptr()), C.c_void_p(sa.data_ptr()), N.vec(ua)))),
                                "bytes": 4.0 * faces + 4.0 * n + 8.0 * n + 16.0 * n + 16.0 * faces}
    del ref
    return rec


LARGE_SPINUP = 85  # every timed step of the large grid lies within its 100-step plume


def large_grid_record(args, network_large, shape=LARGE_GRID, spinup=LARGE_SPINUP, warmup=3, steps=5, headline_steps=10):
    import torch
    saved, spin = spin_up(shape, network_large, spinup)
    initial = saved[spinup]
    del spin
    torch.cuda.empty_cache()
    sub = argparse.Namespace(steps=steps, warmup=warmup)
    results = {}
    for name, history, net, coarsening, k in (("plain", 0, None, 0, steps), ("history+coarse", HISTORY, None, COARSENING, headline_steps),
                                              (HEADLINE, HISTORY, network_large, COARSENING, headline_steps)):
        ro = Rollout(shape, history, net, coarsening)
        sub.steps = k
        results[name] = timed_arm(sub, 1, ro, initial)
        results[name]["_steps"] = k
        del ro
        torch.cuda.empty_cache()
    return results


def product_run(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    network = None if args.no_learned else load_network(args, args.shape)
    window = args.adjoint_window
    keep = (max(args.spinup + 20 - window, 0),) if not args.no_adjoint else ()
    saved, spin = spin_up(args.shape, network, args.spinup, keep)
    initial = saved[args.spinup]
    del spin
    torch.cuda.empty_cache()
    arms = [("plain", 0, None, 0), ("history", HISTORY, None, 0)]
    if args.coarsening:
        arms += [("history+coarse", HISTORY, None, args.coarsening)]
    if network is not None:
        arms += [("learned", 0, network, 0), ("learned+history", HISTORY, network, 0)]
        if args.coarsening:
            arms += [(HEADLINE, HISTORY, network, args.coarsening)]
    if args.arms:  # a subset (profiling runs); the last one named is the headline
        keep_arms = args.arms.split(",")
        unknown = [k for k in keep_arms if k not in {a[0] for a in arms}]
        if unknown:
            raise ValueError(f"unknown arms {unknown}: choose from {[a[0] for a in arms]}")
        arms = [a for k in keep_arms for a in arms if a[0] == k]
    headline = arms[-1][0]
    sampler = ClockSampler(local)
    sampler.start()
    results = {}
    extra = {}
    for name, history, net, coarsening in arms:
        ro = Rollout(args.shape, history, net, coarsening)
        results[name] = timed_arm(args, world, ro, initial, e2e=(name == headline))
        if name == headline and not args.no_reference_kernels and world == 1:
            extra["reference_kernels"] = reference_kernels_record(args, ro, args.shape)
        del ro
        torch.cuda.empty_cache()
    clocks = sampler.stop()
    if network is not None and world == 1:
        try:
            extra["network"] = network_record(network, args.shape)
        except Exception as e:  # a record beside the headline: report it, keep the line
            extra["network"] = {"error": f"{type(e).__name__}: {e}"}
    if not args.no_adjoint and world == 1:
        extra["adjoint"] = adjoint_record(args, args.shape, network, saved[keep[0]], window=window)
        torch.cuda.empty_cache()
    if not args.no_large and world == 1 and network is not None:
        from diff_solver_b200.warm_start import WarmStartNetwork
        f = args.network_factor
        big = WarmStartNetwork(tuple(s // f for s in LARGE_GRID), factor=f)
        big.load(args.weights)
        extra["large_grid"] = large_grid_record(args, big)
        big.check()
        del big
        torch.cuda.empty_cache()
    if not args.no_config0 and world == 1 and network is not None:
        try:
            extra["config0"] = config0_record(args, cpu=not args.no_cpu_baseline)
        except Exception as e:  # a record beside the headline: report it, keep the line
            extra["config0"] = {"error": f"{type(e).__name__}: {e}"}
        torch.cuda.empty_cache()
    if network is not None:
        network.check()
    host_state = None
    if world == 1 and not args.no_cpu_baseline:
        from diff_solver_b200.model import tensors_of
        t = [x.double().cpu().numpy() for x in tensors_of(initial)]
        host_state = {"density": t[0], "temperature": t[1], "velocity": t[2:5]}
    return results, headline, clocks, extra, host_state


def reference_run(args):
    """The reference arm: the FP64 oracle's full steps on the host cores, from
    the spun-up state (generated on the GPU by the library outside the timed
    region: the CPU cannot roll a 256^3 plume 180 steps in minutes)."""
    import torch
    torch.cuda.set_device(0)
    network = None if args.no_learned else load_network(args, args.shape)
    saved, spin = spin_up(args.shape, network, args.spinup)
    from diff_solver_b200.model import tensors_of
    t = [x.double().cpu().numpy() for x in tensors_of(saved[args.spinup])]
    del spin, saved
    host_state = {"density": t[0], "temperature": t[1], "velocity": t[2:5]}
    return cpu_steps(host_state, args.shape, budget_s=args.cpu_budget, max_steps=min(args.steps, args.cpu_steps))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # the warm-started arms' iteration counts vary from step to step: 20
    # timed steps per arm keep the mean within a few per cent
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--spinup", type=int, default=180, help="steps from rest before the arms start")
    ap.add_argument("--impl", choices=["product", "reference"], default="product")
    ap.add_argument("--grid", default=str(GRID), help="N for N^3, or nx,ny,nz")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="plain and history arms only")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the 40-step VJP record")
    ap.add_argument("--no-large", action="store_true", help="skip the 512x512x256 record")
    ap.add_argument("--no-reference-kernels", action="store_true", help="skip the per-kernel timing of the reference's kernels")
    ap.add_argument("--no-config0", action="store_true", help="skip the 100-step 64^3 rollout from rest (GPU arms and CPU oracle)")
    ap.add_argument("--adjoint-window", type=int, default=40)
    ap.add_argument("--cpu-steps", type=int, default=3, help="most full FP64 steps the CPU legs time")
    ap.add_argument("--cpu-budget", type=float, default=150.0, help="seconds after which the CPU legs stop adding steps")
    ap.add_argument("--weights", default=WEIGHTS, help="warm-start network parameters (.npz)")
    ap.add_argument("--coarsening", type=int, default=COARSENING, help="coarse-grid correction factor (0: off)")
    # x4: the network runs on 64^3 for the 256^3 grid (8x cheaper than x2 for
    # the same fine-iteration saving, measured: 141.9 against 119.4 steps/s)
    ap.add_argument("--network-factor", type=int, default=4, help="restriction from the grid to the network's grid (1, 2 or 4)")
    ap.add_argument("--arms", default="", help="comma-separated subset of the arms, headline last (profiling; no roofline "
                                               "or CPU baseline without the plain arm)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    args.shape = grid_shape(args.grid)
    world, rank, local = init_distributed()
    n, faces = counts(args.shape)
    name = "x".join(map(str, args.shape))
    config = {"workload": f"smoke plume {name}, timed steps {args.spinup + args.warmup}-{args.spinup + args.warmup + args.steps} after "
                          f"rest (spin-up {args.spinup} steps), Jacobi-PCG to rel. residual 1e-6",
              "grid": list(args.shape), "cells": n, "faces": faces, "dt": "0.5 dx", "steps_per_replica": args.steps,
              "spinup_steps": args.spinup,
              "warm_start": f"Galerkin start over the last {HISTORY} solutions"
                            + (f", 6 Jacobi sweeps and a step along the coarse-grid correction (grid coarsened x{args.coarsening}, "
                               f"solved exactly by the eigenbases of its separable operator; adjoint solves: three such rounds)"
                               if args.coarsening else "")
                            + ("" if args.no_learned else
                               f", step along the U-Net correction (network trained at 128^3, applied on the grid restricted "
                               f"x{args.network_factor})"),
              "l2": f"inputs larger than L2 (state {n * 21 * 4 / 1e6:.0f} MB)", "parallelism": f"replicas{world}"}
    if args.impl == "reference":
        if rank == 0:
            cpu = reference_run(args)
            line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world, "steps": cpu["steps"],
                    "warmup": 0, "ms_per_step": 1e3 * cpu["seconds_per_step"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                    "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                    "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                    "note": "full FP64 steps of the CPU oracle (the reference has no CPU path) from the spun-up state; "
                            "the state is produced on the GPU before the timed region"}
            print(json.dumps(line), flush=True)
        return
    results, headline, clocks, extra, host_state = product_run(args, world, rank, local)
    if rank != 0:
        return
    steps_total = args.steps * world
    arms, pcg_roofline = summarize(results, args, args.shape, world, headline)
    h = results[headline]
    value = arms[headline]["steps_per_s"]
    def with_traffic(rf):
        # the captured workload: each kernel's measured dram bytes per algorithmic byte
        ratio = PCG_TRAFFIC_PER_ALGORITHMIC_BYTE_256 if rf["arm"] == "plain" else PCG_SMOOTH_TRAFFIC_PER_ALGORITHMIC_BYTE_256
        rf["traffic"] = ratio * rf["algorithmic_bytes_per_launch"] if tuple(args.shape) == (GRID,) * 3 else None
        rf["traffic_unit"] = "bytes per launch (the kernel's ncu-measured ratio of dram bytes to algorithmic bytes at 256^3)"
        return rf

    roofline = with_traffic(pcg_roofline(headline))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": h["elapsed_ms"] / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 CG reductions and iterate)", "data": "synthetic", "config": config,
            "method": headline, "speedup_vs_plain": value / arms["plain"]["steps_per_s"] if "plain" in arms else None, "arms": arms,
            "roofline": roofline, "roofline_plain": with_traffic(pcg_roofline("plain")) if "plain" in results else None,
            "gpu_launches": h["launches"], "clocks": clocks,
            "e2e": {"value": steps_total / (h["e2e_ms"] / 1e3), "unit": UNIT, "h2d_bytes_per_step": h["h2d"],
                    "d2h_bytes_per_step": h["d2h"]},
            "example_metrics_last_step": [float(v) for v in h["metrics"]]}
    peak, _ = measured_peaks()
    if "adjoint" in extra:
        a = extra.pop("adjoint")
        n_, f_ = a.pop("_n"), a.pop("_f")
        fwd_it = statistics.mean(arms[headline]["pcg_iterations_per_step"])
        adj_it = statistics.mean(a["adjoint_iterations_per_step"])
        b = reverse_step_bytes(n_, f_, fwd_it, adj_it)
        a["reverse_step_bytes"] = b
        a["reverse_step_gbs"] = b / (a["ms_per_reverse_step"] / 1e3) / 1e9
        a["reverse_step_frac"] = a["reverse_step_gbs"] / peak
        line["adjoint"] = a
    if "network" in extra:
        line["network"] = extra.pop("network")
    if "config0" in extra:
        line["config0"] = extra.pop("config0")
    if "reference_kernels" in extra:
        rk = extra.pop("reference_kernels")
        if "unavailable" not in rk:
            st = arms[headline]["stages"]
            for k in ("advect_constrain", "scalar_advection", "pressure_rhs", "projection"):
                rk[k]["product_ms"] = st[k]["ms"]
                rk[k]["bytes"] = st[k]["bytes"]
            p = arms[headline]
            rk["pressure_iteration"]["product_ms"] = st["fine_pcg"]["ms"] / max(p["mean_pcg_iterations"], 1)
            rk["pressure_iteration"]["product"] = "one Jacobi-PCG iteration of the fine solve (36 B/cell)"
            for k, r in rk.items():
                if "bytes" in r and "product_ms" in r:
                    r["product_gbs"] = r["bytes"] / (r["product_ms"] / 1e3) / 1e9
                    r["reference_gbs"] = r["bytes"] / (r["reference_ms"] / 1e3) / 1e9
                if "product_ms" in r and "reference_ms" in r:
                    r["speedup"] = r["reference_ms"] / r["product_ms"]
        line["reference_kernels"] = rk
    if "large_grid" in extra:
        lg = extra.pop("large_grid")
        sub = argparse.Namespace(steps=1)
        rec = {"grid": list(LARGE_GRID), "spinup_steps": LARGE_SPINUP, "arms": {}}
        for name, r in lg.items():
            sub.steps = r.pop("_steps")
            a_, pr = summarize({name: r}, sub, LARGE_GRID, 1, name)
            rec["arms"][name] = {k: a_[name][k] for k in ("steps_per_s", "ms_per_step", "mean_pcg_iterations", "pcg_iterations_per_step",
                                                           "coarse_iterations_per_step", "stages", "step_roofline")}
            rec["arms"][name]["pcg_roofline"] = pr(name)
        line["large_grid"] = rec
    if host_state is not None and "plain" in arms:
        cpu = cpu_steps(host_state, args.shape, budget_s=30.0, max_steps=1)
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
