"""The forward example driver: Python mirror of the reference's
``xayah.examples.smoke.forward`` module (examples/smoke/forward/
simulation.ixx:8-66, simulation.cpp:15-120).

A 128 x 192 x 128 thermal smoke scene driven by two pulsed Gaussian jets
(``xs_smoke_write_control``) and stepped through ``Model.forward_step``; after
every step the example's metrics are reduced on the device
(``xs_smoke_reduce_metrics``) and, with ``host_metrics``, read back:
density mass, density and temperature maxima, maximum centred speed, CFL
number and the RMS divergence before and after the projection.

The reference's example solves the pressure with its fixed count of
red-black Gauss-Seidel sweeps (160); ``pressure_solver`` (an addition)
selects the Jacobi-PCG solve to a relative residual instead.  With a
converged solve, the divergence left after the projection lies entirely in
the top layer of cells: the open top is a p = 0 boundary in the pressure
system, but the projection leaves every boundary face as it is
(operators.cu:904-910), so the outflow through the top is never corrected.
``divergence_by_layer`` reports that split.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np
import torch

from . import _native as N
from .data import Configuration, PressureSolver, ScalarBoundaryMode, VelocityBoundaryMode
from .model import ExecutionMode, Model, fill_parameters, tensors_of


@dataclass
class ForwardSimulationOptions:
    """simulation.ixx:10-29"""
    resolution: Tuple[int, int, int] = (128, 192, 128)
    cell_size: float = 1.0 / 128.0
    time_step: float = 1.0 / 120.0
    pressure_iterations: int = 160
    density_source_rate: float = 4.0
    temperature_source_rate: float = 8.0
    ambient_temperature: float = 0.0
    density_buoyancy: float = -0.1
    temperature_buoyancy: float = 1.0
    vorticity_confinement: float = 2.0
    left_source_center: Tuple[float, float, float] = (0.25, 0.10, 0.36)
    right_source_center: Tuple[float, float, float] = (0.75, 0.10, 0.64)
    source_radius: float = 0.055
    left_acceleration: Tuple[float, float, float] = (3.5, 5.0, 1.8)
    right_acceleration: Tuple[float, float, float] = (-3.5, 5.0, -1.8)
    pulse_period: float = 0.9
    host_metrics: bool = True
    # additions: the pressure solver (the reference's example runs its fixed
    # sweeps) and, for Jacobi-PCG, the relative residual it solves to
    pressure_solver: PressureSolver = PressureSolver.red_black_gauss_seidel
    pressure_tolerance: float = 1.0e-6


@dataclass
class ForwardSimulationMetrics:
    """simulation.ixx:31-44"""
    step: int = 0
    physical_time: float = 0.0
    density_mass: float = 0.0
    density_maximum: float = 0.0
    temperature_maximum: float = 0.0
    maximum_velocity: float = 0.0
    cfl: float = 0.0
    pre_projection_divergence_rms: float = 0.0
    post_projection_divergence_rms: float = 0.0
    divergence_ratio: float = 0.0
    step_milliseconds: float = 0.0
    average_step_milliseconds: float = 0.0


def make_configuration(o: ForwardSimulationOptions) -> Configuration:
    """simulation.cpp:17-33: walls with a fixed normal velocity on every side
    but the top (zero gradient), pressure, density and temperature fixed (0)
    at the top, vorticity confinement on."""
    cfg = Configuration(resolution=list(o.resolution), cell_size=o.cell_size, time_step=o.time_step,
                        pressure_iterations=o.pressure_iterations, vorticity_confinement_enabled=True)
    vb = cfg.velocity_boundary
    for f in (vb.x_min, vb.x_max, vb.y_min, vb.z_min, vb.z_max):
        f.mode = VelocityBoundaryMode.normal_fixed_tangent_zero_gradient
    vb.y_max.mode = VelocityBoundaryMode.zero_gradient
    cfg.pressure_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
    cfg.density_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
    cfg.temperature_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
    cfg.pressure_solver = o.pressure_solver
    cfg.pressure_tolerance = o.pressure_tolerance
    cfg.pressure_max_iterations = 20000
    return cfg


def _vec3(v) -> N.XsVec3:
    return N.XsVec3(*[float(c) for c in v])


def write_control(ctx, control, step: int, o: ForwardSimulationOptions) -> None:
    """simulation_cuda::launch_write_control (simulation.cu:88-92) into a Control."""
    c = control
    N.check("xs_smoke_write_control", N.lib().xs_smoke_write_control(
        ctx.stream_handle, ctx.native.grid, int(step), float(o.pulse_period), _vec3(o.left_source_center), _vec3(o.right_source_center),
        float(o.source_radius), float(o.density_source_rate), float(o.temperature_source_rate), _vec3(o.left_acceleration),
        _vec3(o.right_acceleration), C.c_void_p(c.density_source.values.data_ptr()), C.c_void_p(c.temperature_source.values.data_ptr()),
        N.vec([c.external_acceleration.x.values, c.external_acceleration.y.values, c.external_acceleration.z.values])))


def reduce_metrics(ctx, state, step_cache, metrics: torch.Tensor) -> None:
    """simulation_cuda::launch_reduce_metrics (simulation.cu:95-100) of a step's
    result into metrics[6] (FP64, device)."""
    N.check("xs_smoke_reduce_metrics", N.lib().xs_smoke_reduce_metrics(
        ctx.stream_handle, C.byref(ctx.native), C.c_void_p(state.density.values.data_ptr()),
        C.c_void_p(state.temperature.values.data_ptr()), N.vec(step_cache.advected_velocity.components()),
        N.vec(state.velocity.components()), C.c_void_p(metrics.data_ptr())))


def divergence_by_layer(state, resolution, cell_size: float):
    """Sum of the squared divergence of a state's velocity over the top layer
    of cells (y = ny - 1) and over all the others, in FP64."""
    ux, uy, uz = (t.double() for t in state.velocity.components())
    nx, ny, nz = resolution
    ux = ux.view(nz, ny, nx + 1)
    uy = uy.view(nz, ny + 1, nx)
    uz = uz.view(nz + 1, ny, nx)
    div = ((ux[:, :, 1:] - ux[:, :, :-1]) + (uy[:, 1:, :] - uy[:, :-1, :]) + (uz[1:] - uz[:-1])) / cell_size
    d2 = div * div
    top = float(d2[:, -1, :].sum())
    return top, float(d2.sum()) - top


class ForwardSimulation:
    """simulation.ixx:46-64, simulation.cpp:72-120"""

    def __init__(self, options: Optional[ForwardSimulationOptions] = None):
        self.options = options if options is not None else ForwardSimulationOptions()
        o = self.options
        self.model = Model(make_configuration(o))
        self.context = self.model.allocate_context(ExecutionMode.forward)
        m, ctx = self.model, self.context
        self.current_state = m.allocate_state(ctx)
        self.metrics = ForwardSimulationMetrics()
        self.device_metrics = torch.zeros(6, dtype=torch.float64, device=ctx.device)
        self._next_state = m.allocate_state(ctx)
        self._control = m.allocate_control(ctx)
        self._parameters = fill_parameters(m.allocate_parameters(ctx), ambient_temperature=o.ambient_temperature,
                                           density_buoyancy=o.density_buoyancy, temperature_buoyancy=o.temperature_buoyancy,
                                           vorticity_confinement=o.vorticity_confinement)
        self._step_cache = m.allocate_step_cache(ctx)
        self.reset()

    @property
    def step_cache(self):
        return self._step_cache

    @property
    def control(self):
        return self._control

    def reset(self) -> None:
        """simulation.cpp:80-92: zero both states and the metrics."""
        with torch.cuda.stream(self.context.stream):
            for s in (self.current_state, self._next_state):
                for t in tensors_of(s):
                    t.zero_()
            self.device_metrics.zero_()
        self.context.synchronize()
        self.context.reset_warm_start()
        self.metrics = ForwardSimulationMetrics()

    def step(self) -> None:
        """simulation.cpp:94-120: write the controls of this step, step the
        model, reduce the metrics of the new state and swap."""
        o = self.options
        begin = time.perf_counter() if o.host_metrics else 0.0
        ctx = self.context
        write_control(ctx, self._control, self.metrics.step, o)
        self.model.forward_step(self.current_state, self._control, self._parameters, self._next_state, self._step_cache, ctx)
        reduce_metrics(ctx, self._next_state, self._step_cache, self.device_metrics)
        values = None
        if o.host_metrics:
            values = self.device_metrics.cpu().tolist()
            ctx.synchronize()
        self.current_state, self._next_state = self._next_state, self.current_state
        m = self.metrics
        # the reference's options are FP32 (simulation.ixx:11-12): the metrics
        # use those values widened to FP64
        dt, h = float(np.float32(o.time_step)), float(np.float32(o.cell_size))
        m.step += 1
        m.physical_time = m.step * dt
        if values is None:
            return
        ms = (time.perf_counter() - begin) * 1e3
        previous = m.step - 1
        cells = float(o.resolution[0] * o.resolution[1] * o.resolution[2])
        m.density_mass = values[0] * h * h * h
        m.density_maximum = values[1]
        m.temperature_maximum = values[2]
        m.maximum_velocity = values[3]
        m.cfl = values[3] * dt / h
        m.pre_projection_divergence_rms = (values[4] / cells) ** 0.5
        m.post_projection_divergence_rms = (values[5] / cells) ** 0.5
        m.divergence_ratio = m.post_projection_divergence_rms / m.pre_projection_divergence_rms if m.pre_projection_divergence_rms else 0.0
        m.step_milliseconds = ms
        m.average_step_milliseconds = (previous * m.average_step_milliseconds + ms) / m.step


def main(argv=None) -> int:
    """examples/smoke/forward/main.cpp: 960 steps, metrics every 60."""
    import argparse
    ap = argparse.ArgumentParser(description="128 x 192 x 128 double-jet thermal smoke")
    ap.add_argument("--steps", type=int, default=960)
    ap.add_argument("--every", type=int, default=60)
    ap.add_argument("--pcg", action="store_true", help="Jacobi-PCG to 1e-6 instead of the 160 red-black sweeps")
    a = ap.parse_args(argv)
    o = ForwardSimulationOptions()
    if a.pcg:
        o.pressure_solver = PressureSolver.jacobi_pcg
    free0 = torch.cuda.mem_get_info()[0]
    sim = ForwardSimulation(o)
    print("128 x 192 x 128 double-jet thermal smoke")
    print(f"GPU allocation: {(free0 - torch.cuda.mem_get_info()[0]) / 2 ** 20:.1f} MiB")
    for _ in range(a.steps):
        sim.step()
        m = sim.metrics
        if m.step % a.every:
            continue
        print(f"step {m.step:3d}  time {m.physical_time:.3f} s  density mass {m.density_mass:.6f} max {m.density_maximum:.5f}  "
              f"temperature max {m.temperature_maximum:.5f}  velocity max {m.maximum_velocity:.5f}  CFL {m.cfl:.4f}  "
              f"divergence {m.pre_projection_divergence_rms:.4e} -> {m.post_projection_divergence_rms:.4e} ({m.divergence_ratio:.4f})  "
              f"step {m.step_milliseconds:.3f} ms  average {m.average_step_milliseconds:.3f} ms")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
