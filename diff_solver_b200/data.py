"""Smoke solver data layout: configuration, boundaries, colliders and fields.

Python mirror of the reference module ``xayah.smoke.data``
(solvers/smoke/data.ixx:8-204).  Enum values are fixed by the reference
(data.ixx:14-25) because they cross the C ABI unchanged.

Additions with no reference counterpart, all defaulting to "off":

* ``Configuration.inflows``: spheres whose cells are *set* to a density and
  temperature before the step (the reference only has additive sources,
  operators.cu:286-290);
* ``Configuration.pressure_solver`` with ``pressure_tolerance`` and
  ``pressure_max_iterations``: the Jacobi-PCG solve that replaces the fixed
  red-black Gauss-Seidel sweep count (operators.cu:1004-1013), and
  ``PressureSolver.red_black_gauss_seidel`` which keeps the reference's
  fixed-count sweeps;
* ``Configuration.warm_start``: the learned pressure warm start.
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import List, Union


@dataclass
class Vector3:
    """data.ixx:8-12"""
    x: float = 0.0
    y: float = 0.0
    z: float = 0.0


class ScalarBoundaryMode(enum.IntEnum):
    """data.ixx:14-18"""
    fixed_value = 0
    zero_gradient = 1
    periodic = 2


class VelocityBoundaryMode(enum.IntEnum):
    """data.ixx:20-25"""
    fixed_value = 0
    zero_gradient = 1
    normal_fixed_tangent_zero_gradient = 2
    periodic = 3


@dataclass
class ScalarBoundaryFace:
    """data.ixx:27-30"""
    mode: ScalarBoundaryMode = ScalarBoundaryMode.zero_gradient
    value: float = 0.0


@dataclass
class VelocityBoundaryFace:
    """data.ixx:32-35"""
    mode: VelocityBoundaryMode = VelocityBoundaryMode.zero_gradient
    value: Vector3 = field(default_factory=Vector3)


@dataclass
class ScalarBoundary:
    """data.ixx:37-44; faces in the packing order x-, x+, y-, y+, z-, z+"""
    x_min: ScalarBoundaryFace = field(default_factory=ScalarBoundaryFace)
    x_max: ScalarBoundaryFace = field(default_factory=ScalarBoundaryFace)
    y_min: ScalarBoundaryFace = field(default_factory=ScalarBoundaryFace)
    y_max: ScalarBoundaryFace = field(default_factory=ScalarBoundaryFace)
    z_min: ScalarBoundaryFace = field(default_factory=ScalarBoundaryFace)
    z_max: ScalarBoundaryFace = field(default_factory=ScalarBoundaryFace)

    def faces(self):
        return (self.x_min, self.x_max, self.y_min, self.y_max, self.z_min, self.z_max)


@dataclass
class VelocityBoundary:
    """data.ixx:46-53"""
    x_min: VelocityBoundaryFace = field(default_factory=VelocityBoundaryFace)
    x_max: VelocityBoundaryFace = field(default_factory=VelocityBoundaryFace)
    y_min: VelocityBoundaryFace = field(default_factory=VelocityBoundaryFace)
    y_max: VelocityBoundaryFace = field(default_factory=VelocityBoundaryFace)
    z_min: VelocityBoundaryFace = field(default_factory=VelocityBoundaryFace)
    z_max: VelocityBoundaryFace = field(default_factory=VelocityBoundaryFace)

    def faces(self):
        return (self.x_min, self.x_max, self.y_min, self.y_max, self.z_min, self.z_max)


@dataclass
class Ellipsoid:
    """data.ixx:55-58"""
    center: Vector3 = field(default_factory=Vector3)
    radius: Vector3 = field(default_factory=lambda: Vector3(1.0, 1.0, 1.0))


@dataclass
class Box:
    """data.ixx:60-63"""
    center: Vector3 = field(default_factory=Vector3)
    half_extent: Vector3 = field(default_factory=lambda: Vector3(1.0, 1.0, 1.0))


@dataclass
class Collider:
    """data.ixx:65-70"""
    shape: Union[Ellipsoid, Box] = field(default_factory=Ellipsoid)
    velocity: Vector3 = field(default_factory=Vector3)
    density: float = 0.0
    temperature: float = 0.0


@dataclass
class Inflow:
    """Sphere whose cells (tested at cell centres) are set to ``density`` and
    ``temperature`` at the start of every step, before buoyancy."""
    center: Vector3 = field(default_factory=Vector3)
    radius: float = 0.0
    density: float = 1.0
    temperature: float = 1.0


class PressureSolver(enum.IntEnum):
    jacobi_pcg = 0
    red_black_gauss_seidel = 1


class WarmStart(enum.IntEnum):
    none = 0
    learned = 1


@dataclass
class Configuration:
    """data.ixx:72-83 plus the pressure-solver, inflow and warm-start fields."""
    resolution: List[int] = field(default_factory=lambda: [32, 48, 32])
    cell_size: float = 1.0 / 32.0
    time_step: float = 1.0 / 60.0
    pressure_iterations: int = 80
    velocity_boundary: VelocityBoundary = field(default_factory=VelocityBoundary)
    pressure_boundary: ScalarBoundary = field(default_factory=ScalarBoundary)
    density_boundary: ScalarBoundary = field(default_factory=ScalarBoundary)
    temperature_boundary: ScalarBoundary = field(default_factory=ScalarBoundary)
    colliders: List[Collider] = field(default_factory=list)
    vorticity_confinement_enabled: bool = True
    # additions
    inflows: List[Inflow] = field(default_factory=list)
    pressure_solver: PressureSolver = PressureSolver.jacobi_pcg
    pressure_tolerance: float = 1.0e-6
    pressure_max_iterations: int = 4000
    warm_start: WarmStart = WarmStart.none
    # previous forward solutions kept for the Galerkin start of the next
    # forward PCG solve (0..5; 0: off)
    warm_start_history: int = 0
    # coarse-grid correction of that start (0: off; else the coarsening
    # factor per axis, dividing the grid; needs a ring and no colliders)
    warm_start_coarsening: int = 0
    # rounds of sweeps and coarse-grid correction before a forward solve (0: defaults)
    warm_start_rounds: int = 0


def plume_configuration(n=(64, 64, 64), cell_size=None, inflow_center=(0.5, 0.1, 0.5), inflow_radius=0.08,
                        vorticity=False) -> Configuration:
    """The synthetic plume of the benchmark configurations: walls with a fixed
    normal velocity on the sides and bottom, an open top (p = 0, zero-gradient
    velocity, density and temperature fixed at 0 outside), dt = 0.5 dx and an
    inflow sphere that sets density = temperature = 1.  The boundary set is the
    one of examples/smoke/forward/simulation.cpp:27-33."""
    nx, ny, nz = n
    h = cell_size if cell_size is not None else 1.0 / nx
    cfg = Configuration(resolution=[nx, ny, nz], cell_size=h, time_step=0.5 * h, vorticity_confinement_enabled=vorticity)
    vb = cfg.velocity_boundary
    for f in (vb.x_min, vb.x_max, vb.y_min, vb.z_min, vb.z_max):
        f.mode = VelocityBoundaryMode.normal_fixed_tangent_zero_gradient
    vb.y_max.mode = VelocityBoundaryMode.zero_gradient
    cfg.pressure_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
    cfg.density_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
    cfg.temperature_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
    cfg.inflows = [Inflow(Vector3(*inflow_center), inflow_radius, 1.0, 1.0)]
    return cfg
