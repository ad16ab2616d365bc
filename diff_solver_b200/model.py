"""The smoke model: Python mirror of ``xayah::smoke::Model``
(solvers/smoke/model.ixx:51-96, model.cpp:32-389).

Fields are flat CUDA tensors in the reference layout (cell x + nx*(y + ny*z),
one array per face component with extent +1 on its own axis, FP32 state and
tangents, FP64 adjoints).  Every step runs through the C ABI of
``libdiffsmoke.so`` on the context's CUDA stream (PyTorch's current stream by
default, so PyTorch and the solver stay ordered without synchronisation).
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, fields
from typing import Optional

import torch

from . import _native as N
from .data import Configuration, PressureSolver


class ExecutionMode(enum.IntEnum):
    """model.ixx:10-13"""
    forward = 0
    differentiable = 1


# ----------------------------------------------------------------- fields
@dataclass
class ScalarField:
    values: torch.Tensor


@dataclass
class CenteredVectorField:
    x: ScalarField
    y: ScalarField
    z: ScalarField


@dataclass
class StaggeredVectorField:
    x: torch.Tensor
    y: torch.Tensor
    z: torch.Tensor

    def components(self):
        return (self.x, self.y, self.z)


@dataclass
class State:
    """data.ixx:117-121 (also StateTangent, :136-140)"""
    density: ScalarField
    temperature: ScalarField
    velocity: StaggeredVectorField


@dataclass
class Control:
    """data.ixx:123-127 (also ControlTangent)"""
    density_source: ScalarField
    temperature_source: ScalarField
    external_acceleration: CenteredVectorField


@dataclass
class Parameters:
    """data.ixx:129-134 (also ParameterTangent); one-element device tensors."""
    ambient_temperature: torch.Tensor
    density_buoyancy: torch.Tensor
    temperature_buoyancy: torch.Tensor
    vorticity_confinement: torch.Tensor


@dataclass
class StepCache:
    """data.ixx:189-196; ``vorticity`` is one (11, N) tensor holding centred
    velocity (3), vorticity (3), magnitude, normal (3) and normalizer."""
    sourced_density: ScalarField
    sourced_temperature: ScalarField
    force: CenteredVectorField
    vorticity: torch.Tensor
    forced_velocity: StaggeredVectorField
    advected_velocity: StaggeredVectorField


StateTangent = State
ControlTangent = Control
ParameterTangent = Parameters
StateAdjoint = State        # FP64 tensors
ControlAdjoint = Control    # FP64 tensors
ParameterAdjoint = Parameters  # FP64 tensors


@dataclass
class DeviceDomain:
    """data.ixx:198-204"""
    cell_mask: torch.Tensor
    collider_velocity: StaggeredVectorField
    collider_density: ScalarField
    collider_temperature: ScalarField
    pressure_anchor: int
    has_colliders: bool


class ExecutionContext:
    """model.ixx:17-49: device, stream, domain and the step workspace."""

    def __init__(self, model: "Model", mode: ExecutionMode, device=None, stream: Optional[torch.cuda.Stream] = None):
        self.device = torch.device(device if device is not None else "cuda")
        self.mode = ExecutionMode(mode)
        self._stream = stream
        self.domain: DeviceDomain
        self.workspace: torch.Tensor
        self.native: N.XsSmokeModel
        self._inflows = None
        self._warm_start: Optional[torch.Tensor] = None

    @property
    def stream(self) -> torch.cuda.Stream:
        return self._stream if self._stream is not None else torch.cuda.current_stream(self.device)

    @property
    def stream_handle(self):
        return C.c_void_p(self.stream.cuda_stream)

    def synchronize(self) -> None:
        """cuda.cpp:64-66"""
        self.stream.synchronize()

    def read_solve_stats(self) -> dict:
        """Statistics of the last pressure solve run in this context."""
        st = N.XsSolveStats()
        N.check("xs_smoke_read_solve_stats",
                N.lib().xs_smoke_read_solve_stats(self.stream_handle, C.byref(self.native), C.c_void_p(self.workspace.data_ptr()),
                                                  int(self.mode), C.byref(st), None))
        return st.as_dict()

    def set_warm_start(self, guess: Optional[torch.Tensor]) -> None:
        """Initial guess (N FP32 cells, device) for the next PCG pressure solves;
        None restores the zero guess.  The solve falls back to zero by itself
        whenever the guess' residual exceeds the zero guess'."""
        self._warm_start = guess
        self.native.pressure.initial_guess = None if guess is None else guess.data_ptr()

    def reset_warm_start(self) -> None:
        """Forgets the previous solutions of the Galerkin warm start (a new
        trajectory starts)."""
        N.check("xs_smoke_reset_warm_start", N.lib().xs_smoke_reset_warm_start(self.stream_handle, C.byref(self.native),
                                                                                 C.c_void_p(self.workspace.data_ptr()), int(self.mode)))

    def set_inflow(self, index: int, center=None, radius=None) -> None:
        """Moves or resizes inflow ``index`` for the following steps (the
        inflow table travels to the device with every launch)."""
        if not 0 <= index < int(self.native.inflow_count):
            raise IndexError(index)
        f = self._inflows[index]
        if center is not None:
            f.center[:] = [float(v) for v in center]
        if radius is not None:
            f.radius = float(radius)

    def set_learned_warm_start(self, network) -> None:
        """Warm-start the forward pressure solves with a
        :class:`~diff_solver_b200.warm_start.WarmStartNetwork` whose grid times
        its factor equals this model's grid (None: zero guess).  The guess is
        energy-scaled and PCG falls back to zero whenever it does not help."""
        self._learned = network
        self.native.warm_start = None if network is None else network.handle.value

    def pressure_fields(self):
        """(pressure, rhs) of the last forward pressure solve, as device tensors
        viewing the workspace: the pairs the warm-start network trains on."""
        p, b = C.c_void_p(), C.c_void_p()
        N.check("xs_smoke_pressure_fields", N.lib().xs_smoke_pressure_fields(C.byref(self.native), C.c_void_p(self.workspace.data_ptr()),
                                                                               C.byref(p), C.byref(b)))
        return self._workspace_view(p), self._workspace_view(b)

    def warm_start_fields(self):
        """(x0, b - A x0) of the last forward solve, x0 the Galerkin start from
        the ring of previous solutions (configuration.warm_start_history > 0),
        as device tensors viewing the workspace."""
        x, r = C.c_void_p(), C.c_void_p()
        N.check("xs_smoke_warm_start_fields", N.lib().xs_smoke_warm_start_fields(self.stream_handle, C.byref(self.native),
                                                                                   C.c_void_p(self.workspace.data_ptr()), C.byref(x),
                                                                                   C.byref(r)))
        return self._workspace_view(x), self._workspace_view(r)

    def _workspace_view(self, ptr):
        n = int(self.native.grid.nx) * int(self.native.grid.ny) * int(self.native.grid.nz)
        off = ptr.value - self.workspace.data_ptr()
        return self.workspace[off:off + 4 * n].view(torch.float32)


def _grid(cfg: Configuration) -> N.XsGrid:
    nx, ny, nz = (int(v) for v in cfg.resolution)
    return N.XsGrid(nx, ny, nz, float(cfg.cell_size), float(cfg.time_step))


def scalar_boundary(b) -> N.XsScalarBoundary:
    """operators.cpp:85-93"""
    out = N.XsScalarBoundary()
    for i, f in enumerate(b.faces()):
        out.modes[i] = int(f.mode)
        out.values[i] = float(f.value)
    return out


def velocity_boundary(b) -> N.XsVelocityBoundary:
    """operators.cpp:95-105"""
    out = N.XsVelocityBoundary()
    for i, f in enumerate(b.faces()):
        out.modes[i] = int(f.mode)
        out.values[3 * i + 0] = float(f.value.x)
        out.values[3 * i + 1] = float(f.value.y)
        out.values[3 * i + 2] = float(f.value.z)
    return out


class Model:
    """model.ixx:51-96"""

    def __init__(self, configuration: Configuration):
        self.configuration = configuration
        nx, ny, nz = (int(v) for v in configuration.resolution)
        self.resolution = (nx, ny, nz)
        self.cell_count = nx * ny * nz
        self.face_counts = ((nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))
        if len(configuration.inflows) > N.XS_MAX_INFLOWS:
            raise ValueError(f"at most {N.XS_MAX_INFLOWS} inflows are supported")

    # ------------------------------------------------------------ context
    def allocate_context(self, mode: ExecutionMode = ExecutionMode.forward, device=None,
                         stream: Optional[torch.cuda.Stream] = None) -> ExecutionContext:
        """model.cpp:32-183: domain on the device, pressure anchor, scratch."""
        cfg = self.configuration
        L = N.lib()
        ctx = ExecutionContext(self, mode, device, stream)
        dev = ctx.device
        n = self.cell_count
        mask = torch.zeros(n, dtype=torch.int32, device=dev)
        cv = StaggeredVectorField(*[torch.zeros(f, dtype=torch.float32, device=dev) for f in self.face_counts])
        cd = torch.zeros(n, dtype=torch.float32, device=dev)
        ct = torch.zeros(n, dtype=torch.float32, device=dev)
        cols = (N.XsCollider * max(1, len(cfg.colliders)))()
        for i, k in enumerate(cfg.colliders):
            shp = k.shape
            if hasattr(shp, "radius"):
                cols[i].shape = 0
                cols[i].size[:] = [shp.radius.x, shp.radius.y, shp.radius.z]
            else:
                cols[i].shape = 1
                cols[i].size[:] = [shp.half_extent.x, shp.half_extent.y, shp.half_extent.z]
            cols[i].center[:] = [shp.center.x, shp.center.y, shp.center.z]
            cols[i].velocity[:] = [k.velocity.x, k.velocity.y, k.velocity.z]
            cols[i].density = k.density
            cols[i].temperature = k.temperature
        anchor = C.c_uint32(0)
        pb = scalar_boundary(cfg.pressure_boundary)
        N.check("xs_smoke_build_domain",
                L.xs_smoke_build_domain(ctx.stream_handle, _grid(cfg), pb, C.cast(cols, C.c_void_p), len(cfg.colliders), mask.data_ptr(),
                                        N.vec(cv.components()), cd.data_ptr(), ct.data_ptr(), C.byref(anchor)))
        has_colliders = len(cfg.colliders) > 0
        ctx.domain = DeviceDomain(mask, cv, ScalarField(cd), ScalarField(ct), int(anchor.value), has_colliders)
        m = N.XsSmokeModel()
        m.grid = _grid(cfg)
        m.velocity_boundary = velocity_boundary(cfg.velocity_boundary)
        m.pressure_boundary = pb
        m.density_boundary = scalar_boundary(cfg.density_boundary)
        m.temperature_boundary = scalar_boundary(cfg.temperature_boundary)
        m.vorticity_confinement_enabled = 1 if cfg.vorticity_confinement_enabled else 0
        m.pressure_anchor = ctx.domain.pressure_anchor
        if int(cfg.pressure_solver) == int(PressureSolver.red_black_gauss_seidel):
            m.pressure = N.XsPressureSolve(N.XS_SOLVER_RED_BLACK_GAUSS_SEIDEL, int(cfg.pressure_iterations), 0.0, None)
        else:
            m.pressure = N.XsPressureSolve(N.XS_SOLVER_JACOBI_PCG, int(cfg.pressure_max_iterations), float(cfg.pressure_tolerance), None)
        inflows = (N.XsInflow * max(1, len(cfg.inflows)))()
        for i, f in enumerate(cfg.inflows):
            inflows[i].center[:] = [f.center.x, f.center.y, f.center.z]
            inflows[i].radius = f.radius
            inflows[i].density = f.density
            inflows[i].temperature = f.temperature
        ctx._inflows = inflows
        m.inflows = C.cast(inflows, C.c_void_p)
        m.inflow_count = len(cfg.inflows)
        m.cell_mask = mask.data_ptr() if has_colliders else None
        m.collider_velocity = N.vec(cv.components()) if has_colliders else N.XsVector(None, None, None)
        m.collider_density = cd.data_ptr() if has_colliders else None
        m.collider_temperature = ct.data_ptr() if has_colliders else None
        m.warm_start_history = int(cfg.warm_start_history)
        m.warm_start_coarsening = int(cfg.warm_start_coarsening)
        m.warm_start_rounds = int(cfg.warm_start_rounds)
        ctx.native = m
        nbytes = L.xs_smoke_workspace_bytes(C.byref(m), int(mode))
        if nbytes == 0:
            raise ValueError("invalid model configuration (grid, inflows or warm-start history)")
        ctx.workspace = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        ctx.reset_warm_start()
        return ctx

    # ------------------------------------------------------------ allocation
    def _scalar(self, ctx, dtype=torch.float32):
        return ScalarField(torch.zeros(self.cell_count, dtype=dtype, device=ctx.device))

    def _centered(self, ctx, dtype=torch.float32):
        return CenteredVectorField(self._scalar(ctx, dtype), self._scalar(ctx, dtype), self._scalar(ctx, dtype))

    def _staggered(self, ctx, dtype=torch.float32):
        return StaggeredVectorField(*[torch.zeros(f, dtype=dtype, device=ctx.device) for f in self.face_counts])

    def _params(self, ctx, dtype):
        return Parameters(*[torch.zeros(1, dtype=dtype, device=ctx.device) for _ in range(4)])

    def allocate_state(self, ctx) -> State:
        return State(self._scalar(ctx), self._scalar(ctx), self._staggered(ctx))

    def allocate_control(self, ctx) -> Control:
        return Control(self._scalar(ctx), self._scalar(ctx), self._centered(ctx))

    def allocate_parameters(self, ctx) -> Parameters:
        return self._params(ctx, torch.float32)

    def allocate_step_cache(self, ctx) -> StepCache:
        return StepCache(self._scalar(ctx), self._scalar(ctx), self._centered(ctx),
                         torch.zeros((11, self.cell_count), dtype=torch.float32, device=ctx.device),
                         self._staggered(ctx), self._staggered(ctx))

    def allocate_state_tangent(self, ctx) -> State:
        return self.allocate_state(ctx)

    def allocate_control_tangent(self, ctx) -> Control:
        return self.allocate_control(ctx)

    def allocate_parameter_tangent(self, ctx) -> Parameters:
        return self._params(ctx, torch.float32)

    def allocate_state_adjoint(self, ctx) -> State:
        return State(self._scalar(ctx, torch.float64), self._scalar(ctx, torch.float64), self._staggered(ctx, torch.float64))

    def allocate_control_adjoint(self, ctx) -> Control:
        return Control(self._scalar(ctx, torch.float64), self._scalar(ctx, torch.float64), self._centered(ctx, torch.float64))

    def allocate_parameter_adjoint(self, ctx) -> Parameters:
        return self._params(ctx, torch.float64)

    # ------------------------------------------------------------ copies
    @staticmethod
    def _state_tensors(s: State):
        return [s.density.values, s.temperature.values, s.velocity.x, s.velocity.y, s.velocity.z]

    def copy_state(self, source: State, destination: State, ctx) -> None:
        with torch.cuda.stream(ctx.stream):
            for a, b in zip(self._state_tensors(source), self._state_tensors(destination)):
                b.copy_(a, non_blocking=True)

    copy_state_tangent = copy_state
    copy_state_adjoint = copy_state

    def zero_state_adjoint(self, state: State, ctx) -> None:
        with torch.cuda.stream(ctx.stream):
            for t in self._state_tensors(state):
                t.zero_()

    def accumulate_state_adjoint(self, source: State, destination: State, ctx) -> None:
        """model.cpp:332-339 (xs_accumulate on each component)."""
        L = N.lib()
        for a, b in zip(self._state_tensors(source), self._state_tensors(destination)):
            N.check("xs_accumulate", L.xs_accumulate(ctx.stream_handle, a.data_ptr(), b.data_ptr(), a.numel()))

    # ------------------------------------------------------------ views
    @staticmethod
    def _state(s: State) -> N.XsState:
        return N.XsState(s.density.values.data_ptr(), s.temperature.values.data_ptr(), N.vec(s.velocity.components()))

    @staticmethod
    def _control(c: Control) -> N.XsControl:
        a = c.external_acceleration
        return N.XsControl(c.density_source.values.data_ptr(), c.temperature_source.values.data_ptr(),
                           N.vec((a.x.values, a.y.values, a.z.values)))

    @staticmethod
    def _params_view(p: Parameters) -> N.XsParameters:
        return N.XsParameters(p.ambient_temperature.data_ptr(), p.density_buoyancy.data_ptr(), p.temperature_buoyancy.data_ptr(),
                              p.vorticity_confinement.data_ptr())

    @staticmethod
    def _cache(k: StepCache) -> N.XsStepCache:
        f = k.force
        return N.XsStepCache(k.sourced_density.values.data_ptr(), k.sourced_temperature.values.data_ptr(),
                             N.vec((f.x.values, f.y.values, f.z.values)), k.vorticity.data_ptr(),
                             N.vec(k.forced_velocity.components()), N.vec(k.advected_velocity.components()))

    # ------------------------------------------------------------ steps
    def forward_step(self, state: State, control: Control, parameters: Parameters, next_state: State, step_cache: StepCache,
                     ctx: ExecutionContext) -> None:
        """model.cpp:341-349"""
        N.check("xs_smoke_forward_step",
                N.lib().xs_smoke_forward_step(ctx.stream_handle, C.byref(ctx.native), self._state(state), self._control(control),
                                              self._params_view(parameters), self._state(next_state), self._cache(step_cache),
                                              C.c_void_p(ctx.workspace.data_ptr())))

    def jvp_step(self, state: State, control: Control, parameters: Parameters, next_state: State, step_cache: StepCache,
                 state_tangent: State, control_tangent: Control, parameter_tangent: Parameters, next_state_tangent: State,
                 ctx: ExecutionContext) -> None:
        """model.cpp:351-359"""
        self._require_differentiable(ctx)
        N.check("xs_smoke_jvp_step",
                N.lib().xs_smoke_jvp_step(ctx.stream_handle, C.byref(ctx.native), self._state(state), self._params_view(parameters),
                                          self._state(next_state), self._cache(step_cache), self._state(state_tangent),
                                          self._control(control_tangent), self._params_view(parameter_tangent),
                                          self._state(next_state_tangent), C.c_void_p(ctx.workspace.data_ptr())))

    def vjp_step(self, state: State, control: Control, parameters: Parameters, next_state: State, step_cache: StepCache,
                 next_state_adjoint: State, previous_state_adjoint: State, control_adjoint: Control, parameter_adjoint: Parameters,
                 ctx: ExecutionContext) -> None:
        """model.cpp:361-389; accumulates into the three adjoint outputs."""
        self._require_differentiable(ctx)
        N.check("xs_smoke_vjp_step",
                N.lib().xs_smoke_vjp_step(ctx.stream_handle, C.byref(ctx.native), self._state(state), self._params_view(parameters),
                                          self._state(next_state), self._cache(step_cache), self._state(next_state_adjoint),
                                          self._state(previous_state_adjoint), self._control(control_adjoint),
                                          self._params_view(parameter_adjoint), C.c_void_p(ctx.workspace.data_ptr())))

    @staticmethod
    def _require_differentiable(ctx):
        if ctx.mode != ExecutionMode.differentiable:
            raise ValueError("jvp_step / vjp_step need a context allocated with ExecutionMode.differentiable")


def fill_parameters(p: Parameters, ambient_temperature=0.0, density_buoyancy=0.0, temperature_buoyancy=0.0, vorticity_confinement=0.0):
    for t, v in zip((p.ambient_temperature, p.density_buoyancy, p.temperature_buoyancy, p.vorticity_confinement),
                    (ambient_temperature, density_buoyancy, temperature_buoyancy, vorticity_confinement)):
        t.fill_(float(v))
    return p


def tensors_of(obj):
    """Flat list of the tensors of a field dataclass, in declaration order."""
    out = []
    if isinstance(obj, torch.Tensor):
        return [obj]
    for f in fields(obj):
        out.extend(tensors_of(getattr(obj, f.name)))
    return out
