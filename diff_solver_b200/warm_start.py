"""Learned pressure warm start (no reference counterpart).

:class:`WarmStartNetwork` holds the native U-Net (``xs_warm_start_*`` in
``include/diff_smoke.h``: tcgen05 convolutions, hand-written backward pass and
Adam, all on the GPU).  :func:`train_on_plumes` trains it on (right-hand side,
pressure) pairs that the plain PCG solver produces while it runs plume
simulations with seeded random inflow centre, radius and buoyancy.

A model uses a trained network through
``ExecutionContext.set_learned_warm_start``: every forward pressure solve
then restricts its right-hand side to the network grid, runs the network,
prolongs the output, scales it by the energy-optimal factor and starts PCG
from it, falling back to a zero guess whenever that is not better.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np
import torch

from . import _native as N


class WarmStartNetwork:
    """Handle of the native warm-start network on the grid ``shape`` (nx, ny,
    nz, each a multiple of 8 with at least 128 cells per x-y plane at 1/8 of
    the resolution).  ``factor`` is the ratio of a fluid grid to this grid
    when the network serves a model."""

    def __init__(self, shape: Sequence[int], max_batch: int = 1, factor: int = 1, seed: int = 0, stream: Optional[torch.cuda.Stream] = None):
        self.shape = tuple(int(v) for v in shape)
        self.max_batch = int(max_batch)
        self.factor = int(factor)
        self._stream = stream
        self.handle = C.c_void_p()
        N.check("xs_warm_start_create", N.lib().xs_warm_start_create(C.byref(self.handle), self.max_batch, *self.shape, self.factor))
        N.check("xs_warm_start_initialize", N.lib().xs_warm_start_initialize(self.handle, self.stream_handle, int(seed)))

    # ------------------------------------------------------------ plumbing
    @property
    def stream(self) -> torch.cuda.Stream:
        return self._stream if self._stream is not None else torch.cuda.current_stream()

    @property
    def stream_handle(self):
        return C.c_void_p(self.stream.cuda_stream)

    @property
    def cells(self) -> int:
        return self.shape[0] * self.shape[1] * self.shape[2]

    @staticmethod
    def parameter_count() -> int:
        return int(N.lib().xs_warm_start_parameter_count())

    def close(self) -> None:
        if self.handle and self.handle.value:
            N.lib().xs_warm_start_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ parameters
    def parameters(self) -> np.ndarray:
        out = np.empty(self.parameter_count(), dtype=np.float32)
        N.check("xs_warm_start_get_parameters", N.lib().xs_warm_start_get_parameters(self.handle, self.stream_handle, out.ctypes.data))
        return out

    def set_parameters(self, values: np.ndarray) -> None:
        values = np.ascontiguousarray(values, dtype=np.float32)
        if values.size != self.parameter_count():
            raise ValueError(f"expected {self.parameter_count()} parameters, got {values.size}")
        N.check("xs_warm_start_set_parameters", N.lib().xs_warm_start_set_parameters(self.handle, self.stream_handle, values.ctypes.data))

    def save(self, path: str, **metadata) -> None:
        np.savez(path, parameters=self.parameters(), grid=np.array(self.shape), **{k: np.asarray(v) for k, v in metadata.items()})

    def load(self, path: str) -> dict:
        with np.load(path) as f:
            self.set_parameters(f["parameters"])
            return {k: f[k] for k in f.files if k != "parameters"}

    # ------------------------------------------------------------ compute
    def _check_batch(self, t: torch.Tensor) -> int:
        if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous():
            raise ValueError("expected a contiguous CUDA float32 tensor")
        if t.numel() % self.cells:
            raise ValueError(f"size {t.numel()} is not a whole number of {self.cells}-cell samples")
        b = t.numel() // self.cells
        if not 1 <= b <= self.max_batch:
            raise ValueError(f"batch {b} outside 1..{self.max_batch}")
        return b

    def predict(self, rhs: torch.Tensor) -> torch.Tensor:
        """Network output (channel 0) for a batch of right-hand sides on the
        network grid, in units of the predicted pressure's RMS."""
        b = self._check_batch(rhs)
        out = torch.empty_like(rhs)
        N.check("xs_warm_start_predict", N.lib().xs_warm_start_predict(self.handle, self.stream_handle, b, rhs.data_ptr(), out.data_ptr()))
        return out

    def gradient(self, rhs: torch.Tensor, pressure: torch.Tensor):
        """(loss, gradient) of mean (out - p / rms(p))^2 (device tensors)."""
        b = self._check_batch(rhs)
        if pressure.shape != rhs.shape:
            raise ValueError("rhs and pressure differ in shape")
        grad = torch.empty(self.parameter_count(), dtype=torch.float32, device=rhs.device)
        loss = torch.empty(1, dtype=torch.float64, device=rhs.device)
        N.check("xs_warm_start_gradient", N.lib().xs_warm_start_gradient(self.handle, self.stream_handle, b, rhs.data_ptr(),
                                                                         pressure.contiguous().data_ptr(), grad.data_ptr(), loss.data_ptr()))
        return loss, grad

    def set_loss(self, kind: str, pressure_boundary: Optional[N.XsScalarBoundary] = None) -> None:
        """``"l2"``: mean (out - p / rms(p))^2; ``"energy"``: the squared
        relative A-norm error of the energy-optimally scaled guess, with A the
        pressure operator of the network grid under ``pressure_boundary``."""
        k = {"l2": 0, "energy": 1}[kind]
        pb = pressure_boundary if pressure_boundary is not None else N.XsScalarBoundary()
        N.check("xs_warm_start_set_loss", N.lib().xs_warm_start_set_loss(self.handle, k, pb))

    def adam_step(self, learning_rate: float, beta1: float = 0.9, beta2: float = 0.999, epsilon: float = 1e-8) -> None:
        N.check("xs_warm_start_adam_step", N.lib().xs_warm_start_adam_step(self.handle, self.stream_handle, learning_rate, beta1, beta2,
                                                                           epsilon))

    def train_step(self, rhs: torch.Tensor, pressure: torch.Tensor, learning_rate: float, loss: Optional[torch.Tensor] = None):
        b = self._check_batch(rhs)
        if loss is None:
            loss = torch.empty(1, dtype=torch.float64, device=rhs.device)
        N.check("xs_warm_start_train_step", N.lib().xs_warm_start_train_step(self.handle, self.stream_handle, b, rhs.data_ptr(),
                                                                             pressure.data_ptr(), learning_rate, loss.data_ptr()))
        return loss

    def guess(self, grid: N.XsGrid, rhs: torch.Tensor) -> torch.Tensor:
        """Prolonged network guess for a right-hand side on a fluid grid of
        ``factor`` x the network grid (before the solver's energy scaling)."""
        out = torch.empty_like(rhs)
        N.check("xs_warm_start_guess", N.lib().xs_warm_start_guess(self.handle, self.stream_handle, grid, rhs.data_ptr(), out.data_ptr()))
        return out

    def check(self) -> None:
        """Synchronises and raises if a bounded wait inside a network kernel expired."""
        N.check("xs_warm_start_status", N.lib().xs_warm_start_status(self.handle, self.stream_handle))


# ---------------------------------------------------------------- training
@dataclass
class PlumeSampler:
    """Seeded uniform ranges of the training plumes: inflow centre, radius and
    temperature buoyancy (density buoyancy stays -0.1)."""
    centre_low: tuple = (0.3, 0.06, 0.3)
    centre_high: tuple = (0.7, 0.2, 0.7)
    radius: tuple = (0.05, 0.12)
    buoyancy: tuple = (0.2, 1.0)

    def draw(self, rng: np.random.Generator):
        c = tuple(float(rng.uniform(lo, hi)) for lo, hi in zip(self.centre_low, self.centre_high))
        return c, float(rng.uniform(*self.radius)), float(rng.uniform(*self.buoyancy))


class _Plume:
    """One running plume simulation that yields a (rhs, pressure) pair per step."""

    def __init__(self, resolution, rng: np.random.Generator, sampler: PlumeSampler, stream, history: int = 0):
        from .data import plume_configuration
        from .model import ExecutionMode, Model, fill_parameters
        self.rng = rng
        self.sampler = sampler
        centre, radius, buoyancy = sampler.draw(rng)
        cfg = plume_configuration(tuple(resolution), inflow_center=centre, inflow_radius=radius)
        cfg.warm_start_history = int(history)
        self.model = Model(cfg)
        self.ctx = self.model.allocate_context(ExecutionMode.forward, stream=stream)
        self.state = self.model.allocate_state(self.ctx)
        self.next = self.model.allocate_state(self.ctx)
        self.control = self.model.allocate_control(self.ctx)
        self.params = self.model.allocate_parameters(self.ctx)
        self.cache = self.model.allocate_step_cache(self.ctx)
        fill_parameters(self.params, ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=buoyancy)
        self.steps = 0
        self._reset_state()

    def _reset_state(self):
        seed = int(self.rng.integers(1 << 31))
        g = torch.Generator(device="cpu").manual_seed(seed)
        with torch.cuda.stream(self.ctx.stream):
            for t in (self.state.density.values, self.state.temperature.values):
                t.zero_()
            for t in self.state.velocity.components():
                t.copy_((torch.rand(t.shape, generator=g) * 0.02 - 0.01).to(t.device))
        self.ctx.reset_warm_start()
        self.steps = 0

    def restart(self):
        from .model import fill_parameters
        centre, radius, buoyancy = self.sampler.draw(self.rng)
        self.ctx.set_inflow(0, center=centre, radius=radius)
        fill_parameters(self.params, ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=buoyancy)
        self._reset_state()

    def step(self):
        self.model.forward_step(self.state, self.control, self.params, self.next, self.cache, self.ctx)
        self.state, self.next = self.next, self.state
        self.steps += 1
        return self.ctx.pressure_fields()


def train_on_plumes(network: WarmStartNetwork, pairs: int = 20000, batch: int = 8, learning_rate: float = 1e-3,
                    buffer_size: int = 256, episode_steps: int = 200, warmup_pairs: int = 64, seed: int = 0,
                    log: Optional[Callable[[dict], None]] = None, log_every: int = 50, loss: str = "energy",
                    history: int = 0, fine_factor: int = 1) -> List[dict]:
    """Trains ``network`` on ``pairs`` pairs generated by the PCG solver:
    ``batch`` plumes run side by side, each step adds their pairs to a replay
    buffer of ``buffer_size`` pairs in device memory, and one Adam step runs
    on ``batch`` pairs drawn from the buffer.  A plume restarts with new
    random parameters after ``episode_steps`` steps.

    With ``history`` = 0 the pairs are (rhs, pressure) of plain solves; with
    a ring of ``history`` previous solutions they are (b - A x0, p - x0), x0
    the ring's Galerkin start: the correction the network supplies when it
    serves a model that keeps a ring.  With ``fine_factor`` f > 1 the plumes
    run on a grid f times the network's and both members of a pair are
    restricted to the network grid by summing the f^3 children (the
    restriction the solver applies to the network's input).  Returns the
    logged records."""
    if network.max_batch < batch:
        raise ValueError(f"the network was created for batches of at most {network.max_batch}")
    rng = np.random.default_rng(seed)
    sampler = PlumeSampler()
    stream = network.stream
    n = network.cells
    dev = torch.device("cuda")
    f = int(fine_factor)
    fine_shape = tuple(f * s for s in network.shape)
    plumes = [_Plume(fine_shape, rng, sampler, stream, history=history) for _ in range(batch)]

    def coarse(v):
        if f == 1:
            return v
        nx, ny, nz = network.shape
        return v.view(nz, f, ny, f, nx, f).sum(dim=(1, 3, 5)).reshape(-1)
    network.set_loss(loss, plumes[0].ctx.native.pressure_boundary)
    # stagger the episodes so the buffer mixes early and developed plumes
    for i, p in enumerate(plumes):
        p.steps = -(i * episode_steps // batch)
    buf_rhs = torch.empty(buffer_size, n, dtype=torch.float32, device=dev)
    buf_p = torch.empty(buffer_size, n, dtype=torch.float32, device=dev)
    filled, head, generated = 0, 0, 0
    records: List[dict] = []
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    t0 = time.perf_counter()
    it = 0
    with torch.cuda.stream(stream):
        while generated < pairs:
            for p in plumes:
                if p.steps >= episode_steps:
                    p.restart()
                pressure, rhs = p.step()
                if p.steps <= 0:
                    continue
                if history:
                    x0, r0 = p.ctx.warm_start_fields()
                    buf_rhs[head].copy_(coarse(r0))
                    buf_p[head].copy_(coarse(pressure - x0))
                else:
                    buf_rhs[head].copy_(coarse(rhs))
                    buf_p[head].copy_(coarse(pressure))
                head = (head + 1) % buffer_size
                filled = min(filled + 1, buffer_size)
                generated += 1
            if filled < min(warmup_pairs, buffer_size):
                continue
            idx = torch.from_numpy(rng.integers(0, filled, size=batch)).to(dev)
            b_rhs = buf_rhs.index_select(0, idx)
            b_p = buf_p.index_select(0, idx)
            network.train_step(b_rhs, b_p, learning_rate, loss)
            it += 1
            if log_every and it % log_every == 0:
                rec = {"iteration": it, "pairs": generated, "loss": float(loss.item()), "seconds": time.perf_counter() - t0}
                records.append(rec)
                if log:
                    log(rec)
    network.check()
    return records


def evaluate_on_plume(network: WarmStartNetwork, resolution: Sequence[int], steps: int = 100, every: int = 10,
                      centre=(0.5, 0.1, 0.5), radius: float = 0.08, buoyancy: float = 0.5, seed: int = 1234) -> List[dict]:
    """Runs the plain-PCG plume on ``resolution`` (the network grid times its
    factor) for ``steps`` steps and, every ``every`` steps, solves that
    step's pressure problem again from the network's energy-scaled guess.
    Returns one record per evaluated step: the plain and the learned PCG
    iteration counts and the learned start's relative residual."""
    rng = np.random.default_rng(seed)
    sampler = PlumeSampler(centre_low=tuple(centre), centre_high=tuple(centre), radius=(radius, radius), buoyancy=(buoyancy, buoyancy))
    stream = network.stream
    plume = _Plume(resolution, rng, sampler, stream)
    grid = plume.ctx.native.grid
    out: List[dict] = []
    with torch.cuda.stream(stream):
        for s in range(1, steps + 1):
            _, rhs = plume.step()
            if s % every:
                continue
            plain = plume.ctx.read_solve_stats()
            learned = solve_iterations(plume.model, plume.ctx, rhs, network.guess(grid, rhs))
            out.append({"step": s, "plain_iterations": plain["iterations"], "learned_iterations": learned["iterations"],
                        "learned_initial_residual": learned["initial_residual"], "warm_start_used": learned["warm_start_used"],
                        "guess_scale": learned["guess_scale"], "learned_final_residual": learned["final_residual"]})
    network.check()
    return out


def evaluate_arms(network: Optional[WarmStartNetwork], resolution: Sequence[int], steps: int = 100, history: int = 4,
                  centre=(0.5, 0.1, 0.5), radius: float = 0.08, buoyancy: float = 0.5, seed: int = 1234) -> dict:
    """Runs the same plume side by side with the forward solve started from
    zero ("plain"), from the Galerkin combination of the last ``history``
    solutions ("history"), from the learned guess alone ("learned") and from
    both ("learned+history"), and returns each arm's per-step PCG iteration
    counts.  The arms' states agree within the solver tolerance."""
    sampler = PlumeSampler(centre_low=tuple(centre), centre_high=tuple(centre), radius=(radius, radius), buoyancy=(buoyancy, buoyancy))
    stream = network.stream if network is not None else torch.cuda.current_stream()
    arms = {"plain": (0, False), "history": (history, False)}
    if network is not None:
        arms.update({"learned": (0, True), "learned+history": (history, True)})
    plumes = {}
    for name, (h, learned) in arms.items():
        p = _Plume(resolution, np.random.default_rng(seed), sampler, stream, history=h)
        if learned:
            p.ctx.set_learned_warm_start(network)
        plumes[name] = p
    out = {name: [] for name in arms}
    with torch.cuda.stream(stream):
        for _ in range(steps):
            for name, p in plumes.items():
                p.step()
                out[name].append(int(p.ctx.read_solve_stats()["iterations"]))
    if network is not None:
        network.check()
    return out


def solve_iterations(model, ctx, rhs: torch.Tensor, guess: Optional[torch.Tensor], scale: bool = True) -> dict:
    """PCG statistics of one pressure solve of ``rhs`` on ``model``'s grid from
    ``guess`` (None: zero), through xs_pressure_solve."""
    lib = N.lib()
    g = ctx.native.grid
    solve = N.XsPressureSolve(N.XS_SOLVER_JACOBI_PCG, int(model.configuration.pressure_max_iterations),
                              float(model.configuration.pressure_tolerance), None if guess is None else guess.data_ptr(),
                              1 if scale else 0)
    n = rhs.numel()
    ws = torch.empty(lib.xs_projection_workspace_bytes(g), dtype=torch.uint8, device=rhs.device)
    p = torch.empty(n, dtype=torch.float32, device=rhs.device)
    N.check("xs_pressure_solve", lib.xs_pressure_solve(ctx.stream_handle, g, C.byref(solve), ctx.native.pressure_anchor,
                                                       ctx.native.cell_mask, ctx.native.pressure_boundary, rhs.data_ptr(), p.data_ptr(),
                                                       ws.data_ptr()))
    st = N.XsSolveStats()
    N.check("xs_read_solve_stats", lib.xs_read_solve_stats(ctx.stream_handle, C.c_void_p(ws.data_ptr()), C.byref(st)))
    return st.as_dict()
