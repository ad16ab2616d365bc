"""Shared helpers of the test suite: scenario configurations, seeded inputs,
conversions between product tensors and oracle arrays, error metrics."""
from __future__ import annotations

import copy
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from diff_solver_b200.data import (Box, Collider, Configuration, Ellipsoid, Inflow, PressureSolver, ScalarBoundaryMode,  # noqa: E402
                                   Vector3, VelocityBoundaryMode, plume_configuration)

PARAMS = dict(ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=0.5, vorticity_confinement=2.0)


def scenario(name: str, res=(16, 14, 12)) -> Configuration:
    """Small test problems covering every boundary mode the reference has."""
    nx, ny, nz = res
    h = 1.0 / nx
    if name == "plume":
        cfg = plume_configuration(res, cell_size=h, inflow_center=(0.5, 0.15, 0.4), inflow_radius=0.2)
    elif name == "vorticity":
        cfg = plume_configuration(res, cell_size=h, inflow_center=(0.5, 0.15, 0.4), inflow_radius=0.2, vorticity=True)
    elif name == "colliders":
        cfg = plume_configuration(res, cell_size=h, vorticity=True, inflow_center=(0.3, 0.15, 0.3), inflow_radius=0.15)
        cfg.colliders = [
            Collider(Box(Vector3(0.55, 0.45, 0.4), Vector3(0.12, 0.08, 0.1)), Vector3(0.3, -0.2, 0.1), 0.5, 0.25),
            Collider(Ellipsoid(Vector3(0.3, 0.7, 0.35), Vector3(0.15, 0.1, 0.12)), Vector3(-0.1, 0.0, 0.4), 0.2, 0.7),
        ]
    elif name == "periodic":
        cfg = Configuration(resolution=[nx, ny, nz], cell_size=h, time_step=0.5 * h, vorticity_confinement_enabled=True)
        vb = cfg.velocity_boundary
        for f in (vb.x_min, vb.x_max, vb.z_min, vb.z_max):
            f.mode = VelocityBoundaryMode.periodic
        vb.y_min.mode = VelocityBoundaryMode.normal_fixed_tangent_zero_gradient
        vb.y_max.mode = VelocityBoundaryMode.zero_gradient
        for sb in (cfg.pressure_boundary, cfg.density_boundary, cfg.temperature_boundary):
            for f in (sb.x_min, sb.x_max, sb.z_min, sb.z_max):
                f.mode = ScalarBoundaryMode.periodic
        cfg.inflows = [Inflow(Vector3(0.5, 0.2, 0.5), 0.2, 1.0, 1.0)]
    elif name == "fixed_values":
        cfg = Configuration(resolution=[nx, ny, nz], cell_size=h, time_step=0.5 * h, vorticity_confinement_enabled=False)
        vb = cfg.velocity_boundary
        vb.x_min.mode = VelocityBoundaryMode.fixed_value
        vb.x_min.value = Vector3(0.2, 0.05, -0.1)
        vb.x_max.mode = VelocityBoundaryMode.normal_fixed_tangent_zero_gradient
        vb.x_max.value = Vector3(0.1, 0.0, 0.0)
        vb.y_min.mode = VelocityBoundaryMode.normal_fixed_tangent_zero_gradient
        vb.y_max.mode = VelocityBoundaryMode.zero_gradient
        vb.z_min.mode = VelocityBoundaryMode.fixed_value
        vb.z_max.mode = VelocityBoundaryMode.zero_gradient
        cfg.pressure_boundary.y_max.mode = ScalarBoundaryMode.fixed_value
        cfg.pressure_boundary.y_max.value = 0.05
        cfg.pressure_boundary.x_max.mode = ScalarBoundaryMode.fixed_value
        cfg.pressure_boundary.x_max.value = -0.02
        cfg.density_boundary.x_min.mode = ScalarBoundaryMode.fixed_value
        cfg.density_boundary.x_min.value = 0.3
        cfg.temperature_boundary.y_min.mode = ScalarBoundaryMode.fixed_value
        cfg.temperature_boundary.y_min.value = 0.6
    else:
        raise KeyError(name)
    return cfg


SCENARIOS = ("plume", "vorticity", "colliders", "periodic", "fixed_values")


def with_solver(cfg: Configuration, kind: str, iterations=None, tolerance=None) -> Configuration:
    cfg = copy.deepcopy(cfg)
    if kind == "rbgs":
        cfg.pressure_solver = PressureSolver.red_black_gauss_seidel
        if iterations is not None:
            cfg.pressure_iterations = iterations
    else:
        cfg.pressure_solver = PressureSolver.jacobi_pcg
        if iterations is not None:
            cfg.pressure_max_iterations = iterations
        if tolerance is not None:
            cfg.pressure_tolerance = tolerance
    return cfg


def sizes(res):
    nx, ny, nz = res
    n = nx * ny * nz
    return n, ((nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1))


def seeded_state(res, seed=0, amp=0.3, scalars=True):
    rng = np.random.default_rng(seed)
    n, f = sizes(res)
    return {"density": rng.uniform(0, 1, n) if scalars else np.zeros(n),
            "temperature": rng.uniform(0, 1, n) if scalars else np.zeros(n),
            "velocity": [rng.uniform(-amp, amp, f[a]) for a in range(3)]}


def seeded_control(res, seed=1, amp=0.5):
    rng = np.random.default_rng(seed)
    n, _ = sizes(res)
    return {"density_source": rng.uniform(0, amp, n), "temperature_source": rng.uniform(0, amp, n),
            "acceleration": [rng.uniform(-amp, amp, n) for _ in range(3)]}


def inflow_mask(cfg):
    """Cells whose centre lies in an inflow sphere (FP32, as the kernels test it)."""
    nx, ny, nz = (int(v) for v in cfg.resolution)
    h = np.float32(cfg.cell_size)
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32), np.arange(nx, dtype=np.float32), indexing="ij")
    px, py, pz = (x + np.float32(0.5)) * h, (y + np.float32(0.5)) * h, (z + np.float32(0.5)) * h
    hit = np.zeros((nz, ny, nx), bool)
    dens = np.zeros((nz, ny, nx), np.float32)
    temp = np.zeros((nz, ny, nx), np.float32)
    for f in cfg.inflows:
        dx, dy, dz = px - np.float32(f.center.x), py - np.float32(f.center.y), pz - np.float32(f.center.z)
        inside = dx * dx + dy * dy + dz * dz <= np.float32(f.radius) * np.float32(f.radius)
        hit |= inside
        dens[inside] = f.density
        temp[inside] = f.temperature
    return hit.ravel(), dens.ravel(), temp.ravel()


def reference_control(cfg, state, control):
    """Control arrays that make the reference's additive sources
    (operators.cu:286-290) reproduce the inflow spheres: inside a sphere the
    source is (value - state) / dt."""
    hit, dens, temp = inflow_mask(cfg)
    dt = np.float32(cfg.time_step)
    out = {"density_source": np.array(control["density_source"], np.float32),
           "temperature_source": np.array(control["temperature_source"], np.float32),
           "acceleration": [np.array(a, np.float32) for a in control["acceleration"]]}
    rho = np.asarray(state["density"], np.float32)
    tem = np.asarray(state["temperature"], np.float32)
    out["density_source"][hit] = (dens[hit] - rho[hit]) / dt
    out["temperature_source"][hit] = (temp[hit] - tem[hit]) / dt
    return out


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    d = np.linalg.norm(a - b)
    s = max(np.linalg.norm(b), 1e-300)
    return float(d / s)


def state_arrays(s):
    return [s["density"], s["temperature"], *s["velocity"]]


# ---------------------------------------------------------------- torch side
def to_model_state(model, ctx, arrays, dtype=None):
    import torch
    s = model.allocate_state(ctx) if dtype is None else model.allocate_state_adjoint(ctx)
    for t, a in zip(model._state_tensors(s), state_arrays(arrays)):
        t.copy_(torch.as_tensor(np.asarray(a), dtype=t.dtype))
    return s


def to_model_control(model, ctx, arrays, adjoint=False):
    import torch
    c = model.allocate_control_adjoint(ctx) if adjoint else model.allocate_control(ctx)
    ts = [c.density_source.values, c.temperature_source.values, c.external_acceleration.x.values, c.external_acceleration.y.values,
          c.external_acceleration.z.values]
    arrs = [arrays["density_source"], arrays["temperature_source"], *arrays["acceleration"]]
    for t, a in zip(ts, arrs):
        t.copy_(torch.as_tensor(np.asarray(a), dtype=t.dtype))
    return c


def from_model_state(model, s):
    ts = [t.detach().cpu().numpy() for t in model._state_tensors(s)]
    return {"density": ts[0], "temperature": ts[1], "velocity": ts[2:5]}


def cache_arrays(k):
    """Model StepCache -> oracle cache dict."""
    v = k.vorticity.detach().cpu().numpy()
    return {"sourced_density": k.sourced_density.values.cpu().numpy(), "sourced_temperature": k.sourced_temperature.values.cpu().numpy(),
            "force": [k.force.x.values.cpu().numpy(), k.force.y.values.cpu().numpy(), k.force.z.values.cpu().numpy()],
            "centered_velocity": [v[0], v[1], v[2]], "vorticity": [v[3], v[4], v[5]], "magnitude": v[6],
            "normal": [v[7], v[8], v[9]], "normalizer": v[10],
            "forced_velocity": [t.cpu().numpy() for t in k.forced_velocity.components()],
            "advected_velocity": [t.cpu().numpy() for t in k.advected_velocity.components()]}


# ---------------------------------------------------------------- differentiable plume
PLUME_PARAMS = dict(ambient_temperature=0.0, density_buoyancy=-0.1, temperature_buoyancy=0.5, vorticity_confinement=0.0)


def differentiable_plume(n=128):
    """The differentiable plume at n^3: the benchmark physics (inflow sphere
    r = 0.08 at (0.5, 0.1, 0.5) setting density = temperature = 1, buoyancy
    0.5 T - 0.1 rho, walls with a fixed normal velocity, open top), initial
    velocity = seeded uniform noise in +-0.01 (FP32-representable, so the FP32
    product and the FP64 oracle start from the same state), density and
    temperature 0, zero controls.  The target is a Gaussian blob (sigma 0.1,
    amplitude 1) at a seeded uniform centre in [0.3, 0.7]^3.
    Returns (configuration, [u0 per face component], target)."""
    cfg = plume_configuration((n, n, n), inflow_center=(0.5, 0.1, 0.5), inflow_radius=0.08)
    rng = np.random.default_rng(0)
    _, f = sizes((n, n, n))
    u0 = [rng.uniform(-0.01, 0.01, f[a]).astype(np.float32).astype(np.float64) for a in range(3)]
    centre = np.random.default_rng(1).uniform(0.3, 0.7, 3)
    c = (np.arange(n) + 0.5) / n
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    target = np.exp(-((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2) / (2 * 0.1 ** 2)).reshape(-1)
    return cfg, u0, target


def plume_directions(n, count):
    """The first `count` of the seeded unit directions of the finite-difference
    check: smooth random velocity fields (Gaussian bumps per face component)
    scaled to unit L2 norm over all faces, flattened per component."""
    from diff_solver_b200.gradcheck import smooth_direction
    rng = np.random.default_rng(2)
    shapes = [(n, n, n + 1), (n, n + 1, n), (n + 1, n, n)]  # (z, y, x) extents of the face components
    return [[x.reshape(-1) for x in smooth_direction(rng, shapes, n)] for _ in range(count)]


def density_distance(density, target):
    """The loss of the differentiable plume: ||rho_T - target||_2."""
    d = np.asarray(density, np.float64) - target
    return float(np.sqrt(d @ d))


# ---------------------------------------------------------------- parity report
def report(name, **values):
    """Appends one JSON line of measured errors to $XS_PARITY_REPORT (when set),
    so that a GPU run leaves the per-field numbers behind."""
    import json
    path = os.environ.get("XS_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"test": name, **values}) + "\n")


def field_errors(got, want):
    """Relative L2 errors of density, temperature and the velocity field (the
    three face components together) of two state dicts."""
    cat = lambda s: np.concatenate([np.asarray(v, np.float64).ravel() for v in s["velocity"]])
    return {"density": rel_l2(got["density"], want["density"]), "temperature": rel_l2(got["temperature"], want["temperature"]),
            "velocity": rel_l2(cat(got), cat(want))}


def reference_step(cfg, domain, state, control, params, tolerance=0.0, max_sweeps=400000):
    """One step of the reference's own kernels (oracle/_ref) from host state
    arrays: RBGS with the configured sweep count, or (tolerance > 0) iterated
    until the FP64 relative residual reaches `tolerance` or stops falling.
    Inflow spheres are emulated with sources.  Returns (next state dict,
    sweeps, residual)."""
    import torch
    from oracle import ref_binding as rb
    ref = rb.Reference(cfg, domain)
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float32, device=dev).contiguous()
    s_in = [t(a) for a in state_arrays(state)]
    rctl = reference_control(cfg, state, control)
    c_in = [t(rctl["density_source"]), t(rctl["temperature_source"])] + [t(a) for a in rctl["acceleration"]]
    p_in = [torch.tensor([params[k]], dtype=torch.float32, device=dev) for k in
            ("ambient_temperature", "density_buoyancy", "temperature_buoyancy", "vorticity_confinement")]
    out = [torch.zeros_like(x) for x in s_in]
    n = s_in[0].numel()
    cache = [torch.zeros(n, device=dev) for _ in range(5)] + [torch.zeros((11, n), device=dev)] + \
            [torch.zeros_like(x) for x in s_in[2:]] + [torch.zeros_like(x) for x in s_in[2:]]
    sweeps, residual = ref.forward_step(s_in, c_in, p_in, out, cache, tolerance=tolerance, max_sweeps=max_sweeps)
    torch.cuda.synchronize()
    o = [x.cpu().numpy() for x in out]
    return {"density": o[0], "temperature": o[1], "velocity": o[2:5]}, sweeps, residual


def product_domain(ctx):
    """The rasterised domain of a product context, as the reference harness takes it."""
    d = ctx.domain
    return {"mask": d.cell_mask, "cv": list(d.collider_velocity.components()), "cd": d.collider_density.values,
            "ct": d.collider_temperature.values, "anchor": d.pressure_anchor}
