"""ctypes binding of the CPU oracle (oracle/smoke_oracle.c).

TEST INFRASTRUCTURE ONLY.  Tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use this module as the checker; the product path
never imports it.

Two builds of the same C source are loaded side by side:
``precision="f32"`` follows the reference kernels' FP32 operation order
(solvers/smoke/operators.cu), ``precision="f64"`` is the FP64 oracle.

A problem description is any object with the attributes of
``diff_solver_b200.data.Configuration`` (resolution, cell_size, time_step,
the four boundaries, colliders, inflows, vorticity_confinement_enabled and the
pressure-solver settings); this module reads them duck-typed.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")


def build(force: bool = False) -> None:
    """Compile both oracle precisions with the committed Makefile."""
    targets = [os.path.join(_BUILD, f"libsmoke_oracle_{p}.so") for p in ("f32", "f64")]
    if force or not all(os.path.exists(t) for t in targets) or any(
        os.path.getmtime(t) < os.path.getmtime(os.path.join(_HERE, "smoke_oracle.c")) for t in targets
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)


class og_grid(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("cell_size", C.c_double), ("time_step", C.c_double)]


class og_sbnd(C.Structure):
    _fields_ = [("modes", C.c_uint32 * 6), ("values", C.c_double * 6)]


class og_vbnd(C.Structure):
    _fields_ = [("modes", C.c_uint32 * 6), ("values", C.c_double * 18)]


class og_inflow(C.Structure):
    _fields_ = [("center", C.c_double * 3), ("radius", C.c_double), ("density", C.c_double), ("temperature", C.c_double)]


class og_collider(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("center", C.c_double * 3), ("size", C.c_double * 3), ("velocity", C.c_double * 3),
                ("density", C.c_double), ("temperature", C.c_double)]


class og_config(C.Structure):
    _fields_ = [
        ("grid", og_grid), ("velocity_boundary", og_vbnd), ("pressure_boundary", og_sbnd), ("density_boundary", og_sbnd),
        ("temperature_boundary", og_sbnd), ("pressure_anchor", C.c_uint32), ("vorticity_enabled", C.c_uint32),
        ("solver", C.c_uint32), ("iterations", C.c_uint32), ("tolerance", C.c_double), ("inflow_count", C.c_uint32),
        ("inflows", C.c_void_p), ("cell_mask", C.c_void_p), ("collider_velocity", C.c_void_p * 3),
        ("collider_density", C.c_void_p), ("collider_temperature", C.c_void_p), ("pressure_guess", C.c_void_p),
    ]


class og_solve_stats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("initial_residual", C.c_double), ("final_residual", C.c_double), ("converged", C.c_uint32)]


def _ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _p3(arrs):
    """A C array of three pointers; ctypes passes arrays by address, which is
    what a ``real* const u[3]`` parameter expects."""
    return (C.c_void_p * 3)(*[None if a is None else a.ctypes.data for a in arrs])


def _make_struct(name, names):
    fields = []
    for n in names:
        if n.endswith("[3]"):
            fields.append((n[:-3], C.c_void_p * 3))
        else:
            fields.append((n, C.c_void_p))
    return type(name, (C.Structure,), {"_fields_": fields})


og_state = _make_struct("og_state", ["density", "temperature", "velocity[3]"])
og_control = _make_struct("og_control", ["density_source", "temperature_source", "acceleration[3]"])
og_cache = _make_struct("og_cache", ["sourced_density", "sourced_temperature", "force[3]", "centered_velocity[3]", "vorticity[3]",
                                     "magnitude", "normal[3]", "normalizer", "forced_velocity[3]", "advected_velocity[3]"])
og_scratch = _make_struct("og_scratch", ["raw_advected[3]", "pressure", "rhs"])


def _params_struct(ctype):
    return type("og_params", (C.Structure,), {"_fields_": [("ambient_temperature", ctype), ("density_buoyancy", ctype),
                                                           ("temperature_buoyancy", ctype), ("vorticity_confinement", ctype)]})


og_params_adj = _params_struct(C.c_double)

_LIBS = {}


def lib(precision: str):
    if precision not in _LIBS:
        build()
        L = C.CDLL(os.path.join(_BUILD, f"libsmoke_oracle_{precision}.so"), mode=C.RTLD_LOCAL)
        L.og_build_domain.restype = C.c_uint32
        L.og_relative_residual.restype = C.c_double
        L.og_sizeof_config.restype = C.c_size_t
        assert L.og_sizeof_config() == C.sizeof(og_config), "oracle struct layout mismatch"
        _LIBS[precision] = L
    return _LIBS[precision]


def dtype_of(precision):
    return np.float32 if precision == "f32" else np.float64


def set_threads(n: int) -> int:
    r = 1
    for p in ("f32", "f64"):
        r = lib(p).og_set_threads(int(n))
    return r


# --------------------------------------------------------------------------
# field containers
# --------------------------------------------------------------------------

def face_shape(res, axis):
    nx, ny, nz = res
    return (nx + (axis == 0), ny + (axis == 1), nz + (axis == 2))


def n_faces(res, axis):
    s = face_shape(res, axis)
    return s[0] * s[1] * s[2]


def n_cells(res):
    return res[0] * res[1] * res[2]


@dataclass
class Fields:
    """Flat host arrays in the reference layout (x fastest, SoA)."""
    arrays: dict = field(default_factory=dict)

    def __getitem__(self, k):
        return self.arrays[k]

    def __setitem__(self, k, v):
        self.arrays[k] = v


def zeros_state(res, dt):
    n = n_cells(res)
    return {"density": np.zeros(n, dt), "temperature": np.zeros(n, dt),
            "velocity": [np.zeros(n_faces(res, a), dt) for a in range(3)]}


def zeros_control(res, dt):
    n = n_cells(res)
    return {"density_source": np.zeros(n, dt), "temperature_source": np.zeros(n, dt),
            "acceleration": [np.zeros(n, dt) for _ in range(3)]}


def zeros_cache(res, dt):
    n = n_cells(res)
    z = lambda: np.zeros(n, dt)
    return {"sourced_density": z(), "sourced_temperature": z(), "force": [z(), z(), z()],
            "centered_velocity": [z(), z(), z()], "vorticity": [z(), z(), z()], "magnitude": z(),
            "normal": [z(), z(), z()], "normalizer": z(),
            "forced_velocity": [np.zeros(n_faces(res, a), dt) for a in range(3)],
            "advected_velocity": [np.zeros(n_faces(res, a), dt) for a in range(3)]}


def zeros_state_adj(res):
    return zeros_state(res, np.float64)


def zeros_control_adj(res):
    return zeros_control(res, np.float64)


def _state_struct(s):
    st = og_state()
    st.density = s["density"].ctypes.data
    st.temperature = s["temperature"].ctypes.data
    for a in range(3):
        st.velocity[a] = s["velocity"][a].ctypes.data
    return st


def _control_struct(c):
    st = og_control()
    st.density_source = c["density_source"].ctypes.data
    st.temperature_source = c["temperature_source"].ctypes.data
    for a in range(3):
        st.acceleration[a] = c["acceleration"][a].ctypes.data
    return st


def _cache_struct(k):
    st = og_cache()
    for name in ("sourced_density", "sourced_temperature", "magnitude", "normalizer"):
        setattr(st, name, k[name].ctypes.data)
    for name in ("force", "centered_velocity", "vorticity", "normal", "forced_velocity", "advected_velocity"):
        arr = getattr(st, name)
        for a in range(3):
            arr[a] = k[name][a].ctypes.data
    return st


# --------------------------------------------------------------------------
# problem description
# --------------------------------------------------------------------------

def _mode(m):
    return int(getattr(m, "value", m))


class Problem:
    """The oracle-side view of a Configuration plus its rasterised domain."""

    def __init__(self, cfg, precision="f64", solver=None, iterations=None, tolerance=None):
        self.cfg = cfg
        self.precision = precision
        self.dt = dtype_of(precision)
        self.res = tuple(int(v) for v in cfg.resolution)
        L = lib(precision)
        c = og_config()
        c.grid = og_grid(self.res[0], self.res[1], self.res[2], float(cfg.cell_size), float(cfg.time_step))
        vb = cfg.velocity_boundary
        for i, f in enumerate((vb.x_min, vb.x_max, vb.y_min, vb.y_max, vb.z_min, vb.z_max)):
            c.velocity_boundary.modes[i] = _mode(f.mode)
            c.velocity_boundary.values[3 * i + 0] = float(f.value.x)
            c.velocity_boundary.values[3 * i + 1] = float(f.value.y)
            c.velocity_boundary.values[3 * i + 2] = float(f.value.z)
        for name in ("pressure_boundary", "density_boundary", "temperature_boundary"):
            sb = getattr(cfg, name)
            dst = getattr(c, name)
            for i, f in enumerate((sb.x_min, sb.x_max, sb.y_min, sb.y_max, sb.z_min, sb.z_max)):
                dst.modes[i] = _mode(f.mode)
                dst.values[i] = float(f.value)
        c.vorticity_enabled = 1 if cfg.vorticity_confinement_enabled else 0
        kind = solver if solver is not None else ("pcg" if _mode(cfg.pressure_solver) == 0 else "rbgs")
        c.solver = 1 if kind == "pcg" else 0
        if kind == "pcg":
            c.iterations = int(iterations if iterations is not None else cfg.pressure_max_iterations)
            c.tolerance = float(tolerance if tolerance is not None else cfg.pressure_tolerance)
        else:
            c.iterations = int(iterations if iterations is not None else cfg.pressure_iterations)
            c.tolerance = 0.0
        # inflows
        self._inflows = (og_inflow * max(1, len(cfg.inflows)))()
        for i, f in enumerate(cfg.inflows):
            self._inflows[i].center[:] = [f.center.x, f.center.y, f.center.z]
            self._inflows[i].radius = f.radius
            self._inflows[i].density = f.density
            self._inflows[i].temperature = f.temperature
        c.inflow_count = len(cfg.inflows)
        c.inflows = C.cast(self._inflows, C.c_void_p)
        # domain
        n = n_cells(self.res)
        self.mask = np.zeros(n, np.uint32)
        self.collider_velocity = [np.zeros(n_faces(self.res, a), self.dt) for a in range(3)]
        self.collider_density = np.zeros(n, self.dt)
        self.collider_temperature = np.zeros(n, self.dt)
        cols = (og_collider * max(1, len(cfg.colliders)))()
        for i, k in enumerate(cfg.colliders):
            shp = k.shape
            if hasattr(shp, "radius"):
                cols[i].shape = 0
                cols[i].center[:] = [shp.center.x, shp.center.y, shp.center.z]
                cols[i].size[:] = [shp.radius.x, shp.radius.y, shp.radius.z]
            else:
                cols[i].shape = 1
                cols[i].center[:] = [shp.center.x, shp.center.y, shp.center.z]
                cols[i].size[:] = [shp.half_extent.x, shp.half_extent.y, shp.half_extent.z]
            cols[i].velocity[:] = [k.velocity.x, k.velocity.y, k.velocity.z]
            cols[i].density = k.density
            cols[i].temperature = k.temperature
        fv = _p3(self.collider_velocity)
        self.anchor = int(L.og_build_domain(C.byref(c.grid), C.byref(c.pressure_boundary), cols, len(cfg.colliders),
                                            _ptr(self.mask), fv, _ptr(self.collider_density), _ptr(self.collider_temperature)))
        c.pressure_anchor = self.anchor
        self.has_colliders = len(cfg.colliders) > 0
        c.cell_mask = self.mask.ctypes.data if self.has_colliders else None
        for a in range(3):
            c.collider_velocity[a] = self.collider_velocity[a].ctypes.data
        c.collider_density = self.collider_density.ctypes.data
        c.collider_temperature = self.collider_temperature.ctypes.data
        self.c = c
        self.L = L
        self.params_t = _params_struct(C.c_float if precision == "f32" else C.c_double)

    # ---- helpers -----------------------------------------------------------
    def params(self, p):
        return self.params_t(p["ambient_temperature"], p["density_buoyancy"], p["temperature_buoyancy"],
                             p["vorticity_confinement"])

    def cast_state(self, s):
        return {"density": np.ascontiguousarray(s["density"], self.dt),
                "temperature": np.ascontiguousarray(s["temperature"], self.dt),
                "velocity": [np.ascontiguousarray(v, self.dt) for v in s["velocity"]]}

    def cast_control(self, c):
        return {"density_source": np.ascontiguousarray(c["density_source"], self.dt),
                "temperature_source": np.ascontiguousarray(c["temperature_source"], self.dt),
                "acceleration": [np.ascontiguousarray(v, self.dt) for v in c["acceleration"]]}

    # ---- step composition ---------------------------------------------------
    def forward_step(self, state, control, params, guess=None):
        """model.cpp:341-349.  Returns (next_state, cache, stats, scratch);
        scratch["p"] is the pressure.  `guess` (optional, PCG kind only)
        starts the pressure solve from the given field instead of zero: the
        converged result is the same, a good start only saves iterations."""
        g = None if guess is None else np.ascontiguousarray(guess, self.dt)
        self.c.pressure_guess = None if g is None else g.ctypes.data
        try:
            return self._forward_step(state, control, params)
        finally:
            self.c.pressure_guess = None

    def _forward_step(self, state, control, params):
        s = self.cast_state(state)
        u = self.cast_control(control)
        nxt = zeros_state(self.res, self.dt)
        k = zeros_cache(self.res, self.dt)
        n = n_cells(self.res)
        w = {"raw": [np.zeros(n_faces(self.res, a), self.dt) for a in range(3)], "p": np.zeros(n, self.dt), "rhs": np.zeros(n, self.dt)}
        sc = og_scratch()
        for a in range(3):
            sc.raw_advected[a] = w["raw"][a].ctypes.data
        sc.pressure = w["p"].ctypes.data
        sc.rhs = w["rhs"].ctypes.data
        st = og_solve_stats()
        ss, us, ns, ks = _state_struct(s), _control_struct(u), _state_struct(nxt), _cache_struct(k)
        pr = self.params(params)
        self.L.og_forward_step(C.byref(self.c), C.byref(ss), C.byref(us), C.byref(pr), C.byref(ns), C.byref(ks), C.byref(sc), C.byref(st))
        return nxt, k, st, w

    def vjp_step(self, state, params, next_state, cache, next_adj, prev_adj=None, control_adj=None, param_adj=None):
        """model.cpp:361-389.  Accumulates into prev_adj / control_adj / param_adj."""
        res = self.res
        n = n_cells(res)
        F = sum(n_faces(res, a) for a in range(3))
        prev_adj = prev_adj if prev_adj is not None else zeros_state_adj(res)
        control_adj = control_adj if control_adj is not None else zeros_control_adj(res)
        param_adj = param_adj if param_adj is not None else og_params_adj(0, 0, 0, 0)
        scratch = np.zeros(2 * n + 3 * n + 4 * F + 2 * n + 10 * n, np.float64)
        s = self.cast_state(state)
        nx_ = self.cast_state(next_state)
        st = og_solve_stats()
        ss, ns, ks = _state_struct(s), _state_struct(nx_), _cache_struct(cache)
        na = _state_struct(next_adj)
        pa = _state_struct(prev_adj)
        ca = _control_struct(control_adj)
        pr = self.params(params)
        self.L.og_vjp_step(C.byref(self.c), C.byref(ss), C.byref(pr), C.byref(ns), C.byref(ks), C.byref(na), C.byref(pa),
                           C.byref(ca), C.byref(param_adj), _ptr(scratch), C.byref(st))
        return prev_adj, control_adj, param_adj, st

    def jvp_step(self, state, params, next_state, cache, state_tan, control_tan, param_tan):
        """model.cpp:351-359."""
        res = self.res
        n = n_cells(res)
        F = sum(n_faces(res, a) for a in range(3))
        scratch = np.zeros(2 * n + 3 * n + 3 * F + 2 * n + 10 * n, self.dt)
        s = self.cast_state(state)
        nx_ = self.cast_state(next_state)
        stt = self.cast_state(state_tan)
        ctt = self.cast_control(control_tan)
        out = zeros_state(res, self.dt)
        ss, ns, ks = _state_struct(s), _state_struct(nx_), _cache_struct(cache)
        ts, tc, to = _state_struct(stt), _control_struct(ctt), _state_struct(out)
        pr, pt = self.params(params), self.params(param_tan)
        self.L.og_jvp_step(C.byref(self.c), C.byref(ss), C.byref(pr), C.byref(ns), C.byref(ks), C.byref(ts), C.byref(tc),
                           C.byref(pt), C.byref(to), _ptr(scratch))
        return out

    # ---- pressure -----------------------------------------------------------
    def pressure_rhs(self, velocity):
        u = [np.ascontiguousarray(v, self.dt) for v in velocity]
        rhs = np.zeros(n_cells(self.res), self.dt)
        self.L.og_pressure_rhs(C.byref(self.c), _p3(u), _ptr(rhs))
        return rhs

    def pcg(self, rhs, max_iterations, tolerance, guess=None):
        rhs = np.ascontiguousarray(rhs, self.dt)
        p = np.zeros_like(rhs)
        st = og_solve_stats()
        g = None if guess is None else np.ascontiguousarray(guess, self.dt)
        self.L.og_pcg(C.byref(self.c), _ptr(rhs), _ptr(g), C.c_uint32(max_iterations), C.c_double(tolerance), _ptr(p), C.byref(st))
        return p, st

    def rbgs(self, rhs, iterations, p=None):
        rhs = np.ascontiguousarray(rhs, self.dt)
        p = np.zeros_like(rhs) if p is None else np.ascontiguousarray(p, self.dt).copy()
        self.L.og_rbgs(C.byref(self.c), _ptr(rhs), _ptr(p), C.c_uint32(iterations))
        return p

    def relative_residual(self, rhs, p):
        rhs = np.ascontiguousarray(rhs, self.dt)
        p = np.ascontiguousarray(p, self.dt)
        return float(self.L.og_relative_residual(C.byref(self.c), _ptr(rhs), _ptr(p)))

    def apply_operator(self, p):
        p = np.ascontiguousarray(p, np.float64)
        q = np.zeros_like(p)
        self.L.og_apply_operator(C.byref(self.c), _ptr(p), _ptr(q))
        return q

    # ---- single operators ---------------------------------------------------
    def advect_velocity(self, velocity):
        u = [np.ascontiguousarray(v, self.dt) for v in velocity]
        out = [np.zeros_like(v) for v in u]
        self.L.og_advect_velocity(C.byref(self.c), _p3(u), _p3(out))
        return out

    def project_velocity(self, velocity, p):
        u = [np.ascontiguousarray(v, self.dt) for v in velocity]
        out = [np.zeros_like(v) for v in u]
        self.L.og_project_velocity(C.byref(self.c), _p3(u), _ptr(np.ascontiguousarray(p, self.dt)), _p3(out))
        return out
