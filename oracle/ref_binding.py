"""ctypes binding of the reference-kernel harness (oracle/_ref/libref_smoke.so).

TEST INFRASTRUCTURE ONLY: the reference's own operators.cu compiled for
sm_100a (oracle/build_ref.sh), driven in the reference's step order.  Used by
the GPU parity tests to pin the CPU oracle and to compare the product with
the reference kernels, and by tests/golden/make_golden.py.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(_HERE, "_ref", "libref_smoke.so")


class RefGrid(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("cell_size", C.c_float), ("time_step", C.c_float)]


class RefScalarBoundary(C.Structure):
    _fields_ = [("modes", C.c_uint32 * 6), ("values", C.c_float * 6)]


class RefVelocityBoundary(C.Structure):
    _fields_ = [("modes", C.c_uint32 * 6), ("values", C.c_float * 18)]


class RefModel(C.Structure):
    _fields_ = [("grid", RefGrid), ("velocity_boundary", RefVelocityBoundary), ("pressure_boundary", RefScalarBoundary),
                ("density_boundary", RefScalarBoundary), ("temperature_boundary", RefScalarBoundary), ("vorticity_enabled", C.c_uint32),
                ("pressure_anchor", C.c_uint32), ("iterations", C.c_uint32), ("cell_mask", C.c_void_p),
                ("collider_velocity", C.c_void_p * 3), ("collider_density", C.c_void_p), ("collider_temperature", C.c_void_p)]


def _p(n):
    return type(f"P{n}", (C.Structure,), {"_fields_": [(f"p{i}", C.c_void_p) for i in range(n)]})


class RefLaunchArgs(C.Structure):
    _fields_ = [("u", C.c_void_p * 3), ("out", C.c_void_p * 3), ("src", C.c_void_p), ("sout", C.c_void_p), ("rhs", C.c_void_p),
                ("pressure", C.c_void_p), ("oa", C.c_void_p * 3), ("ua", C.c_void_p * 3), ("soa", C.c_void_p), ("sa", C.c_void_p)]


# ref_launch kernels
ADVECT_VELOCITY, CONSTRAIN_VELOCITY, ADVECT_SCALAR, PRESSURE_RHS, RBGS_SWEEPS, PROJECT_VELOCITY, ADVECT_VELOCITY_VJP, ADVECT_SCALAR_VJP = range(8)

RefState = _p(5)
RefControl = _p(5)
RefParams = _p(4)
RefCache = _p(12)

_lib = None


def available() -> bool:
    return os.path.exists(LIBRARY)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIBRARY} is missing (build it with oracle/build_ref.sh where the reference is checked out)")
        L = C.CDLL(LIBRARY)
        L.ref_scratch_bytes.restype = C.c_size_t
        L.ref_scratch_bytes.argtypes = [C.POINTER(RefModel)]
        L.ref_relative_residual.restype = C.c_double
        L.ref_forward_step.argtypes = [C.c_void_p, C.POINTER(RefModel), RefState, RefControl, RefParams, RefState, RefCache, C.c_void_p,
                                       C.c_double, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_double)]
        L.ref_jvp_step.argtypes = [C.c_void_p, C.POINTER(RefModel), RefState, RefParams, RefState, RefCache, RefState, RefControl,
                                   RefParams, RefState, C.c_void_p]
        L.ref_vjp_step.argtypes = [C.c_void_p, C.POINTER(RefModel), RefState, RefParams, RefState, RefCache, RefState, RefState,
                                   RefControl, RefParams, C.c_void_p]
        L.ref_advect_velocity.argtypes = [C.c_void_p, C.POINTER(RefModel), C.c_void_p * 3, C.c_void_p * 3]
        L.ref_advect_scalar.argtypes = [C.c_void_p, C.POINTER(RefModel), C.POINTER(RefScalarBoundary), C.c_void_p, C.c_void_p,
                                        C.c_void_p * 3, C.c_void_p]
        L.ref_rbgs.argtypes = [C.c_void_p, C.POINTER(RefModel), C.c_void_p, C.c_void_p, C.c_uint32]
        L.ref_launch.argtypes = [C.c_void_p, C.POINTER(RefModel), C.c_uint32, C.POINTER(RefLaunchArgs)]
        F3 = C.c_float * 3
        L.ref_write_control.argtypes = [C.c_void_p, C.POINTER(RefModel), C.c_uint64, C.c_float, F3, F3, C.c_float, C.c_float, C.c_float, F3, F3,
                                        C.c_void_p, C.c_void_p, C.c_void_p * 3]
        L.ref_reduce_metrics.argtypes = [C.c_void_p, C.POINTER(RefModel), C.c_void_p, C.c_void_p, C.c_void_p * 3, C.c_void_p * 3,
                                         C.c_void_p]
        _lib = L
    return _lib


def _sb(b):
    out = RefScalarBoundary()
    for i, f in enumerate(b.faces()):
        out.modes[i] = int(f.mode)
        out.values[i] = float(f.value)
    return out


def _vb(b):
    out = RefVelocityBoundary()
    for i, f in enumerate(b.faces()):
        out.modes[i] = int(f.mode)
        out.values[3 * i:3 * i + 3] = [float(f.value.x), float(f.value.y), float(f.value.z)]
    return out


class Reference:
    """The reference step on the GPU for a Configuration and a built
    domain (mask / collider tensors and anchor from a product context or
    from the oracle)."""

    def __init__(self, cfg, domain, iterations=None, device="cuda"):
        import torch
        self.torch = torch
        self.cfg = cfg
        self.device = device
        nx, ny, nz = (int(v) for v in cfg.resolution)
        m = RefModel()
        m.grid = RefGrid(nx, ny, nz, float(cfg.cell_size), float(cfg.time_step))
        m.velocity_boundary = _vb(cfg.velocity_boundary)
        m.pressure_boundary = _sb(cfg.pressure_boundary)
        m.density_boundary = _sb(cfg.density_boundary)
        m.temperature_boundary = _sb(cfg.temperature_boundary)
        m.vorticity_enabled = 1 if cfg.vorticity_confinement_enabled else 0
        m.pressure_anchor = int(domain["anchor"])
        m.iterations = int(iterations if iterations is not None else cfg.pressure_iterations)
        self._keep = [domain[k] for k in ("mask", "cd", "ct")] + list(domain["cv"])
        m.cell_mask = domain["mask"].data_ptr()
        for a in range(3):
            m.collider_velocity[a] = domain["cv"][a].data_ptr()
        m.collider_density = domain["cd"].data_ptr()
        m.collider_temperature = domain["ct"].data_ptr()
        self.m = m
        self.L = lib()
        self.scratch = torch.zeros(int(self.L.ref_scratch_bytes(C.byref(m))), dtype=torch.uint8, device=device)

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _ptrs(ts, cls):
        return cls(*[t.data_ptr() for t in ts])

    def forward_step(self, state, control, params, next_state, cache, tolerance=0.0, max_sweeps=200000):
        """state/next_state: [rho, T, ux, uy, uz]; control: [rs, ts, ax, ay, az];
        params: [amb, br, bt, conf]; cache: 12 tensors in StepCache order
        (vorticity as one (11, N) tensor)."""
        sweeps = C.c_uint32(0)
        res = C.c_double(0.0)
        r = self.L.ref_forward_step(self._stream(), C.byref(self.m), self._ptrs(state, RefState), self._ptrs(control, RefControl),
                                    self._ptrs(params, RefParams), self._ptrs(next_state, RefState), self._ptrs(cache, RefCache),
                                    C.c_void_p(self.scratch.data_ptr()), C.c_double(tolerance), C.c_uint32(max_sweeps),
                                    C.byref(sweeps), C.byref(res))
        if r != 0:
            raise RuntimeError(f"reference forward step failed ({r})")
        return int(sweeps.value), float(res.value)

    def jvp_step(self, state, params, next_state, cache, st, ct, pt, nt):
        r = self.L.ref_jvp_step(self._stream(), C.byref(self.m), self._ptrs(state, RefState), self._ptrs(params, RefParams),
                                self._ptrs(next_state, RefState), self._ptrs(cache, RefCache), self._ptrs(st, RefState),
                                self._ptrs(ct, RefControl), self._ptrs(pt, RefParams), self._ptrs(nt, RefState),
                                C.c_void_p(self.scratch.data_ptr()))
        if r != 0:
            raise RuntimeError(f"reference jvp step failed ({r})")

    def vjp_step(self, state, params, next_state, cache, na, pa, ca, qa):
        r = self.L.ref_vjp_step(self._stream(), C.byref(self.m), self._ptrs(state, RefState), self._ptrs(params, RefParams),
                                self._ptrs(next_state, RefState), self._ptrs(cache, RefCache), self._ptrs(na, RefState),
                                self._ptrs(pa, RefState), self._ptrs(ca, RefControl), self._ptrs(qa, RefParams),
                                C.c_void_p(self.scratch.data_ptr()))
        if r != 0:
            raise RuntimeError(f"reference vjp step failed ({r})")

    def advect_velocity(self, u, out):
        arr_in = (C.c_void_p * 3)(*[t.data_ptr() for t in u])
        arr_out = (C.c_void_p * 3)(*[t.data_ptr() for t in out])
        if self.L.ref_advect_velocity(self._stream(), C.byref(self.m), arr_in, arr_out) != 0:
            raise RuntimeError("reference advect_velocity failed")

    def rbgs(self, rhs, pressure, sweeps):
        if self.L.ref_rbgs(self._stream(), C.byref(self.m), C.c_void_p(rhs.data_ptr()), C.c_void_p(pressure.data_ptr()), sweeps) != 0:
            raise RuntimeError("reference rbgs failed")

    def launch(self, which, u=None, out=None, src=None, sout=None, rhs=None, pressure=None, oa=None, ua=None, soa=None, sa=None):
        """Enqueues one reference launcher (ref_launch) on the current stream,
        without synchronising: for per-kernel timing with CUDA events."""
        a = RefLaunchArgs()
        ptr = lambda t: None if t is None else t.data_ptr()
        for name, ts in (("u", u), ("out", out), ("oa", oa), ("ua", ua)):
            if ts is not None:
                getattr(a, name)[:] = [ptr(t) for t in ts]
        a.src, a.sout, a.rhs, a.pressure, a.soa, a.sa = ptr(src), ptr(sout), ptr(rhs), ptr(pressure), ptr(soa), ptr(sa)
        r = self.L.ref_launch(self._stream(), C.byref(self.m), int(which), C.byref(a))
        if r != 0:
            raise RuntimeError(f"reference launch {which} failed ({r})")

    def write_control(self, step, o, density_source, temperature_source, acceleration):
        """The example driver's launch_write_control (simulation.cu:88-92) for
        options `o` (any object with the ForwardSimulationOptions fields)."""
        F3 = C.c_float * 3
        v = lambda t: F3(*[float(c) for c in t])
        r = self.L.ref_write_control(self._stream(), C.byref(self.m), int(step), float(o.pulse_period), v(o.left_source_center),
                                     v(o.right_source_center), float(o.source_radius), float(o.density_source_rate),
                                     float(o.temperature_source_rate), v(o.left_acceleration), v(o.right_acceleration),
                                     C.c_void_p(density_source.data_ptr()), C.c_void_p(temperature_source.data_ptr()),
                                     (C.c_void_p * 3)(*[t.data_ptr() for t in acceleration]))
        if r != 0:
            raise RuntimeError(f"reference write_control failed ({r})")

    def reduce_metrics(self, density, temperature, pre, post, metrics):
        """The example driver's launch_reduce_metrics (simulation.cu:95-100)
        into a zeroed metrics[6] (FP64, device)."""
        r = self.L.ref_reduce_metrics(self._stream(), C.byref(self.m), C.c_void_p(density.data_ptr()), C.c_void_p(temperature.data_ptr()),
                                      (C.c_void_p * 3)(*[t.data_ptr() for t in pre]), (C.c_void_p * 3)(*[t.data_ptr() for t in post]),
                                      C.c_void_p(metrics.data_ptr()))
        if r != 0:
            raise RuntimeError(f"reference reduce_metrics failed ({r})")
