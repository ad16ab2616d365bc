"""ctypes declarations of the C ABI in ``include/diff_smoke.h``.

The native library ``libdiffsmoke.so`` is the product: there is no CPU or
PyTorch fallback.  Importing this module without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libdiffsmoke.so")

XS_OK, XS_CUDA_ERROR, XS_NOT_CONVERGED, XS_NUMERICAL_ERROR, XS_INVALID_ARGUMENT, XS_TIMEOUT, XS_CAPACITY_EXCEEDED = range(7)
XS_STATIC_SOLVE_MAX_CELLS = 64 * 64 * 64
XS_SOLVER_JACOBI_PCG, XS_SOLVER_RED_BLACK_GAUSS_SEIDEL = 0, 1
XS_MODE_FORWARD, XS_MODE_DIFFERENTIABLE = 0, 1
XS_MAX_INFLOWS = 8


class XsGrid(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("cell_size", C.c_float), ("time_step", C.c_float)]


class XsScalarBoundary(C.Structure):
    _fields_ = [("modes", C.c_uint32 * 6), ("values", C.c_float * 6)]


class XsVelocityBoundary(C.Structure):
    _fields_ = [("modes", C.c_uint32 * 6), ("values", C.c_float * 18)]


class XsVector(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p)]


XsAdjointVector = XsVector  # same layout: three pointers


class XsVec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class XsInflow(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_float), ("density", C.c_float), ("temperature", C.c_float)]


class XsPressureSolve(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("max_iterations", C.c_uint32), ("tolerance", C.c_double), ("initial_guess", C.c_void_p),
                ("scale_guess", C.c_uint32)]


class XsSolveStats(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("status", C.c_uint32), ("refinements", C.c_uint32), ("warm_start_used", C.c_uint32),
                ("rhs_norm", C.c_double), ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("guess_scale", C.c_double), ("coarse_iterations", C.c_uint32), ("smoothed_iterations", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class XsCollider(C.Structure):
    _fields_ = [("shape", C.c_uint32), ("center", C.c_float * 3), ("size", C.c_float * 3), ("velocity", C.c_float * 3),
                ("density", C.c_float), ("temperature", C.c_float)]


class XsSmokeModel(C.Structure):
    _fields_ = [("grid", XsGrid), ("velocity_boundary", XsVelocityBoundary), ("pressure_boundary", XsScalarBoundary),
                ("density_boundary", XsScalarBoundary), ("temperature_boundary", XsScalarBoundary),
                ("vorticity_confinement_enabled", C.c_uint32), ("pressure_anchor", C.c_uint32), ("pressure", XsPressureSolve),
                ("inflows", C.c_void_p), ("inflow_count", C.c_uint32), ("cell_mask", C.c_void_p), ("collider_velocity", XsVector),
                ("collider_density", C.c_void_p), ("collider_temperature", C.c_void_p), ("solve_begin", C.c_void_p),
                ("solve_end", C.c_void_p), ("warm_start", C.c_void_p), ("warm_start_history", C.c_uint32),
                ("warm_start_coarsening", C.c_uint32), ("warm_start_rounds", C.c_uint32), ("stage_events", C.c_void_p)]


XS_STEP_STAGES = 9


class XsState(C.Structure):
    _fields_ = [("density", C.c_void_p), ("temperature", C.c_void_p), ("velocity", XsVector)]


class XsControl(C.Structure):
    _fields_ = [("density_source", C.c_void_p), ("temperature_source", C.c_void_p), ("external_acceleration", XsVector)]


class XsParameters(C.Structure):
    _fields_ = [("ambient_temperature", C.c_void_p), ("density_buoyancy", C.c_void_p), ("temperature_buoyancy", C.c_void_p),
                ("vorticity_confinement", C.c_void_p)]


class XsStepCache(C.Structure):
    _fields_ = [("sourced_density", C.c_void_p), ("sourced_temperature", C.c_void_p), ("force", XsVector), ("vorticity", C.c_void_p),
                ("forced_velocity", XsVector), ("advected_velocity", XsVector)]


XsStateAdjoint = XsState
XsControlAdjoint = XsControl
XsParameterAdjoint = XsParameters

_V = C.c_void_p
_G = XsGrid
_S = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "xs_accumulate": (_S, [_V, _V, _V, C.c_uint64]),
    "xs_source_forward": (_S, [_V, _G, _V, _V, _V, _V, C.c_uint32, C.c_uint32, _V]),
    "xs_source_jvp": (_S, [_V, _G, _V, _V, _V, _V, C.c_uint32, _V]),
    "xs_source_vjp": (_S, [_V, _G, _V, _V, _V, C.c_uint32, _V, _V]),
    "xs_buoyancy_forward": (_S, [_V, _G, _V, _V, _V, XsVector, _V, _V, _V, XsVector]),
    "xs_buoyancy_jvp": (_S, [_V, _G, _V, _V, _V, _V, _V, XsVector, _V, _V, _V, _V, _V, _V, XsVector]),
    "xs_buoyancy_vjp": (_S, [_V, _G, _V, _V, _V, _V, _V, _V, XsVector, _V, _V, XsVector, _V, _V, _V]),
    "xs_integrate_velocity_forward": (_S, [_V, _G, _V, XsVector, XsVector, XsVector]),
    "xs_integrate_velocity_jvp": (_S, [_V, _G, _V, XsVector, XsVector, XsVector]),
    "xs_integrate_velocity_vjp": (_S, [_V, _G, _V, XsVector, XsVector, XsVector]),
    "xs_advect_velocity_forward": (_S, [_V, _G, _V, XsVector, XsVelocityBoundary, XsVector]),
    "xs_advect_velocity_jvp": (_S, [_V, _G, _V, XsVector, XsVector, XsVelocityBoundary, XsVector]),
    "xs_advect_velocity_vjp": (_S, [_V, _G, _V, XsVector, XsVelocityBoundary, XsVector, XsVector]),
    "xs_constrain_velocity_forward": (_S, [_V, _G, _V, XsVector, XsVector, XsVelocityBoundary, XsVector]),
    "xs_constrain_velocity_jvp": (_S, [_V, _G, _V, XsVector, XsVelocityBoundary, XsVector]),
    "xs_constrain_velocity_vjp": (_S, [_V, _G, _V, XsVector, XsVelocityBoundary, XsVector]),
    "xs_advect_scalar_forward": (_S, [_V, _G, _V, _V, _V, XsVector, XsScalarBoundary, XsVelocityBoundary, _V]),
    "xs_advect_scalar_jvp": (_S, [_V, _G, _V, _V, _V, XsVector, XsVector, XsScalarBoundary, XsVelocityBoundary, _V]),
    "xs_advect_scalar_vjp": (_S, [_V, _G, _V, _V, XsVector, XsScalarBoundary, XsVelocityBoundary, _V, _V, XsVector]),
    "xs_vorticity_forward": (_S, [_V, _G, _V, XsVector, _V, _V, XsVector]),
    "xs_vorticity_jvp": (_S, [_V, _G, _V, XsVector, _V, _V, _V, XsVector, _V]),
    "xs_vorticity_vjp": (_S, [_V, _G, _V, _V, _V, XsVector, XsVector, _V, _V]),
    "xs_projection_workspace_bytes": (C.c_size_t, [_G]),
    "xs_projection_forward": (_S, [_V, _G, C.POINTER(XsPressureSolve), C.c_uint32, _V, XsVector, XsVelocityBoundary, XsScalarBoundary,
                                   _V, _V, XsVector, _V]),
    "xs_projection_jvp": (_S, [_V, _G, C.POINTER(XsPressureSolve), C.c_uint32, _V, XsVector, XsVelocityBoundary, XsScalarBoundary,
                               _V, _V, XsVector, _V]),
    "xs_projection_vjp": (_S, [_V, _G, C.POINTER(XsPressureSolve), C.c_uint32, _V, XsVector, XsVelocityBoundary, XsScalarBoundary,
                               _V, _V, XsVector, _V]),
    "xs_pressure_solve": (_S, [_V, _G, C.POINTER(XsPressureSolve), C.c_uint32, _V, XsScalarBoundary, _V, _V, _V]),
    "xs_read_solve_stats": (_S, [_V, _V, C.POINTER(XsSolveStats)]),
    "xs_solve_stats_offset": (C.c_size_t, []),
    "xs_separable_solve_scratch_bytes": (C.c_size_t, []),
    "xs_separable_solve": (_S, [_V, _G, XsScalarBoundary, C.c_uint32, _V, _V, _V]),
    "xs_pressure_solve_static": (_S, [_V, _G, C.POINTER(XsPressureSolve), C.c_uint32, _V, XsScalarBoundary, _V, _V,
                                      C.POINTER(XsSolveStats)]),
    "xs_smoke_build_domain": (_S, [_V, _G, XsScalarBoundary, _V, C.c_uint32, _V, XsVector, _V, _V, C.POINTER(C.c_uint32)]),
    "xs_smoke_workspace_bytes": (C.c_size_t, [C.POINTER(XsSmokeModel), C.c_uint32]),
    "xs_smoke_forward_step": (_S, [_V, C.POINTER(XsSmokeModel), XsState, XsControl, XsParameters, XsState, XsStepCache, _V]),
    "xs_smoke_jvp_step": (_S, [_V, C.POINTER(XsSmokeModel), XsState, XsParameters, XsState, XsStepCache, XsState, XsControl,
                               XsParameters, XsState, _V]),
    "xs_smoke_vjp_step": (_S, [_V, C.POINTER(XsSmokeModel), XsState, XsParameters, XsState, XsStepCache, XsState, XsState,
                               XsControl, XsParameters, _V]),
    "xs_smoke_write_control": (_S, [_V, _G, C.c_uint64, C.c_float, XsVec3, XsVec3, C.c_float, C.c_float, C.c_float, XsVec3, XsVec3, _V, _V,
                                     XsVector]),
    "xs_smoke_reduce_metrics": (_S, [_V, C.POINTER(XsSmokeModel), _V, _V, XsVector, XsVector, _V]),
    "xs_smoke_read_solve_stats": (_S, [_V, C.POINTER(XsSmokeModel), _V, C.c_uint32, C.POINTER(XsSolveStats),
                                       C.POINTER(XsSolveStats)]),
    "xs_smoke_reset_warm_start": (_S, [_V, C.POINTER(XsSmokeModel), _V, C.c_uint32]),
    "xs_smoke_warm_start_fields": (_S, [_V, C.POINTER(XsSmokeModel), _V, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "xs_smoke_pressure_fields":(_S, [C.POINTER(XsSmokeModel), _V, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "xs_conv3d_bf16": (_S, [_V, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _V, _V, _V, _V, C.c_uint32,
                            _V]),
    "xs_conv3d_weight_grad_bf16": (_S, [_V, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _V, _V, _V, _V,
                                        C.c_uint32, _V]),
    "xs_conv3d_weight_grad_scratch_floats": (C.c_size_t, [C.c_uint32] * 6),
    "xs_warm_start_create": (_S, [C.POINTER(C.c_void_p), C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]),
    "xs_warm_start_destroy": (_S, [_V]),
    "xs_warm_start_parameter_count": (C.c_size_t, []),
    "xs_warm_start_initialize": (_S, [_V, _V, C.c_uint64]),
    "xs_warm_start_set_parameters": (_S, [_V, _V, _V]),
    "xs_warm_start_get_parameters": (_S, [_V, _V, _V]),
    "xs_warm_start_predict": (_S, [_V, _V, C.c_uint32, _V, _V]),
    "xs_warm_start_gradient": (_S, [_V, _V, C.c_uint32, _V, _V, _V, _V]),
    "xs_warm_start_set_loss": (_S, [_V, C.c_uint32, XsScalarBoundary]),
    "xs_warm_start_adam_step":(_S, [_V, _V, C.c_float, C.c_float, C.c_float, C.c_float]),
    "xs_warm_start_train_step": (_S, [_V, _V, C.c_uint32, _V, _V, C.c_float, _V]),
    "xs_warm_start_guess": (_S, [_V, _V, _G, _V, _V]),
    "xs_warm_start_status": (_S, [_V, _V]),
    "xs_launch_count": (C.c_uint64, []),
    "xs_last_cuda_error": (C.c_int, []),
    "xs_status_string": (C.c_char_p, [C.c_int]),
}

_lib = None


def library_available() -> bool:
    return os.path.exists(LIBRARY_PATH)


def lib():
    """Load the native library (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError(f"{LIBRARY_PATH} is missing: build it with `python -m diff_solver_b200.build` "
                               "(the smoke solver has no fallback implementation)")
        L = C.CDLL(LIBRARY_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class SmokeError(RuntimeError):
    def __init__(self, where: str, status: int):
        L = lib()
        msg = L.xs_status_string(status).decode()
        if status == XS_CUDA_ERROR:
            msg += f" (cudaError {L.xs_last_cuda_error()})"
        super().__init__(f"{where}: {msg}")
        self.status = status


def check(where: str, status: int) -> None:
    if status != XS_OK:
        raise SmokeError(where, status)


def vec(tensors) -> XsVector:
    if tensors is None:
        return XsVector(None, None, None)
    return XsVector(*[None if t is None else t.data_ptr() for t in tensors])


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())
