"""B200-native (sm_100a) differentiable smoke solver with the API of
diff-solver's smoke model and solver driver.

The compute path is the native library ``libdiffsmoke.so`` (hand-written
CUDA for sm_100a behind the C ABI in ``include/diff_smoke.h``); this package
is the Python host layer mirroring the reference's modules:

* ``data``   -- xayah.smoke.data (configuration, boundaries, colliders)
* ``model``  -- xayah.smoke.model (Model, ExecutionContext, fields)
* ``solver`` -- xayah.solver (simulate / jvp / vjp, tape modes)
"""
from .data import (Box, Collider, Configuration, Ellipsoid, Inflow, PressureSolver, ScalarBoundary, ScalarBoundaryFace,
                   ScalarBoundaryMode, Vector3, VelocityBoundary, VelocityBoundaryFace, VelocityBoundaryMode, WarmStart,
                   plume_configuration)

__all__ = [
    "Box", "Collider", "Configuration", "Ellipsoid", "Inflow", "PressureSolver", "ScalarBoundary", "ScalarBoundaryFace",
    "ScalarBoundaryMode", "Vector3", "VelocityBoundary", "VelocityBoundaryFace", "VelocityBoundaryMode", "WarmStart",
    "plume_configuration",
]


def load():
    """Load the native library; raises if it has not been built."""
    from . import _native
    return _native.lib()
