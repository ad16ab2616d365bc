"""The exact separable solve of the warm start's coarse-grid correction
(xs_separable_solve, csrc/spectral.cu) against the FP64 oracle's Jacobi-PCG
solution of the same system, for every kind of axis: zero-gradient at both
ends, fixed value at both ends, mixed ends in either order, periodic."""
import ctypes as C

import numpy as np
import pytest

from common import rel_l2
from diff_solver_b200.data import Configuration, ScalarBoundaryMode

pytestmark = pytest.mark.gpu

Z, F, P = ScalarBoundaryMode.zero_gradient, ScalarBoundaryMode.fixed_value, ScalarBoundaryMode.periodic


def configuration(res, modes):
    cfg = Configuration(resolution=list(res), cell_size=1.0 / res[0], time_step=0.5 / res[0])
    pb = cfg.pressure_boundary
    for face, m in zip((pb.x_min, pb.x_max, pb.y_min, pb.y_max, pb.z_min, pb.z_max), modes):
        face.mode = m
        face.value = 0.0
    return cfg


CASES = [
    ((16, 24, 32), (Z, Z, Z, F, Z, Z)),   # the plume's pressure boundary: open top
    ((33, 17, 20), (F, Z, Z, F, F, F)),   # odd extents, mixed ends in both orders
    ((48, 32, 40), (P, P, Z, F, P, P)),   # periodic x and z
    ((64, 8, 12), (F, F, F, F, Z, F)),
    ((128, 128, 128), (Z, Z, Z, F, Z, Z)),  # the coarse grid of the 256^3 plume
    ((200, 24, 16), (Z, F, Z, Z, F, Z)),    # a mixed axis of 129-256 cells: the basis in two halves
    ((256, 72, 12), (P, P, F, F, Z, F)),    # a periodic axis of 256 cells
    ((256, 256, 128), (Z, Z, Z, F, Z, Z)),  # the coarse grid of the 512x512x256 plume
]


@pytest.mark.parametrize("res,modes", CASES, ids=["x".join(map(str, r)) for r, _ in CASES])
def test_separable_solve_matches_the_oracle(cuda, res, modes):
    import torch
    from diff_solver_b200 import _native as N
    from diff_solver_b200.model import ExecutionMode, Model
    from oracle import binding as ob
    cfg = configuration(res, modes)
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.forward)
    L = N.lib()
    n = int(np.prod(res))
    rng = np.random.default_rng(11)
    rhs = rng.normal(size=n)
    scratch = torch.zeros(L.xs_separable_solve_scratch_bytes(), dtype=torch.uint8, device="cuda")
    b = torch.as_tensor(rhs, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    N.check("separable", L.xs_separable_solve(None, ctx.native.grid, ctx.native.pressure_boundary, ctx.native.pressure_anchor,
                                              C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(scratch.data_ptr())))
    torch.cuda.synchronize()
    got = x.cpu().numpy().astype(np.float64)
    prob = ob.Problem(cfg, "f64")
    assert prob.anchor >= n  # a fixed face: no anchor cell
    if n <= 64 ** 3:
        want, st = prob.pcg(rhs, 20000, 1e-12)
        assert st.converged == 1
        assert rel_l2(got, want) < 1e-5, rel_l2(got, want)  # FP32 transforms
    # the residual of the FP32 solution in FP64
    r = rhs - prob.apply_operator(got)
    assert np.linalg.norm(r) < 1e-5 * np.linalg.norm(rhs) * max(res) ** 2 / 16, np.linalg.norm(r) / np.linalg.norm(rhs)


def test_separable_solve_rejects_other_grids(cuda):
    import torch
    from diff_solver_b200 import _native as N
    from diff_solver_b200.model import ExecutionMode, Model
    L = N.lib()
    scratch = torch.zeros(L.xs_separable_solve_scratch_bytes(), dtype=torch.uint8, device="cuda")
    b = torch.zeros(1, dtype=torch.float64, device="cuda")
    x = torch.zeros(1, dtype=torch.float32, device="cuda")
    # an anchored (all zero-gradient) box and an axis longer than the basis
    for res, modes in (((16, 16, 16), (Z,) * 6), ((264, 16, 16), (Z, Z, Z, F, Z, Z))):
        ctx = Model(configuration(res, modes)).allocate_context(ExecutionMode.forward)
        status = L.xs_separable_solve(None, ctx.native.grid, ctx.native.pressure_boundary, ctx.native.pressure_anchor,
                                      C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), C.c_void_p(scratch.data_ptr()))
        assert status == N.XS_INVALID_ARGUMENT
