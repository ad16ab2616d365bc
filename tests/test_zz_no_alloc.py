"""The allocation-free pressure solve (xs_pressure_solve_static).

It serves callers that cannot allocate device memory: they hand over only
the right-hand side and the output, and the solve runs in a fixed,
library-owned scratch array.  Its results must equal those of the regular
entry point (xs_pressure_solve with a caller-allocated workspace), and the
array's leftovers from one call must not leak into the next.  This file is
collected last on purpose, and passes both alone and after the rest of the
suite."""
import ctypes as C

import numpy as np
import pytest

from common import rel_l2, scenario, seeded_state, with_solver

from oracle import binding as ob

pytestmark = pytest.mark.gpu

TOLERANCE = 1e-6  # the relative L2 used for FP32 pressure fields in the suite


def _problem(seed):
    cfg = with_solver(scenario("plume", res=(48, 40, 32)), "pcg", iterations=20000, tolerance=1e-8)
    P = ob.Problem(cfg, "f32")
    rhs = P.pressure_rhs(seeded_state(P.res, seed=seed)["velocity"])
    return cfg, P, rhs


def test_static_solve_matches_the_workspace_solve_on_consecutive_calls(cuda):
    import torch
    from diff_solver_b200 import _native as N
    from diff_solver_b200.model import scalar_boundary
    L = N.lib()
    results = []
    for seed in (61, 62):  # two calls in a row, different right-hand sides
        cfg, P, rhs = _problem(seed)
        g = N.XsGrid(*P.res, float(cfg.cell_size), float(cfg.time_step))
        solve = N.XsPressureSolve(N.XS_SOLVER_JACOBI_PCG, 20000, 1e-8, None)
        pb = scalar_boundary(cfg.pressure_boundary)
        rhs_t = torch.as_tensor(rhs, dtype=torch.float32, device="cuda")
        # regular entry point, caller-owned workspace
        workspace = torch.zeros(L.xs_projection_workspace_bytes(g), dtype=torch.uint8, device="cuda")
        expected = torch.zeros_like(rhs_t)
        N.check("xs_pressure_solve", L.xs_pressure_solve(None, g, solve, P.anchor, None, pb, rhs_t.data_ptr(), expected.data_ptr(),
                                                         workspace.data_ptr()))
        # allocation-free entry point
        got = torch.full_like(rhs_t, float("nan"))
        stats = N.XsSolveStats()
        N.check("xs_pressure_solve_static", L.xs_pressure_solve_static(None, g, solve, P.anchor, None, pb, rhs_t.data_ptr(),
                                                                       got.data_ptr(), C.byref(stats)))
        torch.cuda.synchronize()
        e, o = expected.cpu().numpy(), got.cpu().numpy()
        assert np.isfinite(o).all()
        assert rel_l2(o, e) < TOLERANCE, (seed, rel_l2(o, e))
        assert stats.status == N.XS_OK and stats.final_residual <= 1e-8
        results.append(o)
    assert rel_l2(results[0], results[1]) > 1e-3  # the two calls solved different problems


def test_static_solve_rejects_grids_beyond_its_capacity(cuda):
    from diff_solver_b200 import _native as N
    L = N.lib()
    g = N.XsGrid(65, 64, 64, 1.0 / 64, 0.5 / 64)
    solve = N.XsPressureSolve(N.XS_SOLVER_JACOBI_PCG, 100, 1e-6, None)
    status = L.xs_pressure_solve_static(None, g, solve, 0, None, N.XsScalarBoundary(), 1, 1, None)
    assert status == N.XS_CAPACITY_EXCEEDED
