"""GPU parity of the forward step: CUDA product vs the CPU oracle and vs the
reference's own kernels (oracle/_ref), through the C ABI."""
import numpy as np
import pytest

from common import (PARAMS, SCENARIOS, cache_arrays, from_model_state, reference_control, rel_l2, scenario, seeded_control,
                    seeded_state, state_arrays, to_model_control, to_model_state, with_solver)

from oracle import binding as ob

pytestmark = pytest.mark.gpu

STATE_FIELDS = ("density", "temperature", "u", "v", "w")


def run_product(cfg, st_arr, ctl_arr, mode=0):
    import torch
    from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode(mode))
    st = to_model_state(model, ctx, st_arr)
    ctl = to_model_control(model, ctx, ctl_arr)
    par = fill_parameters(model.allocate_parameters(ctx), **PARAMS)
    nxt = model.allocate_state(ctx)
    k = model.allocate_step_cache(ctx)
    model.forward_step(st, ctl, par, nxt, k, ctx)
    torch.cuda.synchronize()
    return model, ctx, from_model_state(model, nxt), cache_arrays(k), ctx.read_solve_stats()


def domain_of(ctx):
    d = ctx.domain
    return {"mask": d.cell_mask, "cv": list(d.collider_velocity.components()), "cd": d.collider_density.values,
            "ct": d.collider_temperature.values, "anchor": d.pressure_anchor}


@pytest.mark.parametrize("name", SCENARIOS)
def test_forward_step_matches_fp64_oracle(cuda, name):
    cfg = with_solver(scenario(name), "pcg", iterations=20000, tolerance=1e-10)
    st, ctl = seeded_state(tuple(cfg.resolution), seed=21), seeded_control(tuple(cfg.resolution), seed=22)
    _, _, nxt, k, stats = run_product(cfg, st, ctl)
    assert stats["status"] == 0 and stats["final_residual"] <= 1e-10
    P = ob.Problem(cfg, "f64", solver="pcg", iterations=20000, tolerance=1e-13)
    onxt, ok, ost, _ = P.forward_step(st, ctl, PARAMS)
    for f, a, b in zip(STATE_FIELDS, state_arrays(nxt), state_arrays(onxt)):
        assert rel_l2(a, b) < 1e-5, (name, f, rel_l2(a, b))
    for key in ("sourced_density", "sourced_temperature"):
        assert rel_l2(k[key], ok[key]) < 1e-6
    for a in range(3):
        assert rel_l2(k["force"][a], ok["force"][a]) < 1e-5
        assert rel_l2(k["forced_velocity"][a], ok["forced_velocity"][a]) < 1e-6
        assert rel_l2(k["advected_velocity"][a], ok["advected_velocity"][a]) < 1e-5


@pytest.mark.parametrize("name", SCENARIOS)
def test_fixed_sweeps_match_the_reference_kernels(cuda, name):
    """RBGS kind, same sweep count: the product against the reference's own
    operators.cu on identical seeded inputs (1e-5 relative L2 per field)."""
    import torch
    from oracle import ref_binding as rb
    if not rb.available():
        pytest.skip("reference harness not built")
    cfg = with_solver(scenario(name), "rbgs", iterations=40)
    res = tuple(cfg.resolution)
    st, ctl = seeded_state(res, seed=23), seeded_control(res, seed=24)
    model, ctx, nxt, k, _ = run_product(cfg, st, ctl)
    ref = rb.Reference(cfg, domain_of(ctx))
    dev = torch.device("cuda")
    t = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float32, device=dev).contiguous()
    s_in = [t(a) for a in state_arrays(st)]
    rctl = reference_control(cfg, st, ctl)  # the reference has no inflow primitive: emulate it with sources
    c_in = [t(rctl["density_source"]), t(rctl["temperature_source"])] + [t(a) for a in rctl["acceleration"]]
    p_in = [torch.tensor([PARAMS[k_]], dtype=torch.float32, device=dev) for k_ in
            ("ambient_temperature", "density_buoyancy", "temperature_buoyancy", "vorticity_confinement")]
    out = [torch.zeros_like(x) for x in s_in]
    n = s_in[0].numel()
    cache = [torch.zeros(n, device=dev) for _ in range(5)] + [torch.zeros((11, n), device=dev)] + \
            [torch.zeros_like(x) for x in s_in[2:]] * 2
    cache = cache[:6] + [torch.zeros_like(x) for x in s_in[2:]] + [torch.zeros_like(x) for x in s_in[2:]]
    ref.forward_step(s_in, c_in, p_in, out, cache)
    torch.cuda.synchronize()
    for f, a, b in zip(STATE_FIELDS, state_arrays(nxt), [o.cpu().numpy() for o in out]):
        assert rel_l2(a, b) < 1e-5, (name, f, rel_l2(a, b))
    # and the CPU oracle (FP32 build) is pinned by the same kernels
    P = ob.Problem(cfg, "f32", solver="rbgs", iterations=40)
    onxt, _, _, _ = P.forward_step(st, ctl, PARAMS)
    for f, a, b in zip(STATE_FIELDS, state_arrays(onxt), [o.cpu().numpy() for o in out]):
        assert rel_l2(a, b) < 1e-5, ("oracle", name, f, rel_l2(a, b))


def test_pcg_step_matches_reference_kernels_with_converged_sweeps(cuda):
    """The plain method (Jacobi-PCG stopped at a 1e-6 relative residual)
    against the reference kernels with their red-black sweeps iterated until
    their FP32 rounding floor: both solve the same system, and the solve
    error a 1e-6 residual leaves in the velocity (~1e-8 relative, measured
    with the FP64 oracle) lies far below the 1e-5 bar.  Sweeps stopped at
    1e-6 themselves would not do: Gauss-Seidel's error at a given residual is
    dominated by smooth modes and measured 2.8e-5 on v at 24^3."""
    from common import product_domain, reference_step
    cfg = with_solver(scenario("plume", res=(24, 24, 24)), "pcg", iterations=20000, tolerance=1e-6)
    res = tuple(cfg.resolution)
    st, ctl = seeded_state(res, seed=25, amp=0.2), seeded_control(res, seed=26)
    model, ctx, nxt, k, stats = run_product(cfg, st, ctl)
    assert stats["final_residual"] <= 1e-6
    ref, sweeps, residual = reference_step(cfg, product_domain(ctx), st, ctl, PARAMS, tolerance=1e-9)
    assert residual < 3e-7 and sweeps > 0
    for f, a, b in zip(STATE_FIELDS, state_arrays(nxt), state_arrays(ref)):
        assert rel_l2(a, b) < 1e-5, (f, rel_l2(a, b), sweeps, residual)


def test_pressure_solve_reports_convergence_and_respects_the_cap(cuda):
    cfg = with_solver(scenario("plume", res=(20, 20, 20)), "pcg", iterations=20000, tolerance=1e-6)
    st, ctl = seeded_state(tuple(cfg.resolution), seed=27), seeded_control(tuple(cfg.resolution), seed=28)
    _, _, _, _, stats = run_product(cfg, st, ctl)
    assert stats["status"] == 0 and 0 < stats["final_residual"] <= 1e-6 and stats["iterations"] > 10
    capped = with_solver(cfg, "pcg", iterations=5, tolerance=1e-6)
    _, _, _, _, s2 = run_product(capped, st, ctl)
    assert s2["status"] == 2 and s2["iterations"] <= 5 and s2["final_residual"] > 1e-6


def test_warm_start_exact_guess_and_fallback(cuda):
    import torch
    from diff_solver_b200 import _native as N
    cfg = scenario("colliders", res=(20, 18, 16))
    model_cfg = with_solver(cfg, "pcg", iterations=20000, tolerance=1e-8)
    st = seeded_state(tuple(cfg.resolution), seed=29)
    P = ob.Problem(model_cfg, "f64")
    rhs = P.pressure_rhs(st["velocity"])
    p, _ = P.pcg(rhs, 20000, 1e-13)
    from diff_solver_b200.model import ExecutionMode, Model
    model = Model(model_cfg)
    ctx = model.allocate_context(ExecutionMode.forward)
    L = N.lib()
    g = ctx.native.grid
    ws = torch.zeros(L.xs_projection_workspace_bytes(g), dtype=torch.uint8, device="cuda")
    rhs_t = torch.as_tensor(rhs, dtype=torch.float32, device="cuda")
    out = torch.zeros_like(rhs_t)
    mask = ctx.native.cell_mask

    def solve(guess):
        s = N.XsPressureSolve(0, 20000, 1e-8, None if guess is None else guess.data_ptr())
        N.check("solve", L.xs_pressure_solve(None, g, s, ctx.native.pressure_anchor, mask, ctx.native.pressure_boundary,
                                             rhs_t.data_ptr(), out.data_ptr(), ws.data_ptr()))
        st_ = N.XsSolveStats()
        N.check("stats", L.xs_read_solve_stats(None, ws.data_ptr(), st_))
        return st_
    cold = solve(None)
    exact = solve(torch.as_tensor(p, dtype=torch.float32, device="cuda"))
    assert exact.warm_start_used == 1 and exact.iterations < cold.iterations // 4
    garbage = solve(torch.full_like(rhs_t, 1e3))
    assert garbage.warm_start_used == 0 and garbage.status == 0 and garbage.iterations == cold.iterations
    assert rel_l2(out.cpu().numpy(), p) < 1e-5


@pytest.mark.parametrize("name,res", [("plume", (40, 20, 14)), ("periodic", (32, 24, 16)), ("fixed_values", (64, 16, 12)),
                                      ("vorticity", (32, 32, 32))])
@pytest.mark.parametrize("amp", [0.3, 3.0])
def test_tiled_advection_is_bit_identical_to_the_general_kernels(cuda, name, res, amp):
    """On grids without colliders and with a power-of-two spacing the step
    advects through the tile-staged kernels.  Their results must equal, bit
    for bit, those of the general per-face kernels on the same input (the
    operator-level entry points given an all-fluid cell mask, which selects
    the general kernels without changing the semantics): partial tiles, every
    boundary mode, and traces long enough (amp 3: up to 1.5 cells per step)
    to leave the staged halo."""
    import ctypes as C

    import torch
    from diff_solver_b200 import _native as N
    cfg = scenario(name, res=res)
    cfg.cell_size = 1.0 / 32.0
    cfg.time_step = 0.5 / 32.0
    cfg = with_solver(cfg, "pcg", iterations=20000, tolerance=1e-6)
    st, ctl = seeded_state(res, seed=31, amp=amp), seeded_control(res, seed=32)
    model, ctx, nxt, k, _ = run_product(cfg, st, ctl)
    L = N.lib()
    g = ctx.native.grid
    dev = torch.device("cuda")
    forced = [torch.as_tensor(a, device=dev).contiguous() for a in k["forced_velocity"]]
    raw = [torch.zeros_like(a) for a in forced]
    out = [torch.zeros_like(a) for a in forced]
    vb = ctx.native.velocity_boundary
    fluid = torch.zeros(int(np.prod(res)), dtype=torch.int32, device=dev)
    mask = C.c_void_p(fluid.data_ptr())
    N.check("advect", L.xs_advect_velocity_forward(None, g, mask, N.vec(forced), vb, N.vec(raw)))
    N.check("constrain", L.xs_constrain_velocity_forward(None, g, mask, N.vec([None, None, None]), N.vec(raw), vb, N.vec(out)))
    torch.cuda.synchronize()
    for a in range(3):
        assert np.array_equal(out[a].cpu().numpy().view(np.uint32), k["advected_velocity"][a].view(np.uint32)), (name, a)
    u = [torch.as_tensor(a, device=dev).contiguous() for a in nxt["velocity"]]
    for field, boundary in (("sourced_density", ctx.native.density_boundary), ("sourced_temperature", ctx.native.temperature_boundary)):
        src = torch.as_tensor(k[field], device=dev).contiguous()
        res_t = torch.zeros_like(src)
        N.check("advect_scalar", L.xs_advect_scalar_forward(None, g, mask, None, C.c_void_p(src.data_ptr()), N.vec(u), boundary, vb,
                                                            C.c_void_p(res_t.data_ptr())))
        torch.cuda.synchronize()
        want = nxt["density" if field == "sourced_density" else "temperature"]
        assert np.array_equal(res_t.cpu().numpy().view(np.uint32), want.view(np.uint32)), (name, field)
    # the operator-level entry points without a mask take the tile kernels
    tiled = [torch.zeros_like(a) for a in forced]
    N.check("advect tiled", L.xs_advect_velocity_forward(None, g, None, N.vec(forced), vb, N.vec(tiled)))
    torch.cuda.synchronize()
    for a in range(3):
        assert torch.equal(tiled[a].view(torch.int32), raw[a].view(torch.int32)), (name, "raw", a)
    # integration: the 3D-indexed collider-free kernel against the general one
    u0 = [torch.as_tensor(np.asarray(a, np.float32), device=dev).contiguous() for a in st["velocity"]]
    force = [torch.as_tensor(a, device=dev).contiguous() for a in k["force"]]
    integrated = {}
    for key, m in (("fast", None), ("general", mask)):
        o = [torch.zeros_like(a) for a in u0]
        N.check("integrate", L.xs_integrate_velocity_forward(None, g, m, N.vec(u0), N.vec(force), N.vec(o)))
        integrated[key] = o
    torch.cuda.synchronize()
    for a in range(3):
        assert torch.equal(integrated["fast"][a].view(torch.int32), integrated["general"][a].view(torch.int32)), (name, "integrate", a)
        assert np.array_equal(integrated["fast"][a].cpu().numpy().view(np.uint32), k["forced_velocity"][a].view(np.uint32))
