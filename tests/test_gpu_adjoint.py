"""GPU parity of the tangent (JVP) and adjoint (VJP) steps: CUDA product vs
the CPU oracle, vs the reference's own kernels, transposition and finite
differences."""
import numpy as np
import pytest

from common import (PARAMS, SCENARIOS, cache_arrays, from_model_state, rel_l2, scenario, seeded_control, seeded_state, state_arrays,
                    to_model_control, to_model_state, with_solver)

from oracle import binding as ob

pytestmark = pytest.mark.gpu

TPARAMS = dict(ambient_temperature=0.3, density_buoyancy=-0.2, temperature_buoyancy=0.4, vorticity_confinement=0.5)


class Setup:
    def __init__(self, cfg, seed=41):
        import torch
        from diff_solver_b200.model import ExecutionMode, Model, fill_parameters
        self.cfg = cfg
        self.res = tuple(cfg.resolution)
        self.model = Model(cfg)
        self.ctx = self.model.allocate_context(ExecutionMode.differentiable)
        self.st_arr, self.ctl_arr = seeded_state(self.res, seed), seeded_control(self.res, seed + 1)
        m, ctx = self.model, self.ctx
        self.st = to_model_state(m, ctx, self.st_arr)
        self.ctl = to_model_control(m, ctx, self.ctl_arr)
        self.par = fill_parameters(m.allocate_parameters(ctx), **PARAMS)
        self.nxt = m.allocate_state(ctx)
        self.cache = m.allocate_step_cache(ctx)
        m.forward_step(self.st, self.ctl, self.par, self.nxt, self.cache, ctx)
        torch.cuda.synchronize()

    def vjp(self, w_arr):
        import torch
        m, ctx = self.model, self.ctx
        w = to_model_state(m, ctx, w_arr, dtype="adjoint")
        prev = m.allocate_state_adjoint(ctx)
        ca = m.allocate_control_adjoint(ctx)
        pa = m.allocate_parameter_adjoint(ctx)
        m.vjp_step(self.st, self.ctl, self.par, self.nxt, self.cache, w, prev, ca, pa, ctx)
        torch.cuda.synchronize()
        cad = {"density_source": ca.density_source.values.cpu().numpy(), "temperature_source": ca.temperature_source.values.cpu().numpy(),
               "acceleration": [ca.external_acceleration.x.values.cpu().numpy(), ca.external_acceleration.y.values.cpu().numpy(),
                                ca.external_acceleration.z.values.cpu().numpy()]}
        pad = [float(t.item()) for t in (pa.ambient_temperature, pa.density_buoyancy, pa.temperature_buoyancy, pa.vorticity_confinement)]
        return from_model_state(m, prev), cad, pad

    def jvp(self, v_state, v_ctl, v_par):
        import torch
        from diff_solver_b200.model import fill_parameters
        m, ctx = self.model, self.ctx
        st = to_model_state(m, ctx, v_state)
        ct = to_model_control(m, ctx, v_ctl)
        pt = fill_parameters(m.allocate_parameter_tangent(ctx), **v_par)
        out = m.allocate_state_tangent(ctx)
        m.jvp_step(self.st, self.ctl, self.par, self.nxt, self.cache, st, ct, pt, out, ctx)
        torch.cuda.synchronize()
        return from_model_state(m, out)


def _dot_state(a, b):
    return sum(float(np.dot(np.asarray(x, np.float64), np.asarray(y, np.float64))) for x, y in zip(state_arrays(a), state_arrays(b)))


@pytest.mark.parametrize("name", SCENARIOS)
def test_vjp_matches_oracle(cuda, name):
    cfg = with_solver(scenario(name), "pcg", iterations=20000, tolerance=1e-10)
    s = Setup(cfg)
    w = seeded_state(s.res, seed=43, amp=1.0)
    prev, cad, pad = s.vjp(w)
    P = ob.Problem(cfg, "f32", solver="pcg", iterations=20000, tolerance=1e-13)
    oprev, ocad, opad, _ = P.vjp_step(s.st_arr, PARAMS, from_model_state(s.model, s.nxt), cache_arrays(s.cache), w)
    for f, a, b in zip(("density", "temperature", "u", "v", "w"), state_arrays(prev), state_arrays(oprev)):
        assert rel_l2(a, b) < 1e-4, (name, f, rel_l2(a, b))
    assert rel_l2(cad["density_source"], ocad["density_source"]) < 1e-4
    for a in range(3):
        assert rel_l2(cad["acceleration"][a], ocad["acceleration"][a]) < 1e-4
    want = [opad.ambient_temperature, opad.density_buoyancy, opad.temperature_buoyancy, opad.vorticity_confinement]
    for g, o in zip(pad, want):
        assert abs(g - o) <= 1e-4 * max(abs(o), 1e-6), (name, pad, want)


@pytest.mark.parametrize("name", SCENARIOS)
def test_jvp_matches_oracle(cuda, name):
    cfg = with_solver(scenario(name), "pcg", iterations=20000, tolerance=1e-10)
    s = Setup(cfg)
    vs, vc = seeded_state(s.res, seed=44, amp=1.0), seeded_control(s.res, seed=45, amp=1.0)
    out = s.jvp(vs, vc, TPARAMS)
    P = ob.Problem(cfg, "f32", solver="pcg", iterations=20000, tolerance=1e-13)
    want = P.jvp_step(s.st_arr, PARAMS, from_model_state(s.model, s.nxt), cache_arrays(s.cache), vs, vc, TPARAMS)
    for f, a, b in zip(("density", "temperature", "u", "v", "w"), state_arrays(out), state_arrays(want)):
        assert rel_l2(a, b) < 1e-4, (name, f, rel_l2(a, b))


@pytest.mark.parametrize("name", SCENARIOS)
def test_vjp_is_the_transpose_of_jvp(cuda, name):
    cfg = with_solver(scenario(name), "pcg", iterations=20000, tolerance=1e-10)
    s = Setup(cfg)
    vs, vc = seeded_state(s.res, seed=46, amp=1.0), seeded_control(s.res, seed=47, amp=1.0)
    w = seeded_state(s.res, seed=48, amp=1.0)
    jv = s.jvp(vs, vc, TPARAMS)
    prev, cad, pad = s.vjp(w)
    lhs = _dot_state(jv, w)
    rhs = _dot_state(vs, prev)
    rhs += float(np.dot(vc["density_source"], cad["density_source"]) + np.dot(vc["temperature_source"], cad["temperature_source"]))
    rhs += sum(float(np.dot(a, b)) for a, b in zip(vc["acceleration"], cad["acceleration"]))
    tp = [TPARAMS[k] for k in ("ambient_temperature", "density_buoyancy", "temperature_buoyancy", "vorticity_confinement")]
    rhs += sum(t * p for t, p in zip(tp[:3], pad[:3]))
    if cfg.vorticity_confinement_enabled:
        rhs += tp[3] * pad[3]
    assert abs(lhs - rhs) <= 1e-5 * max(abs(lhs), 1.0), (name, lhs, rhs)


@pytest.mark.parametrize("name", SCENARIOS)
def test_fixed_sweep_adjoint_matches_the_reference_kernels(cuda, name):
    """RBGS kind: the product's reversed sweeps (gather form) and tangent
    against the reference's own vjp/jvp kernels on identical inputs."""
    import torch
    from oracle import ref_binding as rb
    if not rb.available():
        pytest.skip("reference harness not built")
    cfg = with_solver(scenario(name), "rbgs", iterations=30)
    cfg.inflows = []  # set-inflows have no reference counterpart; their adjoint is checked against the oracle
    s = Setup(cfg)
    w = seeded_state(s.res, seed=49, amp=1.0)
    prev, cad, pad = s.vjp(w)
    vs, vc = seeded_state(s.res, seed=50, amp=1.0), seeded_control(s.res, seed=51, amp=1.0)
    jv = s.jvp(vs, vc, TPARAMS)
    d = s.ctx.domain
    ref = rb.Reference(cfg, {"mask": d.cell_mask, "cv": list(d.collider_velocity.components()), "cd": d.collider_density.values,
                             "ct": d.collider_temperature.values, "anchor": d.pressure_anchor})
    dev = torch.device("cuda")
    f32 = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float32, device=dev).contiguous()
    f64 = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64, device=dev).contiguous()
    m = s.model
    state = m._state_tensors(s.st)
    nxt = m._state_tensors(s.nxt)
    k = s.cache
    cache = [k.sourced_density.values, k.sourced_temperature.values, k.force.x.values, k.force.y.values, k.force.z.values, k.vorticity,
             *k.forced_velocity.components(), *k.advected_velocity.components()]
    params = [s.par.ambient_temperature, s.par.density_buoyancy, s.par.temperature_buoyancy, s.par.vorticity_confinement]
    na = [f64(a) for a in state_arrays(w)]
    pa = [torch.zeros_like(x) for x in na]
    n = na[0].numel()
    ca = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(5)]
    qa = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(4)]
    ref.vjp_step(state, params, nxt, cache, na, pa, ca, qa)
    nt = [torch.zeros_like(x) for x in state]
    pt = [torch.tensor([TPARAMS[q]], dtype=torch.float32, device=dev) for q in
          ("ambient_temperature", "density_buoyancy", "temperature_buoyancy", "vorticity_confinement")]
    ref.jvp_step(state, params, nxt, cache, [f32(a) for a in state_arrays(vs)],
                 [f32(vc["density_source"]), f32(vc["temperature_source"])] + [f32(a) for a in vc["acceleration"]], pt, nt)
    torch.cuda.synchronize()
    for f, a, b in zip(("density", "temperature", "u", "v", "w"), state_arrays(prev), [t.cpu().numpy() for t in pa]):
        assert rel_l2(a, b) < 1e-5, ("vjp", name, f, rel_l2(a, b))
    for f, a, b in zip(("density", "temperature", "u", "v", "w"), state_arrays(jv), [t.cpu().numpy() for t in nt]):
        assert rel_l2(a, b) < 1e-5, ("jvp", name, f, rel_l2(a, b))
    for g, o in zip(pad, [q.item() for q in qa]):
        assert abs(g - o) <= 1e-5 * max(abs(o), 1e-6)


@pytest.mark.parametrize("name,res", [("plume", (40, 20, 14)), ("periodic", (32, 24, 16)), ("fixed_values", (64, 16, 12))])
@pytest.mark.parametrize("amp", [0.3, 3.0])
def test_tiled_advection_adjoints_match_the_general_kernels(cuda, name, res, amp):
    """The tile-staged advection adjoints (shared-memory FP64 accumulation,
    grids without colliders and with a power-of-two spacing) against the
    general per-face kernels (selected by an all-fluid cell mask, same
    semantics) on the same seeded adjoints: the same products, summed in
    another order, so equal to FP64 rounding (1e-12 relative L2)."""
    import ctypes as C

    import torch
    from diff_solver_b200 import _native as N
    from diff_solver_b200.model import ExecutionMode, Model
    cfg = scenario(name, res=res)
    cfg.cell_size = 1.0 / 32.0
    cfg.time_step = 0.5 / 32.0
    model = Model(cfg)
    ctx = model.allocate_context(ExecutionMode.forward)
    L = N.lib()
    g = ctx.native.grid
    vb = ctx.native.velocity_boundary
    dev = torch.device("cuda")
    rng = np.random.default_rng(51)
    n = int(np.prod(res))
    fsz = [(res[0] + 1) * res[1] * res[2], res[0] * (res[1] + 1) * res[2], res[0] * res[1] * (res[2] + 1)]
    u = [torch.as_tensor(rng.uniform(-amp, amp, f), dtype=torch.float32, device=dev) for f in fsz]
    oa = [torch.as_tensor(rng.normal(size=f), dtype=torch.float64, device=dev) for f in fsz]
    fluid = torch.zeros(n, dtype=torch.int32, device=dev)
    mask = C.c_void_p(fluid.data_ptr())
    results = []
    for m in (None, mask):
        ua = [torch.zeros(f, dtype=torch.float64, device=dev) for f in fsz]
        N.check("vjp", L.xs_advect_velocity_vjp(None, g, m, N.vec(u), vb, N.vec(oa), N.vec(ua)))
        src = torch.as_tensor(rng.uniform(0, 1, n), dtype=torch.float32, device=dev) if m is None else results[0][1]
        so = torch.as_tensor(rng.normal(size=n), dtype=torch.float64, device=dev) if m is None else results[0][2]
        sa = torch.zeros(n, dtype=torch.float64, device=dev)
        ua2 = [torch.zeros(f, dtype=torch.float64, device=dev) for f in fsz]
        N.check("scalar vjp", L.xs_advect_scalar_vjp(None, g, m, C.c_void_p(src.data_ptr()), N.vec(u), ctx.native.density_boundary, vb,
                                                     C.c_void_p(so.data_ptr()), C.c_void_p(sa.data_ptr()), N.vec(ua2)))
        torch.cuda.synchronize()
        results.append(([t.cpu().numpy() for t in ua], src, so, sa.cpu().numpy(), [t.cpu().numpy() for t in ua2]))
    tiled, general = results
    for a in range(3):
        assert rel_l2(tiled[0][a], general[0][a]) < 1e-12, (name, "velocity", a, rel_l2(tiled[0][a], general[0][a]))
        assert rel_l2(tiled[4][a], general[4][a]) < 1e-12, (name, "scalar->velocity", a)
    assert rel_l2(tiled[3], general[3]) < 1e-12, (name, "scalar->source")


@pytest.mark.parametrize("name,res", [("plume", (40, 20, 14)), ("periodic", (32, 24, 16))])
def test_open_integrate_adjoint_is_bit_identical_to_the_general_kernel(cuda, name, res):
    """Without colliders the integration adjoint's per-face division by the
    fluid cells beside the face is an exact halving (two) or nothing (one, on
    the domain boundary): the mask-free kernel matches the general one (an
    all-fluid mask) bit for bit."""
    import torch
    from diff_solver_b200 import _native as N
    from diff_solver_b200.model import ExecutionMode, Model
    cfg = scenario(name, res=res)
    ctx = Model(cfg).allocate_context(ExecutionMode.forward)
    L = N.lib()
    n = int(np.prod(res))
    fsz = [(res[0] + 1) * res[1] * res[2], res[0] * (res[1] + 1) * res[2], res[0] * res[1] * (res[2] + 1)]
    dev = torch.device("cuda")
    gen = torch.Generator(device="cuda").manual_seed(5)
    oa = [torch.randn(f, dtype=torch.float64, device=dev, generator=gen) for f in fsz]
    fluid = torch.zeros(n, dtype=torch.int32, device=dev)
    out = []
    for mask in (None, C_ptr(fluid)):
        ua = [torch.zeros(f, dtype=torch.float64, device=dev) for f in fsz]
        fa = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(3)]
        N.check("integrate vjp", L.xs_integrate_velocity_vjp(None, ctx.native.grid, mask, N.vec(oa), N.vec(ua), N.vec(fa)))
        torch.cuda.synchronize()
        out.append([t.cpu().numpy() for t in ua + fa])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def C_ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())
