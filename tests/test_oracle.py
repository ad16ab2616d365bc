"""Known-answer and self-consistency tests of the CPU oracle (no GPU)."""
import numpy as np
import pytest

from common import PARAMS, SCENARIOS, rel_l2, scenario, seeded_control, seeded_state, sizes, state_arrays, with_solver

from oracle import binding as ob


@pytest.mark.parametrize("name", SCENARIOS)
def test_pressure_operator_is_symmetric(name):
    P = ob.Problem(scenario(name), "f64")
    n, _ = sizes(P.res)
    rng = np.random.default_rng(3)
    p, q = rng.standard_normal(n), rng.standard_normal(n)
    ap, aq = P.apply_operator(p), P.apply_operator(q)
    assert abs(ap @ q - p @ aq) <= 1e-12 * (abs(ap @ q) + 1)
    # positive definite on the active cells
    assert p @ ap > 0


@pytest.mark.parametrize("name", SCENARIOS)
def test_pcg_reaches_tolerance_and_matches_converged_rbgs(name):
    cfg = scenario(name)
    P = ob.Problem(cfg, "f64")
    st = seeded_state(P.res, seed=4)
    rhs = P.pressure_rhs(st["velocity"])
    p, stats = P.pcg(rhs, 5000, 1e-12)
    assert stats.converged and stats.final_residual <= 1e-11
    # the PCG solution is a fixed point of the reference's red-black sweep,
    # i.e. both solve the same system ...
    swept = P.rbgs(rhs, 1, p=p)
    assert rel_l2(swept, p) < 1e-9
    # ... and the sweeps drive the residual down towards it
    assert P.relative_residual(rhs, P.rbgs(rhs, 2000)) < P.relative_residual(rhs, P.rbgs(rhs, 200)) < 1e-1


def test_zero_velocity_advection_is_identity():
    cfg = scenario("plume")
    P = ob.Problem(cfg, "f64")
    st = seeded_state(P.res, seed=5)
    zero = [np.zeros_like(v) for v in st["velocity"]]
    out = P.advect_velocity(zero)
    for a in range(3):
        assert np.array_equal(out[a], zero[a])


def test_uniform_flow_keeps_a_constant_scalar():
    cfg = with_solver(scenario("plume"), "rbgs", iterations=10)
    cfg.inflows = []
    for f in cfg.density_boundary.faces():
        f.mode = ob._mode(1) and 1
    cfg.density_boundary.y_max.mode = 1
    P = ob.Problem(cfg, "f64")
    n, fc = sizes(P.res)
    st = {"density": np.full(n, 0.7), "temperature": np.full(n, 0.2), "velocity": [np.full(fc[0], 0.3), np.zeros(fc[1]), np.zeros(fc[2])]}
    ctl = {"density_source": np.zeros(n), "temperature_source": np.zeros(n), "acceleration": [np.zeros(n)] * 3}
    nxt, k, _, _ = P.forward_step(st, ctl, dict(PARAMS, density_buoyancy=0.0, temperature_buoyancy=0.0))
    assert np.allclose(nxt["density"], 0.7, atol=1e-12)


def test_projection_removes_divergence():
    cfg = with_solver(scenario("plume"), "pcg", iterations=5000, tolerance=1e-12)
    P = ob.Problem(cfg, "f64")
    st = seeded_state(P.res, seed=6)
    rhs = P.pressure_rhs(st["velocity"])
    p, _ = P.pcg(rhs, 5000, 1e-12)
    out = P.project_velocity(st["velocity"], p)
    rhs2 = P.pressure_rhs(out)
    # The reference never corrects boundary faces (operators.cu:904-910), so
    # the cells beside the open (fixed-pressure) top keep the ghost-cell part
    # of their divergence; every other cell is divergence free up to the
    # residual of the solve.
    nx, ny, nz = P.res
    interior = rhs2.reshape(nz, ny, nx)[:, : ny - 1, :]
    assert np.linalg.norm(interior) <= 1e-9 * np.linalg.norm(rhs)
    assert np.linalg.norm(rhs2.reshape(nz, ny, nx)[:, ny - 1, :]) > 1e-3 * np.linalg.norm(rhs)


@pytest.mark.parametrize("name", SCENARIOS)
def test_fp32_and_fp64_builds_agree(name):
    cfg = with_solver(scenario(name), "rbgs", iterations=20)
    P64, P32 = ob.Problem(cfg, "f64"), ob.Problem(cfg, "f32")
    st, ctl = seeded_state(P64.res, seed=7), seeded_control(P64.res, seed=8)
    a, _, _, _ = P64.forward_step(st, ctl, PARAMS)
    b, _, _, _ = P32.forward_step(st, ctl, PARAMS)
    for x, y in zip(state_arrays(a), state_arrays(b)):
        assert rel_l2(y, x) < 2e-5


@pytest.mark.parametrize("name", SCENARIOS)
def test_tangent_and_adjoint_are_transposes(name):
    """<J v, w> = <v, J^T w> for the reference step linearisation (fixed
    sweeps make the pressure map linear and exactly transposed)."""
    cfg = with_solver(scenario(name), "rbgs", iterations=15)
    P = ob.Problem(cfg, "f64")
    res = P.res
    st, ctl = seeded_state(res, seed=9), seeded_control(res, seed=10)
    nxt, k, _, _ = P.forward_step(st, ctl, PARAMS)
    v_state, v_ctl = seeded_state(res, seed=11, amp=1.0), seeded_control(res, seed=12, amp=1.0)
    v_par = dict(ambient_temperature=0.3, density_buoyancy=-0.2, temperature_buoyancy=0.4, vorticity_confinement=0.5)
    jv = P.jvp_step(st, PARAMS, nxt, k, v_state, v_ctl, v_par)
    w = seeded_state(res, seed=13, amp=1.0)
    prev, cadj, padj, _ = P.vjp_step(st, PARAMS, nxt, k, w)
    lhs = sum(float(np.dot(a, b)) for a, b in zip(state_arrays(jv), state_arrays(w)))
    rhs = sum(float(np.dot(a, b)) for a, b in zip(state_arrays(v_state), state_arrays(prev)))
    rhs += float(np.dot(v_ctl["density_source"], cadj["density_source"]) + np.dot(v_ctl["temperature_source"], cadj["temperature_source"]))
    rhs += sum(float(np.dot(a, b)) for a, b in zip(v_ctl["acceleration"], cadj["acceleration"]))
    rhs += (v_par["ambient_temperature"] * padj.ambient_temperature + v_par["density_buoyancy"] * padj.density_buoyancy +
            v_par["temperature_buoyancy"] * padj.temperature_buoyancy)
    if cfg.vorticity_confinement_enabled:
        rhs += v_par["vorticity_confinement"] * padj.vorticity_confinement
    assert abs(lhs - rhs) <= 1e-9 * max(abs(lhs), 1.0), (lhs, rhs)


def test_network_reference_operator_matches_the_c_oracle():
    """The 7-point operator of the warm-start network's energy loss (oracle/
    unet_reference.py) is the pressure matrix the C oracle restates from the
    reference's red-black Gauss-Seidel, on grids without solids."""
    import torch
    from common import scenario
    from oracle import binding as ob
    from oracle import unet_reference as R
    checked = 0
    for name in ("plume", "periodic", "fixed_values"):
        cfg = scenario(name, (12, 10, 8))
        P = ob.Problem(cfg, "f64", solver="pcg", iterations=10, tolerance=1e-8)
        if P.anchor < 12 * 10 * 8:  # an anchored (all-Neumann) problem drops one row
            continue
        rng = np.random.default_rng(1)
        u = rng.normal(size=12 * 10 * 8)
        want = P.apply_operator(u)
        modes = [int(f.mode) for f in cfg.pressure_boundary.faces()]
        got = R.apply_operator(torch.from_numpy(u.reshape(1, 8, 10, 12)), modes).numpy().reshape(-1)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
        checked += 1
    assert checked >= 2
