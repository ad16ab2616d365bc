"""The forward example driver (examples/smoke/forward) against the
reference's own example kernels, built into oracle/_ref from
simulation.cu: the pulsed double-jet controls (write_control), the per-step
metrics (reduce_metrics), and whole ForwardSimulation steps at the example's
128 x 192 x 128 grid with its 160 red-black sweeps."""
import numpy as np
import pytest

from common import product_domain, rel_l2

pytestmark = pytest.mark.gpu

STEPS = (0, 1, 54, 107)


def _reference(sim, iterations=None):
    from oracle import ref_binding as rb
    if not rb.available():
        pytest.skip("reference harness not built")
    return rb.Reference(sim.model.configuration, product_domain(sim.context), iterations=iterations)


def test_write_control_matches_the_reference_kernel(cuda):
    import torch
    from diff_solver_b200.simulation import ForwardSimulation, write_control
    sim = ForwardSimulation()
    ref = _reference(sim)
    n = sim.model.cell_count
    for step in STEPS:
        write_control(sim.context, sim.control, step, sim.options)
        acc = sim.control.external_acceleration
        mine = [t.clone() for t in (sim.control.density_source.values, sim.control.temperature_source.values, acc.x.values,
                                    acc.y.values, acc.z.values)]
        theirs = [torch.zeros(n, device="cuda") for _ in range(5)]
        ref.write_control(step, sim.options, theirs[0], theirs[1], theirs[2:])
        torch.cuda.synchronize()
        for a, b in zip(mine, theirs):
            assert float(b.abs().max()) > 0.0
            assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-6, step


def test_reduce_metrics_matches_the_reference_kernel(cuda):
    import torch
    from diff_solver_b200.simulation import ForwardSimulation, reduce_metrics
    sim = ForwardSimulation()
    ref = _reference(sim)
    gen = torch.Generator(device="cuda").manual_seed(4)
    state, cache = sim.current_state, sim.step_cache
    for t in (state.density.values, state.temperature.values, *state.velocity.components(), *cache.advected_velocity.components()):
        t.uniform_(-0.5, 1.0, generator=gen)
    mine = torch.zeros(6, dtype=torch.float64, device="cuda")
    theirs = torch.zeros(6, dtype=torch.float64, device="cuda")
    reduce_metrics(sim.context, state, cache, mine)
    ref.reduce_metrics(state.density.values, state.temperature.values, cache.advected_velocity.components(), state.velocity.components(),
                       theirs)
    torch.cuda.synchronize()
    a, b = mine.cpu().numpy(), theirs.cpu().numpy()
    # maxima are exact; sums differ only in the order of the FP64 additions
    assert a[1] == b[1] and a[2] == b[2] and a[3] == b[3], (a, b)
    for k in (0, 4, 5):
        assert abs(a[k] - b[k]) <= 1e-12 * abs(b[k]), (k, a[k], b[k])


def test_forward_simulation_matches_the_reference_example(cuda):
    """Twelve example steps (controls, step with 160 red-black sweeps,
    metrics) through the library and through the reference's kernels in the
    example's order (simulation.cpp:94-120): metrics per step and the final
    state agree to 1e-5 relative."""
    import torch
    from common import PLUME_PARAMS  # noqa: F401
    from diff_solver_b200.simulation import ForwardSimulation
    sim = ForwardSimulation()
    o = sim.options
    ref = _reference(sim, iterations=o.pressure_iterations)
    n = sim.model.cell_count
    faces = sim.model.face_counts
    dev = "cuda"
    state = [torch.zeros(n, device=dev), torch.zeros(n, device=dev)] + [torch.zeros(f, device=dev) for f in faces]
    nxt = [torch.zeros_like(t) for t in state]
    control = [torch.zeros(n, device=dev) for _ in range(5)]
    params = [torch.tensor([v], dtype=torch.float32, device=dev) for v in
              (o.ambient_temperature, o.density_buoyancy, o.temperature_buoyancy, o.vorticity_confinement)]
    cache = [torch.zeros(n, device=dev) for _ in range(5)] + [torch.zeros((11, n), device=dev)] + \
            [torch.zeros(f, device=dev) for f in faces] + [torch.zeros(f, device=dev) for f in faces]
    metrics = torch.zeros(6, dtype=torch.float64, device=dev)
    cells = float(n)
    for step in range(12):
        sim.step()
        ref.write_control(step, o, control[0], control[1], control[2:])
        ref.forward_step(state, control, params, nxt, cache)
        ref.reduce_metrics(nxt[0], nxt[1], cache[9:12], nxt[2:5], metrics)
        torch.cuda.synchronize()
        r = metrics.cpu().numpy()
        m = sim.metrics
        h = float(np.float32(o.cell_size))
        want = {"density_mass": r[0] * h * h * h, "density_maximum": r[1], "temperature_maximum": r[2],
                "maximum_velocity": r[3], "pre_projection_divergence_rms": (r[4] / cells) ** 0.5,
                "post_projection_divergence_rms": (r[5] / cells) ** 0.5}
        for k, v in want.items():
            got = getattr(m, k)
            assert abs(got - v) <= 1e-5 * max(abs(v), 1e-30), (step, k, got, v)
        state, nxt = nxt, state
    from diff_solver_b200.model import tensors_of
    for a, b in zip(tensors_of(sim.current_state), state):
        assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 1e-5


def test_divergence_after_a_converged_projection_lies_in_the_top_layer(cuda):
    """With Jacobi-PCG to 1e-6, the divergence the example's metrics report
    after the projection sits in the top layer of cells: the open top is a
    p = 0 face of the pressure system, but the projection leaves boundary
    faces as they are (operators.cu:904-910).  The reduction's total equals
    the per-layer split."""
    from diff_solver_b200.data import PressureSolver
    from diff_solver_b200.simulation import ForwardSimulation, ForwardSimulationOptions, divergence_by_layer
    o = ForwardSimulationOptions(pressure_solver=PressureSolver.jacobi_pcg, pressure_tolerance=1e-6)
    sim = ForwardSimulation(o)
    for _ in range(20):
        sim.step()
    top, rest = divergence_by_layer(sim.current_state, o.resolution, o.cell_size)
    total = sim.metrics.post_projection_divergence_rms ** 2 * sim.model.cell_count
    assert top + rest > 0.0
    assert top >= 0.999 * (top + rest), (top, rest)
    assert abs(total - (top + rest)) <= 1e-6 * (top + rest), (total, top, rest)
    assert sim.metrics.divergence_ratio > 0.0
