"""Pins the CPU oracle (FP32 build) against golden vectors produced by the
reference's own kernels (tests/golden/make_golden.py, run on a B200)."""
import glob
import os

import numpy as np
import pytest

from common import PARAMS, ROOT, rel_l2, scenario, seeded_control, seeded_state, state_arrays, with_solver

from oracle import binding as ob

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "reference_*.npz")))
TPARAMS = dict(ambient_temperature=0.3, density_buoyancy=-0.2, temperature_buoyancy=0.4, vorticity_confinement=0.5)
FIELDS = ("density", "temperature", "u", "v", "w")


def test_golden_vectors_are_committed():
    assert len(GOLDEN) >= 5, "tests/golden/reference_*.npz missing (generate with tests/golden/make_golden.py on a GPU)"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[10:-4] for p in GOLDEN])
def test_oracle_matches_reference_kernels(path):
    g = np.load(path)
    name = os.path.basename(path)[len("reference_"):-len(".npz")]
    res = tuple(int(v) for v in g["resolution"])
    seeds = dict(zip([str(s) for s in g["seed_names"]], [int(s) for s in g["seeds"]]))
    cfg = with_solver(scenario(name, res=res), "rbgs", iterations=int(g["sweeps"]))
    cfg.inflows = []  # the reference kernels know no inflow spheres
    P = ob.Problem(cfg, "f32")
    st, ctl = seeded_state(res, seeds["state"]), seeded_control(res, seeds["control"])
    nxt, k, _, _ = P.forward_step(st, ctl, PARAMS)
    for f, a in zip(FIELDS, state_arrays(nxt)):
        assert rel_l2(a, g[f"next_{f}"]) < 1e-5, (name, f, rel_l2(a, g[f"next_{f}"]))
    assert rel_l2(k["sourced_density"], g["sourced_density"]) < 1e-6
    for a, c in enumerate("xyz"):
        assert rel_l2(k["force"][a], g[f"force_{c}"]) < 1e-6
        assert rel_l2(k["forced_velocity"][a], g[f"forced_{c}"]) < 1e-6
        assert rel_l2(k["advected_velocity"][a], g[f"advected_{c}"]) < 1e-5
    vt, vc = seeded_state(res, seeds["state_tangent"], amp=1.0), seeded_control(res, seeds["control_tangent"], amp=1.0)
    jv = P.jvp_step(st, PARAMS, nxt, k, vt, vc, TPARAMS)
    for f, a in zip(FIELDS, state_arrays(jv)):
        assert rel_l2(a, g[f"tangent_{f}"]) < 1e-4, (name, "jvp", f, rel_l2(a, g[f"tangent_{f}"]))
    w = seeded_state(res, seeds["state_adjoint"], amp=1.0)
    prev, cadj, padj, _ = P.vjp_step(st, PARAMS, nxt, k, w)
    for f, a in zip(FIELDS, state_arrays(prev)):
        assert rel_l2(a, g[f"adjoint_{f}"]) < 1e-4, (name, "vjp", f, rel_l2(a, g[f"adjoint_{f}"]))
    assert rel_l2(cadj["density_source"], g["control_adjoint_density_source"]) < 1e-4
    want = g["parameter_adjoint"]
    got = [padj.ambient_temperature, padj.density_buoyancy, padj.temperature_buoyancy, padj.vorticity_confinement]
    for i in range(3 + (1 if cfg.vorticity_confinement_enabled else 0)):
        assert abs(got[i] - want[i]) <= 1e-4 * max(abs(want[i]), 1e-6), (name, got, want)
