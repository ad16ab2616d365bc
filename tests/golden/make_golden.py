"""Generates the golden vectors of tests/golden/: outputs of the reference's
own smoke kernels (solvers/smoke/operators.cu compiled for sm_100a by
oracle/build_ref.sh, driven in the order of model.cpp:341-389) on small
seeded problems.  Needs a CUDA GPU and the harness library.

    python tests/golden/make_golden.py <output-dir>

Inputs are not stored: they are regenerated from the seeds recorded in each
file with numpy's default_rng (tests/common.py), so the CPU test suite can
pin the oracle against these files without a GPU.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import torch  # noqa: E402

from common import PARAMS, SCENARIOS, scenario, seeded_control, seeded_state, state_arrays, with_solver  # noqa: E402
from oracle import binding as ob  # noqa: E402
from oracle import ref_binding as rb  # noqa: E402

RES = (12, 10, 8)
SWEEPS = 30
TANGENT_PARAMS = dict(ambient_temperature=0.3, density_buoyancy=-0.2, temperature_buoyancy=0.4, vorticity_confinement=0.5)


def golden_case(name):
    cfg = with_solver(scenario(name, res=RES), "rbgs", iterations=SWEEPS)
    P = ob.Problem(cfg, "f32")
    dev = torch.device("cuda")
    f32 = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float32, device=dev).contiguous()
    f64 = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64, device=dev).contiguous()
    domain = {"mask": torch.as_tensor(P.mask.astype(np.int32), device=dev), "cv": [f32(v) for v in P.collider_velocity],
              "cd": f32(P.collider_density), "ct": f32(P.collider_temperature), "anchor": P.anchor}
    if not P.has_colliders:
        domain["mask"] = torch.zeros_like(domain["mask"])
    ref = rb.Reference(cfg, domain)
    seeds = dict(state=31, control=32, state_tangent=33, control_tangent=34, state_adjoint=35)
    st, ctl = seeded_state(RES, seeds["state"]), seeded_control(RES, seeds["control"])
    s_in = [f32(a) for a in state_arrays(st)]
    c_in = [f32(ctl["density_source"]), f32(ctl["temperature_source"])] + [f32(a) for a in ctl["acceleration"]]
    params = [torch.tensor([PARAMS[k]], dtype=torch.float32, device=dev) for k in
              ("ambient_temperature", "density_buoyancy", "temperature_buoyancy", "vorticity_confinement")]
    nxt = [torch.zeros_like(x) for x in s_in]
    n = s_in[0].numel()
    cache = [torch.zeros(n, device=dev) for _ in range(5)] + [torch.zeros((11, n), device=dev)] + \
            [torch.zeros_like(x) for x in s_in[2:]] + [torch.zeros_like(x) for x in s_in[2:]]
    ref.forward_step(s_in, c_in, params, nxt, cache)
    # tangent
    vt, vc = seeded_state(RES, seeds["state_tangent"], amp=1.0), seeded_control(RES, seeds["control_tangent"], amp=1.0)
    st_t = [f32(a) for a in state_arrays(vt)]
    ct_t = [f32(vc["density_source"]), f32(vc["temperature_source"])] + [f32(a) for a in vc["acceleration"]]
    pt = [torch.tensor([TANGENT_PARAMS[k]], dtype=torch.float32, device=dev) for k in
          ("ambient_temperature", "density_buoyancy", "temperature_buoyancy", "vorticity_confinement")]
    nt = [torch.zeros_like(x) for x in s_in]
    ref.jvp_step(s_in, params, nxt, cache, st_t, ct_t, pt, nt)
    # adjoint
    w = seeded_state(RES, seeds["state_adjoint"], amp=1.0)
    na = [f64(a) for a in state_arrays(w)]
    pa = [torch.zeros_like(x) for x in na]
    ca = [torch.zeros(n, dtype=torch.float64, device=dev) for _ in range(5)]
    qa = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(4)]
    ref.vjp_step(s_in, params, nxt, cache, na, pa, ca, qa)
    torch.cuda.synchronize()
    out = {"resolution": np.array(RES), "sweeps": np.array(SWEEPS), "seeds": np.array([seeds[k] for k in sorted(seeds)]),
           "seed_names": np.array(sorted(seeds))}
    for i, f in enumerate(("density", "temperature", "u", "v", "w")):
        out[f"next_{f}"] = nxt[i].cpu().numpy()
        out[f"tangent_{f}"] = nt[i].cpu().numpy()
        out[f"adjoint_{f}"] = pa[i].cpu().numpy()
    out["sourced_density"] = cache[0].cpu().numpy()
    out["sourced_temperature"] = cache[1].cpu().numpy()
    for a, c in enumerate("xyz"):
        out[f"force_{c}"] = cache[2 + a].cpu().numpy()
        out[f"forced_{c}"] = cache[6 + a].cpu().numpy()
        out[f"advected_{c}"] = cache[9 + a].cpu().numpy()
    for i, f in enumerate(("density_source", "temperature_source", "acceleration_x", "acceleration_y", "acceleration_z")):
        out[f"control_adjoint_{f}"] = ca[i].cpu().numpy()
    out["parameter_adjoint"] = np.array([q.item() for q in qa])
    return out


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name in SCENARIOS:
        np.savez_compressed(os.path.join(outdir, f"reference_{name}.npz"), **golden_case(name))
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
