"""The C++ host API (include/xayah/*.hpp) on the GPU: simulate / jvp / vjp in
every tape mode through a compiled test program."""
import json
import os
import subprocess

import pytest

from common import ROOT

pytestmark = pytest.mark.gpu

SOURCE = os.path.join(ROOT, "tests", "cpp", "test_solver.cpp")
BINARY = os.path.join(ROOT, "tests", "cpp", "_build", "test_solver")


EXAMPLE_SOURCE = os.path.join(ROOT, "tests", "cpp", "forward_simulation.cpp")
EXAMPLE_BINARY = os.path.join(ROOT, "tests", "cpp", "_build", "forward_simulation")


def compile_program(source, binary):
    os.makedirs(os.path.dirname(binary), exist_ok=True)
    lib_dir = os.path.join(ROOT, "diff_solver_b200")
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", source, "-L", lib_dir,
           "-ldiffsmoke", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib_dir}", "-Wl,-rpath,/usr/local/cuda/lib64",
           "-o", binary]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def build_cpp_test():
    """The C++ test programs: the solver's tape modes and the example driver."""
    compile_program(SOURCE, BINARY)
    compile_program(EXAMPLE_SOURCE, EXAMPLE_BINARY)


def inputs():
    """Everything the test program is compiled from: its source and the
    headers it includes (a binary built against an older struct layout of
    the C ABI would pass the library misaligned arguments)."""
    inc = os.path.join(ROOT, "include")
    headers = [os.path.join(d, f) for d, _, fs in os.walk(inc) for f in fs if f.endswith((".h", ".hpp"))]
    return [SOURCE, *headers]


def stale(binary, sources):
    return not os.path.exists(binary) or any(os.path.getmtime(binary) < os.path.getmtime(s) for s in sources)


def test_cpp_forward_simulation_matches_the_python_driver(cuda):
    """The example's main program in C++ (include/xayah/forward_simulation.hpp)
    and the Python driver (diff_solver_b200/simulation.py) step the same scene
    through the same library: their metrics agree (the FP64 sums of the
    reduction only up to the order of their atomic additions)."""
    from diff_solver_b200.simulation import ForwardSimulation
    if stale(EXAMPLE_BINARY, [EXAMPLE_SOURCE, *inputs()]):
        compile_program(EXAMPLE_SOURCE, EXAMPLE_BINARY)
    r = subprocess.run([EXAMPLE_BINARY, "12", "4"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    cpp = [json.loads(line) for line in r.stdout.strip().splitlines()]
    assert [m["step"] for m in cpp] == [4, 8, 12]
    sim = ForwardSimulation()
    for step in range(12):
        sim.step()
        if sim.metrics.step % 4:
            continue
        want = cpp[sim.metrics.step // 4 - 1]
        for k, v in want.items():
            if k.endswith("milliseconds"):
                continue
            assert abs(getattr(sim.metrics, k) - v) <= 1e-12 * max(abs(v), 1e-300), (sim.metrics.step, k, getattr(sim.metrics, k), v)


def test_cpp_solver_tape_modes_agree(cuda):
    if stale(BINARY, inputs()):
        build_cpp_test()
    r = subprocess.run([BINARY], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    # the forward pass is deterministic: checkpointed rollouts reproduce store-all
    assert out["forward_checkpoint_vs_store_all"] == 0.0
    # reverse passes agree up to the order of FP64 atomic additions
    assert out["vjp_recompute_vs_store_all"] < 1e-9
    assert out["vjp_checkpoint_vs_store_all"] < 1e-9
    assert out["checkpoints"] == 3  # steps 0, 4, 6
    assert out["last_solve_status"] == 0
    assert abs(out["dot_jvp"] - out["dot_vjp"]) <= 1e-4 * max(abs(out["dot_jvp"]), 1e-12), out
    # a model carrying the (untrained) learned warm start still solves to 1e-6
    assert out["warm_solve_status"] == 0 and out["warm_solve_residual"] <= 1e-6 and out["warm_states"] == 4
