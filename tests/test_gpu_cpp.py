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


def build_cpp_test():
    os.makedirs(os.path.dirname(BINARY), exist_ok=True)
    lib_dir = os.path.join(ROOT, "diff_solver_b200")
    cmd = ["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", SOURCE, "-L", lib_dir,
           "-ldiffsmoke", "-L", "/usr/local/cuda/lib64", "-lcudart", f"-Wl,-rpath,{lib_dir}", "-Wl,-rpath,/usr/local/cuda/lib64",
           "-o", BINARY]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_solver_tape_modes_agree(cuda):
    if not os.path.exists(BINARY) or os.path.getmtime(BINARY) < os.path.getmtime(SOURCE):
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
