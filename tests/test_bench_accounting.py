"""The benchmark's byte and FLOP accounting on CPU (no GPU): the per-step
byte counts follow the stage table of the smoke step, the U-Net FLOP table
describes the network the library builds (its parameter count), and the CPU
oracle leg of the 64^3 record produces its timing record."""
import os
import sys

from diff_solver_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_convolution_table_matches_the_library_network():
    # every convolution holds 27 x C_in x C_out weights (no biases)
    weights = sum(27 * cin * cout for cin, cout, _ in bench.UNET_CONVOLUTIONS)
    assert weights == _native.lib().xs_warm_start_parameter_count() == 525_312


def test_unet_flops():
    v = 128 ** 3
    # level-0 first layer alone: 2 * 27 * 16 * 16 FLOPs per voxel
    first = 2.0 * 27 * 16 * 16 * v
    assert abs(first - 29.0e9) < 0.05e9
    # 1424 padded MACs per voxel of the network grid summed over the levels
    assert bench.unet_flops(v) == 2.0 * 27 * 1424 * v
    # real channels: 2 inputs to the first layer, 1 output of the last
    assert bench.unet_flops(v, padded=False) == 2.0 * 27 * (1424 - 256 + 32 - 256 + 16) * v
    assert bench.unet_flops(v / 8) * 8 == bench.unet_flops(v)


def test_forward_step_bytes_per_stage():
    n, f = bench.counts((256, 256, 256))
    assert (n, f) == (16_777_216, 50_528_256)
    sb = bench.stage_bytes(n, f)
    assert set(sb) == set(bench.STAGES)
    # the non-solve stages touch 8 FP32 face arrays (32F bytes, the face
    # term of 4 (8N + 8F)); their cell term, 88N, also counts the source,
    # acceleration and force fields the fused kernels read and write
    def fixed(n_, f_):
        return sum(v for v in bench.stage_bytes(n_, f_).values() if v is not None)
    assert fixed(0, 1) == 32.0 and fixed(1, 0) == 88.0
    assert fixed(n, f) == 32.0 * f + 88.0 * n


def test_pcg_bytes():
    n = 1000
    # one true-residual pass, no CG iteration
    assert bench.pcg_algorithmic_bytes(n, 0, 0) == 36.0 * n
    # CG iterations at 36 B/cell, smoothing adds 16 B/cell per smoothed one,
    # each refinement a residual pass and a fold
    assert bench.pcg_algorithmic_bytes(n, 10, 1, 4) == n * (360 + 64 + 72 + 24)


def test_reverse_step_bytes():
    n, f = bench.counts((64, 64, 64))
    b0 = bench.reverse_step_bytes(n, f, 0, 0)
    assert b0 == 4.0 * (8 * n + 8 * f) + 352.0 * n + 224.0 * f
    assert bench.reverse_step_bytes(n, f, 2, 3) - b0 == 36.0 * n * 5


def test_cpu_rollout_record():
    # the CPU leg of the 64^3 record on a small grid: consecutive FP64
    # oracle steps from a seeded start, stopped by the step count
    import numpy as np
    from oracle import binding as ob
    shape = (16, 16, 16)
    rng = np.random.default_rng(0)
    st = ob.zeros_state(shape, np.float64)
    st["velocity"] = [rng.uniform(-0.01, 0.01, v.shape) for v in st["velocity"]]
    rec = bench.cpu_rollout(st, shape, steps=3, budget_s=60.0)
    assert rec["steps"] == 3 and rec["steps_per_s"] > 0 and rec["pcg_iterations"] > 0
    assert rec["kind"] == "port" and rec["cores"] >= 1
