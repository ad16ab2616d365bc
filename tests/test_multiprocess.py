"""The benchmark's multi-rank plumbing on CPU (world size 2, gloo).

bench.py runs one independent replica per GPU (the smoke step does not
shard); its only collectives are the barriers around the timed region and
the max over ranks of every elapsed time.  These run here on two gloo ranks
on 127.0.0.1; the GPU work itself is covered by the -m gpu tests."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # each rank's elapsed time; the benchmark reports the slowest
        elapsed = 10.0 + 5.0 * rank
        slowest = bench.max_over_ranks(elapsed, world)
        bench.barrier(world)
        out.put((rank, slowest))
    finally:
        dist.destroy_process_group()


def test_barrier_and_max_over_ranks_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    results = sorted(out.get(timeout=10) for _ in range(2))
    assert results == [(0, 15.0), (1, 15.0)]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(3.5, 1) == 3.5
