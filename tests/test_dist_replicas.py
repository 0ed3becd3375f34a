"""The multi-GPU layout of bench.py is replicas only (one independent instance
per rank, no collective on the data path).  Its host plumbing — process-group
set-up from the torchrun environment, barriers, the max-over-ranks timing and
the reference arm running on rank 0 alone — is exercised here with two gloo
ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out):
    import sys
    sys.path[:0] = [ROOT, os.path.join(ROOT, "sdpx.jl_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    world, r, local = bench.dist_setup()
    assert (world, r, local) == (2, rank, rank)
    bench.barrier(world)
    mx = bench.max_over_ranks(1.5 + rank, world)
    # the reference arm does its work on rank 0 only; rank 1 returns at once
    if rank == 1:
        class A:
            workload = "sdp_m2000"
            steps = 1
            warmup = 0
        assert bench.run_reference(A, world, rank) is None
    bench.barrier(world)
    dist.destroy_process_group()
    out.put((rank, mx))


def test_two_gloo_ranks_replica_plumbing():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    assert codes == [0, 0], codes
    got = dict(out.get(timeout=5) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}
