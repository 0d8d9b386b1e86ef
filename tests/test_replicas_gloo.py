"""The multi-GPU form of bench.py is N independent replicas: each rank shards
its own seeded batch, and the process group carries only the barriers and the
max-over-ranks of the timings.  This checks that host plumbing with two gloo
ranks on the CPU: the shards differ, the reduction is the maximum, and the
whole-job throughput is the units of all ranks over the slowest rank's time.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as td

    import bench
    dist = bench.init_ranks(world, timeout_s=60)
    assert dist is not None and dist.get_backend() == "gloo"
    mols = bench.molecules_for(rank, 4)
    first = [int(z.sum()) for z, _ in mols]
    gathered = [None] * world
    td.all_gather_object(gathered, first)
    dev_ms = 100.0 + 25.0 * rank  # this rank's timing
    dist.barrier()
    slowest = bench.reduce_max(dist, dev_ms)
    molecules_per_rank, steps = 4, 2
    value = molecules_per_rank * world * steps / (slowest / 1e3)
    out.put((rank, gathered, slowest, value))
    dist.barrier()
    td.destroy_process_group()


def test_two_gloo_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    for rank, gathered, slowest, value in results:
        assert gathered[0] != gathered[1]        # each rank has its own shard
        assert slowest == pytest.approx(125.0)   # max over ranks
        assert value == pytest.approx(4 * 2 * 2 / 0.125)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.init_ranks(1) is None
    assert bench.reduce_max(None, 3.5) == 3.5
