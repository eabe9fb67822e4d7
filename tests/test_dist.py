"""The multi-GPU plumbing of bench.py (replicas only) on CPU: two gloo ranks
agree on the max-over-ranks time and the summed events, and the reference
arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(backend="gloo", timeout_s=60)
    d.barrier()
    mx = d.max(10.0 + rank)          # per-rank device time: the slowest rank counts
    sm = d.sum(1000 * (rank + 1))    # per-rank events: whole-job total
    d.barrier()
    d.close()
    q.put((rank, mx, sm))


@pytest.mark.parametrize("world", [2])
def test_replica_reductions(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, sm in got:
        assert mx == 10.0 + world - 1
        assert sm == sum(1000 * (r + 1) for r in range(world))


def _ref_rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(backend="gloo", timeout_s=60)
    # the reference arm: rank 0 measures, the other ranks leave without work
    q.put((rank, d.rank == 0))
    d.close()


def test_reference_arm_runs_on_rank_zero_only():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ref_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: True, 1: False}
