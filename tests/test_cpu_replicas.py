"""bench.py times every multi-rank measurement as the maximum over ranks of
the device-timed step (one all-reduce of the step time). This checks that
aggregation with world size 2 over gloo on the CPU: both ranks see the
slowest rank's time, and the whole-job throughput of ranks that each do the
same work is N x that work over that time."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, local = bench.dist_env()
    assert (r, w, local) == (rank, world, rank)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms, value = bench.replica_throughput(7.5e10, 40.0 + 5.0 * rank, world, dist, device="cpu")
        out[rank] = (ms, value)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_over_gloo():
    world = 2
    port = free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in (0, 1):
        ms, value = res[rank]
        assert ms == 45.0
        assert abs(value - 2 * 7.5e10 / 0.045) < 1e-3 * value


def test_single_process_needs_no_group():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    ms, value = bench.replica_throughput(1e10, 20.0, 1)
    assert ms == 20.0 and abs(value - 5e11) < 1.0
