"""bench.py's multi-GPU bookkeeping (replicas: one ensemble member per rank)
on CPU with the gloo backend, world size 2: the slowest rank's time sets the
step time, and the job's SYPD is the sum over the replicas."""
import os
import socket

import pytest

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = [10.0, 12.5][rank]  # this rank's timed milliseconds
    q.put((rank, bench.max_over_ranks(t, world, "cpu")))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 12.5, 1: 12.5}


def test_replica_sypd_sums_members():
    one = bench.replica_sypd(2.0, 1)
    assert bench.replica_sypd(2.0, 4) == pytest.approx(4 * one)
    assert one == pytest.approx((86400 / 2e-3) / 8760)
