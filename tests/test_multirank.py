"""Multi-GPU bench path on CPU: two gloo ranks exercise the replica
coordination bench.py uses under torchrun (barrier, max over ranks of the
device time, whole-job throughput). No GPU and no collective on the data
path: every replica runs its own problem."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    bench.barrier(dist)
    ms = bench.max_over_ranks(dist, 10.0 + 5.0 * rank, "cpu")
    v = bench.aggregate_throughput(world, 1_048_576, 100, ms)
    q.put((rank, ms, v))
    bench.barrier(dist)
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]
    assert out[0][2] == pytest.approx(2 * 1_048_576 * 100 / 0.015)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(None, 3.5, "cpu") == 3.5
    assert bench.aggregate_throughput(1, 10, 2, 1000.0) == 20.0
