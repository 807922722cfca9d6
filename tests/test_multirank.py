"""Multi-GPU bench path on CPU: two gloo ranks exercise the coordination
bench.py uses under torchrun (barrier, max over ranks of the device time,
whole-job throughput; the blast runs as replicas) and the split of the
batched ensemble across ranks (greedy size balance, computed on every rank
without a collective; each problem on exactly one rank). No GPU and no
collective on the data path."""
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


def test_ensemble_partition_covers_every_problem_once_and_balances():
    import bench
    import spd_k_b200.batch as B
    cfgs = bench.batched_configs(64)
    dof = [B.problem_dof(c) for c in cfgs]
    for world in (1, 2, 3, 8):
        parts = B.partition(cfgs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cfgs)))
        loads = [sum(dof[i] for i in p) for p in parts]
        # LPT bound: no rank exceeds the mean by more than the largest problem
        assert max(loads) - sum(loads) / world <= max(dof)
    assert B.partition(cfgs[:3], 8)[5] == []          # more ranks than problems
    c = cfgs[0]
    n = c["p"] + 1
    assert B.problem_dof(c) == c["N"][0] * c["N"][1] * n * n


def test_ensemble_waves_keep_order_and_bound_each_wave():
    import bench
    import spd_k_b200.batch as B
    cfgs = bench.batched_configs(512)
    total = sum(B.problem_dof(c) for c in cfgs)
    ws = B.waves(cfgs, 1.0e8)
    assert [c for w in ws for c in w] == cfgs                     # every problem once, in order
    assert all(sum(B.problem_dof(c) for c in w) <= 1.0e8 for w in ws)
    assert len(ws) >= total / 1.0e8
    big = dict(cfgs[0], N=[512, 512, 1])
    assert B.waves([big], 1.0) == [[big]]                         # an oversized problem alone
    assert B.waves(cfgs, total) == [cfgs]


def _shard_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    import spd_k_b200.batch as B
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    idx, mine = B.shard(bench.batched_configs(40), rank, world)
    # the host-side exchange the bench performs: the slowest rank's time
    ms = bench.max_over_ranks(dist, float(sum(B.problem_dof(c) for c in mine)), "cpu")
    got = [None] * world
    dist.all_gather_object(got, idx)
    q.put((rank, idx, ms, got))
    bench.barrier(dist)
    dist.destroy_process_group()


def test_two_gloo_ranks_split_the_ensemble():
    import bench
    import spd_k_b200.batch as B
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, idx0, ms0, got0), (r1, idx1, ms1, got1) = out
    assert got0 == got1 == [idx0, idx1]             # both ranks computed the same split
    assert sorted(idx0 + idx1) == list(range(40)) and not set(idx0) & set(idx1)
    cfgs = bench.batched_configs(40)
    loads = [sum(B.problem_dof(cfgs[i]) for i in ix) for ix in (idx0, idx1)]
    assert ms0 == ms1 == float(max(loads))
