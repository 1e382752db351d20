"""The multi-rank plumbing of bench.py on CPU (two gloo ranks): the tensor
population shards into disjoint per-rank sets that cover it, and the per-rank
byte counts and times reduce to the job's sum and max."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        mine = bench.shard(bench.batch_shapes(25), rank, world)
        tot = bench.reduce_over_ranks([float(len(mine)), 10.0 * (rank + 1)], "sum", world, "cpu")
        mx = bench.reduce_over_ranks([1.5 + rank], "max", world, "cpu")
        out.put((rank, [m[3] for m in mine], tot, mx))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_shard_and_reduce():
    import bench

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = [s[3] for s in bench.batch_shapes(25)]
    got = res[0][1] + res[1][1]
    assert sorted(got) == sorted(seeds) and not set(res[0][1]) & set(res[1][1])
    for _, _, tot, mx in res:
        assert tot == [25.0, 30.0] and mx == [2.5]


def test_single_rank_is_identity():
    import bench

    assert bench.reduce_over_ranks([3.0, 4.0], "sum", 1, "cpu") == [3.0, 4.0]
    assert bench.shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
