"""The multi-process path on CPU: two gloo ranks on 127.0.0.1 shard a batch of scenes, reduce
a timing by max and gather per-rank results (rtb200.dist), the plumbing bench.py --gpus N uses
with nccl."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from rtb200 import dist as rdist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, weights, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = rdist.shard_scenes(weights, rank, world)
        t = rdist.max_over_ranks(10.0 + rank, dist)
        got = rdist.gather_to_rank0(mine, dist)
        if rank == 0:
            q.put(("ok", mine, t, got))
        else:
            q.put(("ok1", mine, t, None))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_reduce_gather():
    weights = [1000, 500000, 2500, 80000, 80000, 1200, 300000, 7000, 45000, 999]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, weights, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    r0 = next(r for r in res if r[0] == "ok")
    r1 = next(r for r in res if r[0] == "ok1")
    assert r0[2] == 11.0 and r1[2] == 11.0              # max over ranks on both
    shards = r0[3]
    assert shards[0] == r0[1] and shards[1] == r1[1]
    assert sorted(shards[0] + shards[1]) == list(range(len(weights)))
    assert not set(shards[0]) & set(shards[1])
    loads = [sum(weights[i] for i in s) for s in shards]
    assert max(loads) <= 0.5 * sum(weights) + max(weights)  # LPT balance bound


def test_shard_single_rank_and_errors():
    assert rdist.shard_scenes([3, 1, 2], 0, 1) == [0, 1, 2]
    with pytest.raises(ValueError):
        rdist.shard_scenes([1], 2, 2)
    assert rdist.max_over_ranks(3.5) == 3.5
    assert rdist.gather_to_rank0({"a": 1}) == [{"a": 1}]
