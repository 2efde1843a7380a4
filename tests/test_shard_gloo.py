"""The multi-GPU plumbing on the CPU: two ranks over gloo agree on the
domain partition without communicating, take the slowest rank's time, and
gather every rank's results (shard.py).  The GPU data path has no collective:
each rank advances its own lattices."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from multiphase_lbm_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        weights = [32 ** 3, 128 ** 3, 64 ** 3, 96 ** 3, 48 ** 3, 128 ** 3, 80 ** 3]
        parts = shard.partition(weights, world)
        t = shard.max_over_ranks(1.5 + rank)
        got = shard.gather_results({"rank": rank, "mine": parts[rank]})
        q.put((rank, parts, t, got))
    finally:
        dist.destroy_process_group()


def test_partition_balances_and_covers():
    from multiphase_lbm_b200 import shard
    w = [5, 1, 4, 4, 2, 3, 3, 8]
    parts = shard.partition(w, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert shard.partition(w, 1) == [list(range(len(w)))]
    assert shard.partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.partition(w, 0)


def test_two_ranks_over_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts0 = res[0][1]
    for rank, parts, t, got in res:
        assert parts == parts0              # same assignment on every rank
        assert t == 2.5                     # slowest rank's time
        assert [g["rank"] for g in got] == [0, 1]
        assert sorted(i for g in got for i in g["mine"]) == list(range(7))
