"""The several-GPU host logic as world_size-2 gloo process groups on the CPU: every search
runs on exactly one rank, the bytes balance, the gathered hit list equals one process's,
and the timing is the slowest rank's."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from seticore_b200.replicas import shard


def test_shard_covers_each_item_once_and_balances():
    costs = [64, 8, 8, 128, 32, 32, 16, 256, 4, 4, 4]
    for world in (1, 2, 3, 4):
        parts = [shard(costs, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    with pytest.raises(ValueError):
        shard(costs, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _fake_search(i):
    """Stands in for one search: a deterministic hit list (index, drift) of search i."""
    return [(i, 1000 * i + k, k - 2) for k in range(i % 4)]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    from seticore_b200.replicas import barrier, gather_hits, max_over_ranks
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        costs = [(i * 37) % 11 + 1 for i in range(23)]
        mine = shard(costs, world, rank)
        local = {i: _fake_search(i) for i in mine}
        barrier(world)
        hits = gather_hits(local, world)
        t = max_over_ranks(float(rank + 1) * 1.5, world)
        q.put((rank, mine, hits, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_gather_equals_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [h for i in range(23) for h in _fake_search(i)]
    mines = {}
    for rank, mine, hits, t in out:
        assert hits == want
        assert t == 3.0
        mines[rank] = mine
    assert sorted(mines[0] + mines[1]) == list(range(23)) and not set(mines[0]) & set(mines[1])
