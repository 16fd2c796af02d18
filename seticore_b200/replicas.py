"""Several GPUs: independent replicas.

Searches share nothing (no exchange step between coarse channels, beams or searches), so
N GPUs run N independent engines, one process per GPU.  The host side here decides which
searches a rank runs (shard: largest first to the least-loaded rank, by input bytes,
identically on every rank), brings the hit lists together (gather_hits: all_gather_object,
then concatenated in search order, the order one process would produce), and takes the
slowest rank's time (max_over_ranks).  It works over any torch.distributed backend:
NCCL on GPUs, gloo on CPUs (the tests).
"""
import heapq
from typing import List, Sequence


def shard(costs: Sequence[int], world: int, rank: int) -> List[int]:
    """Indices (ascending) of the items rank `rank` of `world` takes.  Items go largest
    first to the rank with the least total cost so far (ties: lowest rank, then lowest
    index), so every rank computes the same assignment without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    heap = [(0, r) for r in range(world)]
    mine = []
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        if r == rank:
            mine.append(i)
        heapq.heappush(heap, (load + int(costs[i]), r))
    return sorted(mine)


def gather_hits(local: dict, world: int) -> list:
    """local: {search index: hit list} of this rank.  Returns every rank's lists
    concatenated in search-index order (each search appears on exactly one rank)."""
    if world == 1:
        merged = local
    else:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, local)
        merged = {}
        for p in parts:
            for k, v in p.items():
                if k in merged:
                    raise RuntimeError(f"search {k} ran on two ranks")
                merged[k] = v
    out = []
    for k in sorted(merged):
        out.extend(merged[k])
    return out


def max_over_ranks(x: float, world: int) -> float:
    """The largest value of x over the ranks (the slowest rank's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
