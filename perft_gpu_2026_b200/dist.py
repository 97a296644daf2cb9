"""Multi-GPU sharding of one perft: one process per GPU (torch.distributed).

The perft tree splits into independent subtrees, so ranks need no data
exchange while they count: rank r takes the subtrees r, r+N, r+2N, ... of the
root's positions `split_plies` plies down, and one all-reduce of the u64
counts gives the total.  Works with the nccl backend (GPU engines) and the
gloo backend (host engines, used by the CPU tests).
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import perft_gpu_2026_b200 as pg


def subtrees(root: pg.Pos, plies: int) -> List[pg.Pos]:
    """Positions `plies` plies below root, in generation order (each with
    multiplicity one per move path, so their perfts sum to the root's)."""
    level = [root]
    for _ in range(plies):
        nxt = []
        for p in level:
            for m in pg.generate_moves(p):
                nxt.append(pg.make_move(p, m))
        level = nxt
    return level


def shard(items: Sequence, world: int, rank: int) -> list:
    """Round robin: items rank, rank + world, ..."""
    return list(items[rank::world])


def balanced_assignment(weights: Sequence[float], world: int) -> List[int]:
    """Owner rank of each item by greedy longest-processing-time bin packing:
    items in decreasing weight (ties by index) go to the least-loaded rank
    (ties by lowest rank).  Deterministic, so every rank computes the same
    assignment from the same weights."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    owner = [0] * len(weights)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += weights[i]
    return owner


def shard_balanced(items: Sequence, weights: Sequence[float], world: int, rank: int) -> list:
    """This rank's items under balanced_assignment, in their original order."""
    owner = balanced_assignment(weights, world)
    return [it for it, o in zip(items, owner) if o == rank]


def perft_sharded(root: pg.Pos, depth: int, count: Callable[[List[pg.Pos], int], int], world: int, rank: int,
                  split_plies: int = 2, weight: Callable[[List[pg.Pos]], Sequence[float]] = None) -> int:
    """This rank's share of perft(depth): count(positions, depth) is called on
    the rank's subtrees at depth - split_plies.  With `weight` (estimated
    subtree sizes, e.g. a shallow perft of each subtree or the scheduler
    network's prediction) the subtrees are bin-packed by size, else dealt
    round robin."""
    if depth <= split_plies:
        return count([root], depth) if rank == 0 else 0
    subs = subtrees(root, split_plies)
    mine = shard_balanced(subs, weight(subs), world, rank) if weight else shard(subs, world, rank)
    return count(mine, depth - split_plies) if mine else 0


def all_reduce_count(value: int, device=None) -> int:
    """Sums a u64 count over the process group (one collective)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.int64, device=device)
    dist.all_reduce(t)
    return int(t.item())
