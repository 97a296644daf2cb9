"""Multi-GPU sharding of one perft: one process per GPU (torch.distributed).

The perft tree splits into independent subtrees, so ranks need no data
exchange while they count: each rank takes a share of the root's positions
`split_plies` plies down (round robin, or bin-packed by size), and one
all-gather of the per-rank u64 counts gives the exact total.  Works with the nccl backend (GPU engines) and the
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
    """Sums the ranks' u64 counts exactly (one collective): every rank's count
    travels as the bit pattern of a 64-bit word (all-gather) and the sum is
    taken in Python integers, so it is exact past 2^63 and past 2^64 (the
    128-bit totals the reference prints, uint128.h:13-108)."""
    import torch
    import torch.distributed as dist

    if not 0 <= value < (1 << 64):
        raise ValueError("a rank's count must fit 64 bits")
    word = value - (1 << 64) if value >= (1 << 63) else value
    t = torch.tensor([word], dtype=torch.int64, device=device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    return sum(int(x.item()) & ((1 << 64) - 1) for x in parts)


class ShardedPerft:
    """This rank's share of perft(depth) of one root, as bench.py runs it
    under torchrun: the root's positions `split_plies` plies down are
    bin-packed over the ranks by their exact perft(2) (balanced_assignment;
    every rank computes the same split), and run() counts this rank's
    subtrees at depth - split_plies with count_batch(positions, depth) ->
    counts (the engine's batched GPU call; a host loop in the CPU tests).
    all_reduce_count then gives the total."""

    def __init__(self, root: pg.Pos, depth: int, world: int, rank: int,
                 count_batch: Callable[[List[pg.Pos], int], Sequence[int]], split_plies: int = 2):
        if depth <= split_plies:
            raise ValueError("depth must exceed the split depth")
        self.count_batch = count_batch
        subs = subtrees(root, split_plies)
        self.weights = list(count_batch(subs, 2))
        self.mine = shard_balanced(subs, self.weights, world, rank)
        self.sub_depth = depth - split_plies

    def run(self) -> int:
        return int(sum(self.count_batch(self.mine, self.sub_depth))) if self.mine else 0
