"""The multi-GPU sharding logic, run as two gloo ranks on CPU: every rank
counts its subtrees with the host engine and one all-reduce gives the total,
which must equal the single-process count."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import perft_gpu_2026_b200 as pg
from perft_gpu_2026_b200 import dist as pdist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, fen, depth, balanced, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    eng = pg.Engine(device=-1)
    root = pg.parse_fen(fen)

    def count(positions, d):
        return sum(eng.perft_cpu(p, d) for p in positions)

    weight = (lambda subs: [eng.perft_cpu(p, 2) for p in subs]) if balanced else None
    part = pdist.perft_sharded(root, depth, count, world, rank, weight=weight)
    total = pdist.all_reduce_count(part)
    q.put((rank, part, total))
    dist.barrier()
    dist.destroy_process_group()


def _bench_worker(rank, world, port, depth, q):
    """bench.py's multi-rank path: ShardedPerft's split and per-rank count,
    then the exact u64 reduction (host counting in place of the GPU batch)."""
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    eng = pg.Engine(device=-1)
    root = pg.config_position(4, 1)
    plan = pdist.ShardedPerft(root, depth, world, rank, lambda ps, d: [eng.perft_cpu(p, d) for p in ps])
    part = plan.run()
    total = pdist.all_reduce_count(part)
    # counts past 2^63 (a signed 64-bit all-reduce would wrap): each rank
    # contributes 2^64 - 1 - rank
    big = pdist.all_reduce_count((1 << 64) - 1 - rank)
    q.put((rank, part, total, big, len(plan.mine)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_bench_multi_rank_path_on_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    depth = 4
    procs = [ctx.Process(target=_bench_worker, args=(r, world, port, depth, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = pg.Engine(device=-1).perft_cpu(pg.config_position(4, 1), depth)
    assert all(total == want for _, _, total, _, _ in res)
    assert sum(part for _, part, _, _, _ in res) == want
    assert sum(n for *_, n in res) == len(pdist.subtrees(pg.config_position(4, 1), 2))
    assert all(big == sum((1 << 64) - 1 - r for r in range(world)) for _, _, _, big, _ in res)


@pytest.mark.parametrize("balanced", [False, True])
@pytest.mark.parametrize("fen,depth", [(pg.START_FEN, 4), ("r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -", 3)])
def test_two_rank_gloo_perft(fen, depth, balanced):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, fen, depth, balanced, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = pg.Engine(device=-1).perft_cpu(pg.parse_fen(fen), depth)
    assert all(total == want for _, _, total in res)
    assert sum(part for _, part, _ in res) == want
    assert all(part > 0 for _, part, _ in res)


def test_shard_covers_every_subtree_once():
    root = pg.parse_fen(pg.START_FEN)
    subs = pdist.subtrees(root, 2)
    assert len(subs) == 400
    parts = [pdist.shard(subs, 3, r) for r in range(3)]
    assert sum(len(p) for p in parts) == 400
    keys = sorted(s.key() for p in parts for s in p)
    assert keys == sorted(s.key() for s in subs)


def test_balanced_assignment_covers_every_item_once_and_balances():
    w = [float(x) for x in (97, 3, 50, 50, 12, 88, 7, 41, 41, 1, 66, 30)]
    for world in (1, 2, 3, 4):
        owner = pdist.balanced_assignment(w, world)
        assert len(owner) == len(w) and set(owner) <= set(range(world))
        parts = [pdist.shard_balanced(list(range(len(w))), w, world, r) for r in range(world)]
        assert sorted(i for p in parts for i in p) == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        # greedy LPT: no rank exceeds the mean by more than the largest item
        assert max(loads) <= sum(w) / world + max(w)
        assert owner == pdist.balanced_assignment(list(w), world)  # deterministic


def test_balanced_beats_round_robin_on_bench_subtrees():
    root = pg.config_position(4, 1)
    subs = pdist.subtrees(root, 2)
    eng = pg.Engine(device=-1)
    w = [eng.perft_cpu(p, 2) for p in subs]
    rr = [sum(w[i] for i in range(r, len(w), 4)) for r in range(4)]
    owner = pdist.balanced_assignment(w, 4)
    bal = [sum(x for x, o in zip(w, owner) if o == r) for r in range(4)]
    assert max(bal) <= max(rr)
    assert max(bal) - min(bal) <= max(w)
