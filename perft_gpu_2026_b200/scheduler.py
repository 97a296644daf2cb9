"""The learned scheduler workload: build the training set, train the network
with the library's kernels, and evaluate it by scheduling a held-out batch.

    python -m perft_gpu_2026_b200.scheduler [--train-n 1048576] [--eval-n 16384] [--epochs 12]

Training set: n playouts of 0..60 plies from the initial array (splitmix64
seed 3, per-position streams), each labelled with its exact perft 1..4 by the
engine (batched GPU passes); targets are log2(1 + perft(k)).  Evaluation:
n held-out playouts (seed 3003) with depths uniform in 4..7 (seed 3004),
scheduled three ways on one GPU:
  plain     one count-then-allocate GPU call per position (the reference's
            perft_gpu_host_bfs sizing, host readback at every level)
  batched   one batched pass per depth, levels sized by count-then-allocate
  learned   the planner: predicted level sizes, bin-packing, root splits,
            one captured CUDA graph per batch
All three must give identical counts; prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import perft_gpu_2026_b200 as pg


def keep_movable(positions):
    return [p for p in positions if pg.count_moves(p, True) > 0]


def label(eng: pg.Engine, positions, depths=(1, 2, 3, 4), chunk=262144):
    """Exact perft(k) for every position, as an (n, len(depths)) float64 array."""
    out = np.zeros((len(positions), len(depths)), dtype=np.float64)
    for c0 in range(0, len(positions), chunk):
        part = pg.pack_slice(positions, c0, c0 + chunk)
        for j, d in enumerate(depths):
            out[c0:c0 + len(part), j] = eng.perft_batch(part, d)
    return out


def make_training_set(eng, n, seed=3):
    """(positions as one packed array, log2(1 + perft 1..4) as float32, exact counts)."""
    pos = pg.pack_positions(keep_movable(pg.random_playouts(seed, n, 0, 60)))
    counts = label(eng, pos)
    return pos, np.log2(1.0 + counts).astype(np.float32), counts


def eval_depths(n, seed=3004):
    depths, st = [], seed
    for _ in range(n):
        r, st = pg.splitmix64(st)
        depths.append(4 + ((r * 4) >> 64))
    return depths


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-n", type=int, default=1 << 20)
    ap.add_argument("--eval-n", type=int, default=16384)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--skip-plain", action="store_true")
    args = ap.parse_args()

    eng = pg.Engine(device=0, use_tt=False)
    t0 = time.perf_counter()
    pos, y, counts = make_training_set(eng, args.train_n)
    t_label = time.perf_counter()
    eng.mlp_init(seed=1, out_bias=list(y.mean(0)))
    base = float(((y - y.mean(0)) ** 2).mean())
    t1 = time.perf_counter()
    loss = eng.mlp_train(pos, y, epochs=args.epochs, batch=args.batch, lr=args.lr)
    t_train = time.perf_counter() - t1

    held = keep_movable(pg.random_playouts(3003, args.eval_n + args.eval_n // 8, 0, 60))[:args.eval_n]
    depths = eval_depths(len(held))
    pred = eng.mlp_predict(held)
    truth = np.log2(1.0 + label(eng, held))
    mae = np.abs(pred - truth).mean(0).tolist()

    res = {"train_n": len(pos), "label_s": t_label - t0, "train_s": t_train, "epochs": args.epochs,
           "train_mse": loss, "target_variance": base, "eval_n": len(held), "eval_mae_log2_by_depth": mae}

    t = time.perf_counter()
    learned, st = eng.perft_batch_planned(held, depths)
    res["learned_s"] = time.perf_counter() - t
    res["plan"] = {"batches": st.batches, "graph_batches": st.graph_batches, "retries": st.retries,
                   "split_roots": st.split_roots}
    t = time.perf_counter()
    batched = eng.perft_batch(held, depths)
    res["batched_s"] = time.perf_counter() - t
    assert batched == learned
    if not args.skip_plain:
        t = time.perf_counter()
        plain = [eng.perft_position(p, d) for p, d in zip(held, depths)]
        res["plain_s"] = time.perf_counter() - t
        assert plain == learned
        res["speedup_learned_vs_plain"] = res["plain_s"] / res["learned_s"]
    res["speedup_learned_vs_batched"] = res["batched_s"] / res["learned_s"]
    res["nodes"] = int(sum(learned))
    res["positions_per_s_learned"] = len(held) / res["learned_s"]
    print(json.dumps(res))
    eng.close()


if __name__ == "__main__":
    main()
