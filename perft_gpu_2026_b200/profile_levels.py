"""A workload with large BFS levels, for profiling the HBM-bound level
kernels (make+count, scan, staged generation) rather than the leaf.

    python -m perft_gpu_2026_b200.profile_levels [--roots 262144] [--depth 4]

Runs one batched perft over `roots` playout positions (0..60 plies, seed 3):
at depth 4 the level kernels handle ~30 M positions and ~0.9 G generated
edges.  Prints the level sizes and the device time of the whole pass.
"""
from __future__ import annotations

import argparse
import json
import time

import perft_gpu_2026_b200 as pg


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--roots", type=int, default=1 << 18)
    ap.add_argument("--depth", type=int, default=4)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--arena-gb", type=int, default=24)
    args = ap.parse_args()
    roots = [p for p in pg.random_playouts(3, args.roots, 0, 60) if pg.count_moves(p, True) > 0]
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=args.arena_gb << 30)
    eng.set_timing(True)
    for _ in range(args.reps):
        t = time.perf_counter()
        counts = eng.perft_batch(roots, [args.depth] * len(roots))
        wall = time.perf_counter() - t
    st = eng.last_stats()
    print(json.dumps({"roots": len(roots), "depth": args.depth, "nodes": sum(counts), "wall_s": wall,
                      "device_ms": st.device_ms, "leaf_ms": st.leaf_ms,
                      "level_sizes": [int(st.level_sizes[i]) for i in range(min(st.levels + 1, 16))]}))
    eng.close()


if __name__ == "__main__":
    main()
