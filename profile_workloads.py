"""Workloads for ncu captures of single kernels, each small enough that a
capture ends by itself.  The summaries under profiles/ name the command line
that produced them.

    python profile_workloads.py leaf   [--depth 7] [--arena-gb 2] [--reps 3] [--leaf-kernel K] [--leaf-threads T]
    python profile_workloads.py levels [--roots 16384] [--depth 5] [--arena-gb 6]
    python profile_workloads.py tt     [--depth 8] [--dtt-mb 2000] [--arena-gb 2]
    python profile_workloads.py gemm   [--m 4096] [--n 256] [--k 256] [--ta 0] [--tb 0] [--reps 20]

leaf    the bench position (4 random plies from the initial array, splitmix64
        seed 1) at perft --depth without tables, --reps times: each pass is
        one two-ply leaf launch over the position's perft(depth-2) edges, so
        `-k regex:k_leaf2 -s <reps-1> -c 1` captures the last pass's leaf
        launch, the same launch the benchmark times.  Prints the count, the
        CUDA-event leaf time and the move-count calls of that launch.
levels  one batched perft over --roots playout positions (0..60 plies, seed
        3): large BFS levels for the HBM-bound level kernels (make+count,
        scan, staged generation).
tt      the start position with device tables: perft depth-1 (fills the
        tables), then perft depth (the launch to capture: skip the first
        table-leaf launch).  Counts are checked against the known totals.
gemm    the scheduler network's tcgen05 GEMM on random BF16 operands: one
        checked launch, then --reps timed launches (CUDA events); prints the
        mean time and TFLOP/s.  The network's three products at a 4096-sample
        batch are (--ta 0 --tb 0 --m 4096 --n 256 --k 256: layer 2 forward),
        (--ta 1 --m 256 --k 4096: its weight gradient) and (--tb 1 --m 4096:
        its input gradient).
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import perft_gpu_2026_b200 as pg

START_TOTALS = {5: 4865609, 6: 119060324, 7: 3195901860, 8: 84998978956, 9: 2439530234167}


def leaf(args):
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=args.arena_gb << 30)
    if args.leaf_kernel or args.leaf_threads:
        eng.set_tuning(leaf_kernel=args.leaf_kernel, leaf_threads=args.leaf_threads)
    eng.set_timing(True)
    root = pg.config_position(4, 1)
    out = None
    for _ in range(args.reps):
        got = eng.perft_position(root, args.depth)
        st = eng.last_stats()
        if out is not None and got != out["nodes"]:
            raise SystemExit("count changed between passes")
        out = {"workload": "leaf", "depth": args.depth, "nodes": got, "device_ms": st.device_ms,
               "leaf_ms": st.leaf_ms, "leaf_edges": st.leaf_edges, "leaf_positions": st.leaf_positions,
               "leaf_kernel": eng.get_tuning().leaf_kernel, "leaf_threads": eng.get_tuning().leaf_threads}
    print(json.dumps(out))
    eng.close()


def levels(args):
    roots = [p for p in pg.random_playouts(3, args.roots, 0, 60) if pg.count_moves(p, True) > 0]
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=args.arena_gb << 30)
    eng.set_timing(True)
    for _ in range(args.reps):
        t = time.perf_counter()
        counts = eng.perft_batch(roots, [args.depth] * len(roots))
        wall = time.perf_counter() - t
    st = eng.last_stats()
    print(json.dumps({"workload": "levels", "roots": len(roots), "depth": args.depth, "nodes": sum(counts),
                      "wall_s": wall, "device_ms": st.device_ms, "leaf_ms": st.leaf_ms,
                      "level_sizes": [int(st.level_sizes[i]) for i in range(min(st.levels + 1, 16))]}))
    eng.close()


def tt(args):
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=args.arena_gb << 30, device_tt_mb=args.dtt_mb,
                    host_tt_mb=256)
    p = pg.parse_fen(pg.START_FEN)
    eng.prepare(p, args.depth)
    eng.set_timing(True)
    warm = eng.perft_position(p, args.depth - 1)
    got = eng.perft_position(p, args.depth)
    st = eng.last_stats()
    for d, v in ((args.depth - 1, warm), (args.depth, got)):
        if d in START_TOTALS and v != START_TOTALS[d]:
            raise SystemExit(f"perft {d} = {v}, expected {START_TOTALS[d]}")
    print(json.dumps({"workload": "tt", "depth": args.depth, "nodes": got, "device_ms": st.device_ms,
                      "leaf_ms": st.leaf_ms, "leaf_edges": st.leaf_edges, "leaf_positions": st.leaf_positions}))
    eng.close()


def gemm(args):
    import numpy as np

    rng = np.random.default_rng(1)
    m, n, k = args.m, args.n, args.k
    a = rng.uniform(-1, 1, size=m * k).astype(np.float32)
    b = rng.uniform(-1, 1, size=k * n).astype(np.float32)
    to_bits = lambda x: ((x.view(np.uint32) + 0x8000) >> 16).astype(np.uint16)
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 28)
    c, ms = eng.selftest_gemm(to_bits(a), to_bits(b), bool(args.ta), bool(args.tb), m, n, k, reps=args.reps)
    av = (to_bits(a).astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    bv = (to_bits(b).astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    am = av.reshape(k, m).T if args.ta else av.reshape(m, k)
    bm = bv.reshape(n, k).T if args.tb else bv.reshape(k, n)
    err = float(np.abs(c - am @ bm).max())
    print(json.dumps({"workload": "gemm", "m": m, "n": n, "k": k, "ta": args.ta, "tb": args.tb, "reps": args.reps,
                      "ms": ms, "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12, "max_abs_err": err}))
    eng.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="which", required=True)
    a = sub.add_parser("leaf")
    a.add_argument("--depth", type=int, default=7)
    a.add_argument("--arena-gb", type=int, default=2)
    a.add_argument("--reps", type=int, default=3)
    a.add_argument("--leaf-kernel", type=int, default=0)
    a.add_argument("--leaf-threads", type=int, default=0)
    a = sub.add_parser("levels")
    a.add_argument("--roots", type=int, default=1 << 14)
    a.add_argument("--depth", type=int, default=5)
    a.add_argument("--reps", type=int, default=1)
    a.add_argument("--arena-gb", type=int, default=6)
    a = sub.add_parser("tt")
    a.add_argument("--depth", type=int, default=8)
    a.add_argument("--dtt-mb", type=int, default=2000)
    a.add_argument("--arena-gb", type=int, default=2)
    a = sub.add_parser("gemm")
    a.add_argument("--m", type=int, default=4096)
    a.add_argument("--n", type=int, default=256)
    a.add_argument("--k", type=int, default=256)
    a.add_argument("--ta", type=int, default=0)
    a.add_argument("--tb", type=int, default=0)
    a.add_argument("--reps", type=int, default=20)
    args = ap.parse_args(argv)
    {"leaf": leaf, "levels": levels, "tt": tt, "gemm": gemm}[args.which](args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
