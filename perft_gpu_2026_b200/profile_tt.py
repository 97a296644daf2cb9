"""A small transposition-table workload, for profiling the table leaf.

    python -m perft_gpu_2026_b200.profile_tt [--depth 8] [--dtt-mb 2000] [--arena-gb 2]

Start position with device tables of --dtt-mb MB: perft depth-1 (fills the
tables), then perft depth (the launch to capture: skip the first table-leaf
launch).  Both counts are checked against the known start-position totals.
"""
from __future__ import annotations

import argparse
import json

import perft_gpu_2026_b200 as pg

KNOWN = {5: 4865609, 6: 119060324, 7: 3195901860, 8: 84998978956, 9: 2439530234167}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--dtt-mb", type=int, default=2000)
    ap.add_argument("--arena-gb", type=int, default=2)
    args = ap.parse_args()
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=args.arena_gb << 30, device_tt_mb=args.dtt_mb,
                    host_tt_mb=256)
    p = pg.parse_fen(pg.START_FEN)
    eng.prepare(p, args.depth)
    eng.set_timing(True)
    warm = eng.perft_position(p, args.depth - 1)
    got = eng.perft_position(p, args.depth)
    st = eng.last_stats()
    for d, v in ((args.depth - 1, warm), (args.depth, got)):
        if d in KNOWN and v != KNOWN[d]:
            raise SystemExit(f"perft {d} = {v}, expected {KNOWN[d]}")
    print(json.dumps({"depth": args.depth, "nodes": got, "device_ms": st.device_ms, "leaf_ms": st.leaf_ms,
                      "leaf_edges": st.leaf_edges, "leaf_positions": st.leaf_positions}))
    eng.close()


if __name__ == "__main__":
    main()
