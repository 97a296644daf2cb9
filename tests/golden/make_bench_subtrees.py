"""Regenerates tests/golden/bench_subtrees.json: the benchmark position (4
random plies from the initial array, splitmix64 seed 1) and its children (one
ply down), in generation order.

bench.py's reference arm and CPU-baseline leg run the reference program on
the children (perft depth-1 each, one process per child: units of seconds, so
a process's start-up is a small part of its time); reading them from this
file keeps the engine's library out of those processes.

    python tests/golden/make_bench_subtrees.py
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main() -> None:
    import perft_gpu_2026_b200 as pg

    root = pg.config_position(4, 1)
    children = [pg.to_fen(pg.make_move(root, m)) for m in pg.generate_moves(root)]
    out = {"generator": "tests/golden/make_bench_subtrees.py", "root_fen": pg.to_fen(root),
           "position": "4 random plies from the initial array, splitmix64 seed 1", "children": children}
    with open(os.path.join(HERE, "bench_subtrees.json"), "w") as f:
        json.dump(out, f, indent=0)
        f.write("\n")


if __name__ == "__main__":
    main()
