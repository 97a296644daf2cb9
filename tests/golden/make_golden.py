"""Regenerates tests/golden/ref_cpu_perft.json from the reference program.

Runs the reference's own `-cpu -nott` path (oracle/_ref/perft_gpu_ref, built
from the reference sources by `make -C oracle ref`) on
  * the positions named in the reference itself: the initial array
    (perft.cu:98), Kiwipete (README.md:32) and the 218-move position
    (chess.h:177);
  * hand-built edge cases written for this test suite (en passant with a
    rank discovery, pinned en-passant capturers, castling through/out of
    check, promotions, double check, mate and stalemate, and the two cases
    where the reference's countMoves merges moves);
  * random playouts from the initial array (splitmix64, moves sorted by UCI
    text) produced by the engine's workload generator,
and records the per-depth counts it prints.  Usage:

    python tests/golden/make_golden.py            # writes ref_cpu_perft.json
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF = os.path.join(ROOT, "oracle", "_ref", "perft_gpu_ref")

NAMED = [
    ("initial", "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", 6),
    ("kiwipete", "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -", 5),
    ("max_moves_218", "3Q4/1Q4Q1/4Q3/2Q4R/Q4Q2/3Q4/1Q4Rp/1K1BBNNk w - - 0 1", 3),
]

# Edge cases built for this suite (each legal and reachable in principle).
EDGE = [
    # two white pawns can both capture-promote on c8 (countMoves merges them)
    ("double_capture_promotion", "2n4k/1P1P4/8/8/8/8/8/4K3 w - - 0 1", 4),
    ("double_capture_promotion_black", "4k3/8/8/8/8/8/1p1p4/2N3KR b - - 0 1", 4),
    # black e7-e5 gave check; both d5 and f5 can take en passant
    ("double_ep_evasion", "k7/8/8/3PpP2/5K2/8/8/8 w - e6 0 1", 5),
    # dxe6 e.p. would open the fifth rank to the rook on h5
    ("ep_rank_discovery", "8/8/8/K2Pp2r/8/8/8/7k w - e6 0 1", 5),
    # d5 pinned on the b7-f3 diagonal: dxc6 e.p. stays on the pin line
    ("ep_pinned_on_line", "4k3/1b6/8/2pP4/8/5K2/8/8 w - c6 0 1", 5),
    # f5 pinned on the file: fxe6 e.p. leaves the file
    ("ep_pinned_off_line", "4k3/5r2/8/4pP2/8/8/8/5K2 w - e6 0 1", 5),
    # castling: f1 attacked (no O-O), d1 attacked (no O-O-O), b1 attacked (O-O-O fine)
    ("castle_through_check", "r3k2r/8/8/8/8/8/8/R3K2R w KQkq - 0 1", 4),
    ("castle_blocked_by_attack", "4k3/8/8/8/8/8/5r2/R3K2R w KQ - 0 1", 4),
    ("castle_b1_attacked", "4k3/8/8/8/8/8/1r6/R3K2R w KQ - 0 1", 4),
    ("castle_out_of_check", "4k3/8/8/8/8/8/4r3/R3K2R w KQ - 0 1", 4),
    # promotions, quiet and by capture, both colours
    ("promotions", "1r2k3/P6P/8/8/8/8/p6p/1R2K3 w - - 0 1", 4),
    # double check: only king moves
    ("double_check", "4k3/8/8/8/8/5n2/8/r3K3 w - - 0 1", 5),
    ("checkmate", "7k/6Q1/6K1/8/8/8/8/8 b - - 0 1", 3),
    ("stalemate", "7k/5Q2/6K1/8/8/8/8/8 b - - 0 1", 3),
    # pinned sliders and a pinned knight
    ("pins", "4k3/4r3/8/b7/8/2N5/3R4/4K3 w - - 0 1", 5),
]


def run_ref(fen: str, depth: int):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([REF, fen, str(depth), "-cpu", "-nott"], capture_output=True, text=True, env=env,
                         check=True).stdout
    counts = []
    for line in out.splitlines():
        if line.startswith("Perft("):
            counts.append(int(line.split(":")[1].split(",")[0]))
    if len(counts) != depth:
        raise RuntimeError(f"unexpected reference output for {fen!r}:\n{out}")
    return counts


def main() -> None:
    import perft_gpu_2026_b200 as pg

    cases = []
    for name, fen, d in NAMED + EDGE:
        pg.parse_fen(fen)  # every fixture must be a position the engine accepts
        cases.append({"name": name, "fen": fen, "counts": run_ref(fen, d)})
    # workload configs: 8 plies seed 0 (perft 5) and 4 plies seed 1 (perft 5 here)
    for name, plies, seed, d in [("cfg_8ply_seed0", 8, 0, 5), ("cfg_4ply_seed1", 4, 1, 5), ("cfg_2ply_seed4", 2, 4, 5)]:
        p = pg.config_position(plies, seed)
        fen = pg.to_fen(p)
        cases.append({"name": name, "fen": fen, "counts": run_ref(fen, d), "plies": plies, "seed": seed})
    # random playouts of 10..70 plies
    for seed in range(48):
        plies = 10 + (seed * 37) % 61
        p, played, _ = pg.random_playout(1000 + seed, plies)
        if pg.count_moves(p, True) == 0:
            continue
        fen = pg.to_fen(p)
        cases.append({"name": f"playout_{seed}", "fen": fen, "counts": run_ref(fen, 4),
                      "plies": plies, "seed": 1000 + seed})
    with open(os.path.join(HERE, "ref_cpu_perft.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "source": "reference -cpu -nott",
                   "cases": cases}, f, indent=1)
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    main()
