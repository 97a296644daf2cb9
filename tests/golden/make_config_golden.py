"""Regenerates tests/golden/ref_configs.json: the reference program's own
counts on the benchmark workloads, for the GPU parity tests.

Runs the reference's `-cpu -nott` path (oracle/_ref/perft_gpu_ref, built from
the reference sources by `make -C oracle ref REF=<dir>`), one process per
position, all host cores in parallel, on
  config 1  the position 8 random plies from the initial array (seed 0),
            perft 1..5;
  config 2  the position 4 random plies from the initial array (seed 1),
            perft 1..6 directly, and perft 7 as the sum of the reference's
            perft 6 of each root move's child (the split is checked: the
            children's perft 5 must sum to the reference's direct perft 6);
  config 3  the 4096 uneven roots (6..40-ply playouts, seed 2, roots with a
            legal move), perft 1..5 each; the fixture keeps perft 5 and a
            digest of the roots' FENs so the test knows it regenerated the
            same roots;
  config 4  256 evenly spaced rows of the learned scheduler's training set
            (playouts of 0..60 plies, seed 3, positions with a legal move,
            2^20 drawn), perft 1..4 each (the training labels);
  config 5  the position 2 random plies from the initial array (seed 4),
            perft 1..6 (the deep table run's shallow depths).
Positions come from the engine's workload generator (splitmix64 playouts,
moves sorted by UCI text); every count comes from the reference binary.

    python tests/golden/make_config_golden.py   # writes ref_configs.json
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REF = os.path.join(ROOT, "oracle", "_ref", "perft_gpu_ref")


def run_ref(fen: str, depth: int):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([REF, fen, str(depth), "-cpu", "-nott"], capture_output=True, text=True, env=env,
                         check=True).stdout
    counts = [int(l.split(":")[1].split(",")[0]) for l in out.splitlines() if l.startswith("Perft(")]
    if len(counts) != depth:
        raise RuntimeError(f"unexpected reference output for {fen!r}:\n{out}")
    return counts


def run_many(fens, depth):
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        return list(ex.map(lambda f: run_ref(f, depth), fens))


def fen_digest(fens) -> str:
    return hashlib.sha256("\n".join(fens).encode()).hexdigest()


def main() -> None:
    import perft_gpu_2026_b200 as pg

    out = {"generator": "tests/golden/make_config_golden.py", "source": "reference -cpu -nott (oracle/_ref)"}

    p1 = pg.config_position(8, 0)
    out["config1"] = {"fen": pg.to_fen(p1), "counts": run_ref(pg.to_fen(p1), 5)}
    print("config 1 done", flush=True)

    p2 = pg.config_position(4, 1)
    fen2 = pg.to_fen(p2)
    direct = run_ref(fen2, 6)
    kids = [pg.to_fen(pg.make_move(p2, m)) for m in pg.generate_moves(p2)]
    per_kid = run_many(kids, 6)
    if sum(c[4] for c in per_kid) != direct[5]:
        raise RuntimeError("root-move split disagrees with the direct perft 6")
    out["config2"] = {"fen": fen2, "counts": direct + [sum(c[5] for c in per_kid)],
                      "depth7": "sum of the reference's perft 6 over the root moves' children"}
    print("config 2 done", flush=True)

    roots = pg.uneven_roots(4096, 6, 40, seed=2)
    fens3 = [pg.to_fen(p) for p in roots]
    c3 = run_many(fens3, 5)
    out["config3"] = {"n": len(fens3), "fen_sha256": fen_digest(fens3), "depth": 5,
                      "perft5": [c[4] for c in c3], "total": sum(c[4] for c in c3)}
    print("config 3 done", flush=True)

    train = [p for p in pg.random_playouts(3, 1 << 20, 0, 60) if pg.count_moves(p, True) > 0]
    step = len(train) // 256
    idx = [i * step for i in range(256)]
    fens4 = [pg.to_fen(train[i]) for i in idx]
    out["config4"] = {"train_n": len(train), "rows": idx, "fens": fens4, "perft1_4": run_many(fens4, 4)}
    print("config 4 done", flush=True)

    p5 = pg.config_position(2, 4)
    out["config5"] = {"fen": pg.to_fen(p5), "counts": run_ref(pg.to_fen(p5), 6)}
    print("config 5 done", flush=True)

    with open(os.path.join(HERE, "ref_configs.json"), "w") as f:
        json.dump(out, f, indent=0)
        f.write("\n")


if __name__ == "__main__":
    main()
