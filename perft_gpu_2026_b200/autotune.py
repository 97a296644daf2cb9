"""Autotuner for the GPU path's launch parameters.

Candidates: leaf kernel (one edge per thread / cooperative / one edge per
thread with the CTA's children ranked by move count / ranked with each
child's own-piece squares listed once / the same with four children per
thread balanced across the warps), the leaf's CTA size
(128/256/512), the staged generator's CTA size and tile (64 or 128
threads, 64 moves staged per thread) and the leaf fuse depth (two plies fused
in the leaf, or one with an extra BFS level).  Each candidate runs perft 7
of the bench position on the GPU (device time from the engine's CUDA events, median of 3);
the fastest is cached per GPU model and driver in
$XDG_CACHE_HOME/perft_b200/tuning.json (default ~/.cache/perft_b200) and
applied to the engine.

    python -m perft_gpu_2026_b200.autotune       # tune this GPU, print the result
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
import statistics
import subprocess
from typing import Dict, List, Optional

import perft_gpu_2026_b200 as pg

CACHE_DIR = os.path.join(os.environ.get("XDG_CACHE_HOME", os.path.expanduser("~/.cache")), "perft_b200")
CACHE = os.path.join(CACHE_DIR, "tuning.json")


def gpu_key(device: int = 0) -> str:
    try:
        out = subprocess.run(["nvidia-smi", f"--id={device}", "--query-gpu=name,driver_version",
                              "--format=csv,noheader"], capture_output=True, text=True, timeout=20).stdout.strip()
        return out or "unknown"
    except Exception:
        return "unknown"


def candidates() -> List[Dict[str, int]]:
    out = []
    for lt, gt, fuse in itertools.product((128, 256, 512), (64, 128), (2, 1)):
        out.append({"leaf_kernel": 1, "leaf_threads": lt, "gen_threads": gt, "leaf_fuse": fuse})
    out.append({"leaf_kernel": 2, "leaf_threads": 256, "gen_threads": 128, "leaf_fuse": 2})
    for lk in (4, 5):
        for gt in (64, 128):
            out.append({"leaf_kernel": lk, "leaf_threads": 256, "gen_threads": gt, "leaf_fuse": 2})
    for lt in (512, 1024):
        for gt in (64, 128):
            out.append({"leaf_kernel": 6, "leaf_threads": lt, "gen_threads": gt, "leaf_fuse": 2})
    return out


def measure(eng: pg.Engine, cfg: Dict[str, int], pos: pg.Pos, depth: int, reps: int = 3) -> float:
    eng.set_tuning(**cfg)
    eng.set_timing(True)
    eng.perft_position(pos, depth)  # warm
    ms = []
    for _ in range(reps):
        eng.perft_position(pos, depth)
        ms.append(eng.last_stats().device_ms)
    return statistics.median(ms)


def tune(eng: pg.Engine, pos: Optional[pg.Pos] = None, depth: int = 7, verbose: bool = False) -> Dict:
    pos = pos or pg.config_position(4, 1)
    results = []
    ref = None
    for cfg in candidates():
        n = None
        try:
            t = measure(eng, cfg, pos, depth)
            n = eng.last_stats().nodes
        except pg.PerftError:
            continue
        if ref is None:
            ref = n
        if n != ref:
            raise RuntimeError(f"autotune: configuration {cfg} changed the count ({n} != {ref})")
        results.append((t, cfg))
        if verbose:
            print(f"{t:9.3f} ms  {cfg}")
    results.sort(key=lambda x: x[0])
    best = results[0][1]
    eng.set_tuning(**best)
    return {"best": best, "ms": results[0][0], "depth": depth,
            "table": [{"ms": t, **c} for t, c in results]}


def load_or_tune(eng: pg.Engine, device: int = 0, retune: bool = False) -> Dict:
    # the candidate list is part of the key: a cache made with other
    # candidates is not reused
    tag = hashlib.sha1(json.dumps(candidates(), sort_keys=True).encode()).hexdigest()[:12]
    key = f"{gpu_key(device)}|{tag}"
    cache = {}
    if os.path.exists(CACHE):
        try:
            with open(CACHE) as f:
                cache = json.load(f)
        except Exception:
            cache = {}
    if not retune and key in cache:
        eng.set_tuning(**cache[key]["best"])
        return cache[key]
    res = tune(eng)
    cache[key] = res
    os.makedirs(CACHE_DIR, exist_ok=True)
    with open(CACHE, "w") as f:
        json.dump(cache, f, indent=1)
    return res


if __name__ == "__main__":
    e = pg.Engine(device=0, use_tt=False)
    r = tune(e, verbose=True)
    print(json.dumps({"gpu": gpu_key(), "best": r["best"], "ms": r["ms"]}))
