"""Benchmark: single-position GPU perft throughput (leaf nodes/s) on B200.

Workload: the position reached from the initial array by 4 uniformly random
legal plies (splitmix64 seed 1, moves sorted by UCI text), perft depth 7
without transposition tables.  One step = one whole perft(7) of that
position on the GPU: host-driven BFS levels (make+count, decoupled look-back
scan, shared-memory-staged generation) and the fused two-ply leaf kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Printed JSON line (rank 0):
  value    leaf nodes/s over all ranks, device time from CUDA events on the
           engine stream (first kernel to last kernel of each step)
  e2e      the same metric through the public C ABI call (pb_perft_position)
           with the root in host memory: host->device copy of the root and
           its moves and device->host read of the count inside the timed
           region (host wall clock around the synchronous call)
  roofline the leaf kernel against the integer-issue roofline
  cpu_baseline  the reference's own -cpu path (oracle/_ref) on this host's
           cores, one process per core over the root's children (perft 6
           each), plus a single-process figure and the CPU model
  reference_gpu  the reference's own GPU build (oracle/_ref, sm_100a) on the
           same position and depth, one GPU call (launch depth 7), timed by
           the reference program itself
  scheduler  (one GPU) the learned scheduler: trained on 2^20 positions,
           held-out prediction error per depth, and planned vs
           count-then-allocate vs plain seconds on held-out roots at depths 4..7;
           `gemm_roofline`: the network's tcgen05 GEMM against the measured
           dense BF16 peak
  positions  (one GPU) positions/s on 4096 uneven roots at perft 5: plain
           per-root calls, count-then-allocate batch, learned planner
  tt_run   (one GPU) perft 10 of the 2-ply seed-4 position with 150 GB of
           device tables: host drivers and replacement policies beside the
           reference's own table build
`config` is the same dict in both arms (--impl engine and reference).
With --gpus N > 1 (torchrun, one process per GPU) the depth-2 subtrees of the
root are bin-packed over the ranks by their perft(2) (strong scaling: total
work fixed); the only exchange is one all-gather of the per-rank counts.

The reference arm (--impl reference) runs only the reference program built
from its sources: it reads the children's FENs from tests/golden/
bench_subtrees.json and loads nothing of this repository's library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "leaf nodes/s"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "perft_gpu_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")
DEPTH = 7


def _bench_position():
    """(root FEN, its children's FENs) from the committed fixture."""
    with open(os.path.join(GOLDEN, "bench_subtrees.json")) as f:
        d = json.load(f)
    return d["root_fen"], d["children"]


def _reference_counts():
    """The reference's own per-depth counts of the bench position (1..7)."""
    path = os.path.join(GOLDEN, "ref_configs.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)["config2"]["counts"]


def bench_config(depth: int):
    """The workload description both arms print verbatim."""
    fen, _ = _bench_position()
    ref = _reference_counts()
    return {"workload": "single-position perft", "position": "4 random plies from the initial array, splitmix64 seed 1",
            "fen": fen, "depth": depth, "tt": False,
            "nodes": ref[depth - 1] if ref and depth <= len(ref) else None,
            "l2": "GPU arm: L2 flushed by a 256 MB write before each timed step",
            "parallelism": "one root; with N ranks its depth-2 subtrees bin-packed by perft(2)"}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# leaf kernel launched for each pb_tuning.leaf_kernel value
LEAF_KERNELS = {1: "k_leaf2", 2: "k_leaf2_coop", 3: "k_leaf2_defer", 4: "k_leaf2_sorted", 5: "k_leaf2_listed",
                6: "k_leaf2_balanced"}


def _load_profile_constants():
    path = os.path.join(ROOT, "profiles", "leaf_kernel_constants.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        # raw samples go to $BENCH_CLOCKS_DIR (default: the temp directory);
        # the JSON line carries their summary
        out_dir = os.environ.get("BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
            # nvidia-smi takes a moment to start: wait (at most 3 s) for its
            # first sample so the whole timed region is covered
            t0 = time.time()
            while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        med = statistics.median(sm) if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(torch, dev):
    buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    buf.fill_(1)
    del buf


def cpu_reference_sample(subtrees, sub_depth, max_seconds=20.0, procs=None):
    """The reference's -cpu -nott path on this host: `procs` processes kept
    busy over the subtrees in order (perft sub_depth of each); no subtree is
    started once the sample budget is spent, those started run to the end.
    Returns None when the reference is not built."""
    if not os.path.exists(REF_BIN):
        return None
    procs = procs or len(os.sched_getaffinity(0))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    t0 = time.perf_counter()

    def one(fen):
        if time.perf_counter() - t0 >= max_seconds:
            return None
        out = subprocess.run([REF_BIN, fen, str(sub_depth), "-cpu", "-nott"], capture_output=True, text=True,
                             env=env).stdout
        last = [l for l in out.splitlines() if l.startswith(f"Perft({sub_depth:02d})")]
        return int(last[0].split(":")[1].split(",")[0]) if last else None

    with ThreadPoolExecutor(max_workers=procs) as ex:
        res = list(ex.map(one, subtrees))
    wall = time.perf_counter() - t0
    done = [r for r in res if r is not None]
    nodes = sum(done)
    return {"value": nodes / wall if wall > 0 else 0.0, "unit": METRIC, "cores": procs, "kind": "reference",
            "sample": f"{len(done)} of the bench position's {len(subtrees)} children at perft {sub_depth} "
                      f"(reference -cpu -nott, one process per child, {procs} at a time, {wall:.1f} s wall)",
            "nodes": nodes, "seconds": wall}


def cpu_baseline(children, depth, all_core_s=15.0, single_s=8.0):
    """All host cores (one reference process per core) and one process."""
    allc = cpu_reference_sample(children, depth - 1, max_seconds=all_core_s)
    if allc is None:
        return None
    one = cpu_reference_sample(children, depth - 1, max_seconds=single_s, procs=1)
    out = {k: allc[k] for k in ("value", "unit", "cores", "kind", "sample")}
    out["single_thread"] = {"value": one["value"], "unit": METRIC, "sample": one["sample"]}
    out["cpu_model"] = cpu_model()
    out["host_threads"] = os.cpu_count()
    return out


def reference_gpu(fen, depth, reps=3):
    """The reference's own GPU build on the bench position: perft `depth`
    without tables at launch depth `depth` (one GPU call), the depth line's
    time as the reference program prints it.  Best of `reps` runs."""
    if not os.path.exists(REF_BIN):
        return None
    times, nodes = [], None
    for _ in range(reps):
        out = subprocess.run([REF_BIN, fen, str(depth), "-nott", "-ld", str(depth)], capture_output=True, text=True,
                             timeout=600).stdout
        line = [l for l in out.splitlines() if l.startswith(f"Perft({depth:02d})")]
        if not line:
            return {"unavailable": "reference GPU build printed no depth line"}
        nodes = int(line[0].split(":")[1].split(",")[0])
        times.append(float(line[0].split("time:")[1].split("seconds")[0]))
    best = min(times)
    return {"value": nodes / best, "unit": METRIC, "nodes": nodes, "seconds": times,
            "source": f"oracle/_ref/perft_gpu_ref <fen> {depth} -nott -ld {depth} (reference sources built for "
                      "sm_100a), the time it prints for the depth line, best of the runs"}


def _timed(fn, reps):
    """Best host wall time of `reps` calls after one warm-up call."""
    fn()
    best, out = None, None
    for _ in range(reps):
        t = time.perf_counter()
        out = fn()
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    return out, best


def scheduler_section(pg, eng, train_n=1 << 20, eval_n=16384, timed_n=1024):
    """The learned scheduler (config 4).  Training set: `train_n` playouts of
    0..60 plies (splitmix64 seed 3, positions with a legal move) labelled with
    exact perft 1..4 by batched GPU passes; the network (781 -> 256 -> 256 ->
    4, BF16 weights, FP32 accumulation, Adam) trained by the library's own
    kernels for 12 epochs.  Held out: `eval_n` playouts (seed 3003) with
    depths uniform in 4..7 (seed 3004): mean absolute error of the predicted
    log2(1 + perft(k)) per k against the exact labels (and of a constant guess,
    the training mean), then the first `timed_n` of them counted three ways
    through the public API: one plain call per root, count-then-allocate
    batches, and the planned batches (predicted level sizes, bin-packing, one
    captured graph per batch).  All three must agree."""
    import numpy as np
    from perft_gpu_2026_b200 import scheduler

    t0 = time.perf_counter()
    pos, y, _ = scheduler.make_training_set(eng, train_n)
    t_label = time.perf_counter() - t0
    eng.mlp_init(seed=1, out_bias=list(y.mean(0)))
    t1 = time.perf_counter()
    loss = eng.mlp_train(pos, y, epochs=12, batch=4096, lr=2e-3)
    t_train = time.perf_counter() - t1
    held = scheduler.keep_movable(pg.random_playouts(3003, eval_n + eval_n // 8, 0, 60))[:eval_n]
    depths = scheduler.eval_depths(len(held))
    truth = np.log2(1.0 + scheduler.label(eng, held))
    pred = eng.mlp_predict(held)
    mae = np.abs(pred - truth).mean(0).tolist()
    mae_const = np.abs(y.mean(0)[None, :] - truth).mean(0).tolist()
    sub, dsub = held[:timed_n], depths[:timed_n]
    t = time.perf_counter()
    plain = [eng.perft_position(p, d) for p, d in zip(sub, dsub)]
    t_plain = time.perf_counter() - t
    t = time.perf_counter()
    batched = eng.perft_batch(sub, dsub)
    t_batched = time.perf_counter() - t
    t = time.perf_counter()
    planned, st = eng.perft_batch_planned(sub, dsub)
    t_planned = time.perf_counter() - t
    assert plain == batched == list(planned), "scheduler evaluation: counts differ between modes"
    return {"workload": f"{len(pos)} training positions (0..60-ply playouts, seed 3), {len(held)} held-out "
                        f"(seed 3003) at depths U[4,7] (seed 3004), the first {len(sub)} timed",
            "label_s": t_label, "train_s": t_train, "train_mse": loss,
            "mae_log2_perft1_4": mae, "mae_log2_perft1_4_constant_guess": mae_const,
            "timed": {"roots": len(sub), "nodes": int(sum(plain)), "plain_s": t_plain, "batched_s": t_batched,
                      "learned_s": t_planned, "learned_vs_batched": t_batched / t_planned,
                      "learned_vs_plain": t_plain / t_planned,
                      "plan": {"batches": st.batches, "graph_batches": st.graph_batches, "retries": st.retries,
                               "split_roots": st.split_roots},
                      "timing": "host wall clock around the public call, one run each"}}


def gemm_section(eng, reps=50):
    """The scheduler network's tcgen05 GEMM against the measured dense BF16
    peak (burst figure: each product is timed alone): layer 2's forward
    product at a 4096-sample batch, its weight gradient (K split over 16
    CTAs per tile), and a large product that the network does not need, for
    the kernel's ceiling.  CUDA events around `reps` launches after one
    checked launch; the check compares 64 rows of C with a float64 product
    of the same BF16 values."""
    import numpy as np

    peaks, kind = _peaks()
    peak = peaks.get("bf16_tflops", 1590.0)
    rng = np.random.default_rng(7)
    out = {"unit": "TFLOP/s", "peak": peak, "peak_source": f"bf16_tflops ({kind})",
           "timing": f"CUDA events, mean of {reps} launches after one checked launch"}
    shapes = (("layer2_forward", 4096, 256, 256, False, False),
              ("layer2_weight_gradient", 256, 256, 4096, True, False),
              ("large_8192x2048x2048", 8192, 2048, 2048, False, False))
    for name, m, n, k, ta, tb in shapes:
        a = rng.uniform(-1, 1, size=m * k).astype(np.float32)
        b = rng.uniform(-1, 1, size=k * n).astype(np.float32)
        ab = ((a.view(np.uint32) + 0x8000) >> 16).astype(np.uint16)
        bb = ((b.view(np.uint32) + 0x8000) >> 16).astype(np.uint16)
        c, ms = eng.selftest_gemm(ab, bb, ta, tb, m, n, k, reps=reps)
        av = (ab.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
        bv = (bb.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
        am = av.reshape(k, m).T if ta else av.reshape(m, k)
        bm = bv.reshape(n, k).T if tb else bv.reshape(k, n)
        rows = rng.choice(m, size=min(64, m), replace=False)
        err = float(np.abs(c[rows] - am[rows] @ bm).max())
        assert err <= 1e-5 * k + 1e-4, (name, err)
        tf = 2.0 * m * n * k / (ms * 1e-3) / 1e12
        out[name] = {"m": m, "n": n, "k": k, "ms": ms, "achieved": tf, "frac": tf / peak, "max_abs_err": err}
    return out


def positions_section(pg, eng, reps):
    """Positions/s on 4096 uneven roots (playouts of 6..40 plies, splitmix64
    seed 2), perft 5 each, three ways through the public API (roots in host
    memory, counts read back, host wall clock): one plain call per root, one
    count-then-allocate batched call, and the learned planner (the network
    scheduler_section trained).  The roots are held as one packed pb_pos array
    (pack_positions, the C ABI's batch format) by every mode.  Also the planner
    at perft 3 and 4 of the same roots, where each batch's per-level host round
    trips are a larger share.  All modes must agree."""
    import numpy as np
    from perft_gpu_2026_b200 import scheduler

    roots = pg.pack_positions(pg.uneven_roots(4096, 6, 40, seed=2))
    depths = [5] * len(roots)
    truth = np.log2(1.0 + scheduler.label(eng, roots))
    mae = np.abs(eng.mlp_predict(roots) - truth).mean(0).tolist()
    plain, t_plain = _timed(lambda: [eng.perft_position(r, 5) for r in roots], reps)
    batched, t_batched = _timed(lambda: eng.perft_batch(roots, depths), reps)
    (learned, plan), t_learned = _timed(lambda: eng.perft_batch_planned(roots, depths), reps)
    assert plain == batched == list(learned), "batched or planned counts differ from the plain path"
    n = len(roots)
    shallow = {}
    for d in (3, 4):
        b, tb = _timed(lambda: eng.perft_batch(roots, d), 5)
        (l, _), tl = _timed(lambda: eng.perft_batch_planned(roots, d), 5)
        assert b == list(l)
        shallow[f"perft{d}"] = {"batched": n / tb, "learned": n / tl, "learned_vs_batched": tb / tl}
    return {"workload": "4096 uneven roots (6..40-ply playouts, seed 2), perft 5 each, no TT",
            "unit": "positions/s", "timing": "host wall clock around the public call, roots in one packed "
                                             f"pb_pos array, best of {reps} after one warm-up",
            "nodes": int(sum(plain)), "plain": n / t_plain, "batched": n / t_batched, "learned": n / t_learned,
            "learned_vs_plain": t_plain / t_learned, "batched_vs_plain": t_plain / t_batched,
            "learned_vs_batched": t_batched / t_learned,
            "plan": {"batches": plan.batches, "graph_batches": plan.graph_batches, "retries": plan.retries,
                     "split_roots": plan.split_roots},
            "mae_log2_perft1_4_on_roots": mae, "shallow_depths": shallow}


def tt_section(pg, depth=10, dtt_mb=150000, htt_mb=16384, bf_launch_depth=8):
    """The deep table run (config 5): the position 2 random plies from the
    initial array (splitmix64 seed 4), perft 1..depth through pb_perft (the
    command line's loop) with `dtt_mb` MB of device tables and `htt_mb` MB of
    host tables.  Seconds of the last depth for: the depth-first host driver
    with the reference's always-overwrite replacement; two-slot size-priority
    buckets; the breadth-first host driver with batched table-mode calls; and
    the reference's own table build (oracle/_ref) with the same flags, as it
    prints them.  Every count must agree."""
    fen = pg.to_fen(pg.config_position(2, 4))
    runs = {"depth_first_overwrite": {}, "depth_first_size_priority": {"tt_replace": 2},
            f"breadth_first_ld{bf_launch_depth}_overwrite": {"host_driver": 2}}
    out = {"workload": f"2 random plies (seed 4), perft {depth}, -dtt {dtt_mb} -htt {htt_mb}", "fen": fen,
           "unit": "seconds of the last depth (host wall clock inside pb_perft)"}
    counts = set()
    for name, tun in runs.items():
        ld = bf_launch_depth if tun.get("host_driver") == 2 else 0
        eng = pg.Engine(device=0, use_tt=True, device_tt_mb=dtt_mb, host_tt_mb=htt_mb, launch_depth=ld)
        if tun:
            eng.set_tuning(**tun)
        res = eng.perft(fen, depth)
        eng.close()
        counts.add(res[-1][0])
        out[name] = {"seconds": res[-1][1], "seconds_all_depths": sum(s for _, s in res), "nodes": res[-1][0]}
    if os.path.exists(REF_BIN):
        txt = subprocess.run([REF_BIN, fen, str(depth), "-dtt", str(dtt_mb), "-htt", str(htt_mb)],
                             capture_output=True, text=True, timeout=1200).stdout
        lines = [l for l in txt.splitlines() if l.startswith("Perft(")]
        if lines:
            last = lines[-1]
            n = int(last.split(":")[1].split(",")[0])
            counts.add(n)
            out["reference_tables"] = {"seconds": float(last.split("time:")[1].split("seconds")[0]), "nodes": n,
                                       "seconds_all_depths": sum(float(l.split("time:")[1].split("seconds")[0])
                                                                 for l in lines)}
    assert len(counts) == 1, f"table runs disagree: {counts}"
    return out


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/perft_gpu_ref not built"}))
        return 0
    _, subs = _bench_position()
    vals, last = [], None
    # each step is a bounded sample; the whole run stays near two minutes
    per_step = max(1.0, min(8.0, 120.0 / (args.warmup + args.steps)))
    for i in range(args.warmup + args.steps):
        r = cpu_reference_sample(subs, args.depth - 1, max_seconds=per_step)
        if i >= args.warmup:
            vals.append(r["value"])
            last = r
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": last["seconds"] * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": bench_config(args.depth),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": last["cores"], "kind": "reference",
                             "sample": last["sample"], "cpu_model": cpu_model(), "host_threads": os.cpu_count()},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--depth", type=int, default=DEPTH)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--leaf-kernel", type=int, default=0, help="1 = edge per thread, 2 = cooperative (0 = engine default)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the engine's default launch parameters")
    ap.add_argument("--no-positions", action="store_true", help="skip the batched-roots positions/s section")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip timing the reference's GPU build")
    ap.add_argument("--no-tt", action="store_true", help="skip the deep table run (150 GB of device tables)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import perft_gpu_2026_b200 as pg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    root_fen, child_fens = _bench_position()
    root = pg.parse_fen(root_fen)
    depth = args.depth
    eng = pg.Engine(device=local, use_tt=False)
    tuning = None
    if args.leaf_kernel:
        eng.set_tuning(leaf_kernel=args.leaf_kernel)
    elif not args.no_autotune:
        from perft_gpu_2026_b200 import autotune

        # rank 0 tunes (or reads the cache); the others read what it wrote
        if rank == 0:
            tuning = autotune.load_or_tune(eng, local)["best"]
        if dist:
            dist.barrier()
        if rank != 0:
            tuning = autotune.load_or_tune(eng, local)["best"]
    eng.set_timing(True)

    # shard: depth-2 subtrees bin-packed over ranks by their perft(2), an exact
    # size estimate every rank computes identically (one rank: the whole root)
    from perft_gpu_2026_b200 import dist as pdist

    if world > 1:
        plan = pdist.ShardedPerft(root, depth, world, rank, lambda ps, d: eng.perft_batch(ps, [d] * len(ps)))
        run_once = plan.run
    else:
        def run_once():
            return eng.perft_position(root, depth)

    def step():
        total = run_once()
        st = eng.last_stats()
        return total, st.device_ms, st.leaf_ms, st.leaf_positions, st.kernels, st.h2d_bytes, st.d2h_bytes

    for _ in range(args.warmup):
        step()
    # timed region: device time from the engine's CUDA events per step
    results = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush_l2(torch, dev)
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            results.append(step())
            torch.cuda.synchronize()
    clocks = clk.summary()
    nodes = results[0][0]
    assert all(r[0] == nodes for r in results), "perft result changed between steps"
    dev_ms = [r[1] for r in results]
    leaf_ms = [r[2] for r in results]
    my_ms = sum(dev_ms) / len(dev_ms)
    my_leaf_ms = sum(leaf_ms) / len(leaf_ms)

    # e2e: the public C-ABI call with the root in host memory, wall clock
    e2e_ms = []
    for _ in range(args.steps):
        flush_l2(torch, dev)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        run_once()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    my_e2e = statistics.median(e2e_ms)

    if dist:
        t = torch.tensor([my_ms, my_e2e, my_leaf_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        my_ms, my_e2e, my_leaf_ms = t.tolist()
        nodes = pdist.all_reduce_count(nodes, device=dev)
    config = bench_config(depth)
    if config["nodes"] is not None and nodes != config["nodes"]:
        raise SystemExit(f"count {nodes} differs from the reference's {config['nodes']}")
    if rank == 0:
        peaks, peak_kind = _peaks()
        kernel = LEAF_KERNELS.get(eng.get_tuning().leaf_kernel, "k_leaf2")
        consts = _load_profile_constants().get(kernel, {})
        leaf_pos = results[0][3]
        kernels = results[0][4]
        sm_mhz = peaks.get("sm_max_mhz", 1965.0)
        issue_peak = 148 * 4 * sm_mhz * 1e6 / 1e9  # G warp-instructions / s
        inst_per_pos = consts.get("warp_inst_per_position")
        dram_per_pos = consts.get("dram_bytes_per_position")
        roofline = {"bound": "int_issue", "unit": "Gwarp-inst/s", "peak": issue_peak,
                    "peak_source": f"148 SMs x 4 warp-inst issue/clk x sm_max_mhz ({peak_kind})",
                    "kernel": kernel, "leaf_ms": my_leaf_ms, "positions_per_launch": leaf_pos,
                    "positions_per_s": leaf_pos / (my_leaf_ms / 1e3) if my_leaf_ms > 0 else None,
                    "achieved": None, "frac": None,
                    "traffic": dram_per_pos * leaf_pos if dram_per_pos else None,
                    "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum per move-count call, "
                                    "from the ncu capture of this kernel's depth-7 launch of this position "
                                    "(profiles/), times this launch's calls",
                    "algorithmic_bytes": consts.get("algorithmic_bytes_per_launch"),
                    "algorithmic_note": "the leaf's compulsory DRAM reads: 6 B per edge (move, parent index) "
                                        "and 33 B per parent position; the leaf is bound by integer issue, "
                                        "not by these bytes"}
        if inst_per_pos:
            ach = inst_per_pos * leaf_pos / (my_leaf_ms / 1e3) / 1e9
            roofline["achieved"] = ach
            roofline["frac"] = ach / issue_peak
            roofline["inst_per_position"] = inst_per_pos
        if consts.get("ncu_alu_pipe_pct"):
            # the binding unit: the integer ALU pipe runs at half the issue
            # rate, so the issue fraction cannot reach 1 with this mix
            roofline["binding_unit"] = {"unit": "ALU pipe", "util_pct": consts["ncu_alu_pipe_pct"],
                                        "issue_active_pct": consts.get("ncu_issue_active_pct"),
                                        "source": consts.get("pipe_source",
                                                             "ncu --set full capture of the same kernel (profiles/)")}
        line = {"metric": METRIC, "value": nodes / (my_ms / 1e3), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": my_ms, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
                "config": config, "tuning": eng.get_tuning().as_dict(),
                "count_check": "equal to the reference program's count of this position and depth"
                               if config["nodes"] is not None else "no reference count for this depth",
                "e2e": {"value": nodes / (my_e2e / 1e3), "unit": METRIC, "ms_per_step": my_e2e,
                        "h2d_bytes_per_step": int(results[0][5]), "d2h_bytes_per_step": int(results[0][6]),
                        "timing": "host wall clock around pb_perft_position"},
                "gpu_launches": int(kernels), "clocks": clocks, "roofline": roofline}
        if world == 1 and not args.no_positions:
            line["scheduler"] = scheduler_section(pg, eng)
            line["scheduler"]["gemm_roofline"] = gemm_section(eng)
            line["positions"] = positions_section(pg, eng, reps=min(args.steps, 3))
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(child_fens, depth)
            if cb:
                line["cpu_baseline"] = cb
    eng.close()
    if rank == 0 and world == 1 and not args.no_tt:
        # after the engine released its memory: the tables take 150 GB
        line["tt_run"] = tt_section(pg)
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        # after the engine released its memory; the reference allocates its own
        rg = reference_gpu(root_fen, depth)
        if rg:
            line["reference_gpu"] = rg
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
