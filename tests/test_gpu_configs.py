"""Every benchmark workload pinned to the reference program's own output.

Counts come from tests/golden/ref_configs.json (the reference's -cpu -nott
path, written by tests/golden/make_config_golden.py) and, where the reference's
GPU build (oracle/_ref, compiled from the reference sources) is present, from
running it on this GPU beside the engine's command line:

  config 1  8 random plies (seed 0), perft 1..5: engine vs fixture
  config 2  4 random plies (seed 1), perft 1..7 (the benchmark depth): engine
            vs fixture, and the command line vs the reference GPU build at
            launch depth 7 (one GPU call), every depth's line
  config 3  the 4096 uneven roots at perft 5: plain per-root calls, the
            count-then-allocate batch, the planned batch and the command
            line's -batch file mode, each root vs fixture
  config 4  256 rows of the scheduler's training labels (perft 1..4)
  config 5  2 random plies (seed 4), perft 9 with 150 GB of device tables and
            16 GB of host tables: equal to the run without tables and to the
            reference's own table build, every depth's line
"""
import hashlib
import json
import os
import subprocess

import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "perft_gpu_ref")
CLI = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")
needs_ref = pytest.mark.skipif(not os.path.exists(REF), reason="reference build absent (make -C oracle ref)")


@pytest.fixture(scope="module")
def fixture():
    with open(os.path.join(ROOT, "tests", "golden", "ref_configs.json")) as f:
        return json.load(f)


def _lines(binary, args, timeout=900):
    out = subprocess.run([binary] + args, capture_output=True, text=True, timeout=timeout, check=True).stdout
    return [int(l.split(":")[1].split(",")[0]) for l in out.splitlines() if l.startswith("Perft(")]


def test_config1_matches_reference(gpu_engine, fixture):
    c = fixture["config1"]
    p = pg.config_position(8, 0)
    assert pg.to_fen(p) == c["fen"]
    assert [gpu_engine.perft_position(p, d) for d in range(1, 6)] == c["counts"]


def test_config2_at_benchmark_depth_matches_reference(gpu_engine, fixture):
    c = fixture["config2"]
    p = pg.config_position(4, 1)
    assert pg.to_fen(p) == c["fen"]
    assert [gpu_engine.perft_position(p, d) for d in range(1, 8)] == c["counts"]


@needs_ref
def test_config2_command_line_matches_reference_gpu_build(fixture):
    """Launch depth 7: depth 7 is one GPU call in both programs (BFS levels
    then the fused two-ply leaf), compared line by line."""
    c = fixture["config2"]
    args = [c["fen"], "7", "-nott", "-ld", "7"]
    want = _lines(REF, args)
    got = _lines(CLI, args)
    assert want == c["counts"]
    assert got == want


def test_config3_every_root_every_path_matches_reference(fixture):
    c = fixture["config3"]
    roots = pg.uneven_roots(4096, 6, 40, seed=2)
    fens = [pg.to_fen(p) for p in roots]
    assert hashlib.sha256("\n".join(fens).encode()).hexdigest() == c["fen_sha256"]
    want = c["perft5"]
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=8 << 30)
    try:
        assert eng.perft_batch(roots, [5] * len(roots)) == want
        assert [eng.perft_position(p, 5) for p in roots] == want
        # the planner with an untrained network (a constant guess): wrong
        # sizes may force exact reruns, never a wrong count
        eng.mlp_init(seed=3, out_bias=[4.5, 9.5, 14.5, 19.0])
        planned, _ = eng.perft_batch_planned(roots, [5] * len(roots))
        assert list(planned) == want
    finally:
        eng.close()
    assert sum(want) == c["total"]


def test_config3_batch_file_on_the_gpu(tmp_path, fixture):
    """The command line's -batch mode on the GPU (pb_perft_batch per depth):
    an EPD file of the 4096 roots with ;D5 expectations from the reference."""
    c = fixture["config3"]
    roots = pg.uneven_roots(4096, 6, 40, seed=2)
    f = tmp_path / "config3.epd"
    f.write_text("".join(f"{pg.to_fen(p)} ;D5 {n}\n" for p, n in zip(roots, c["perft5"])))
    out = subprocess.run([CLI, "-batch", str(f), "-json"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr
    assert "4096 positions, 0 mismatches" in out.stdout
    js = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert js[-1]["depth"] == 5 and int(js[-1]["nodes"]) == c["total"]


def test_config4_training_labels_match_reference(fixture):
    from perft_gpu_2026_b200 import scheduler

    c = fixture["config4"]
    train = scheduler.keep_movable(pg.random_playouts(3, 1 << 20, 0, 60))
    assert len(train) == c["train_n"]
    rows = [train[i] for i in c["rows"]]
    assert [pg.to_fen(p) for p in rows] == c["fens"]
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    try:
        labels = scheduler.label(eng, rows)
    finally:
        eng.close()
    assert labels.astype("int64").tolist() == c["perft1_4"]


def test_config5_tables_equal_no_tables_and_reference(fixture):
    """150 GB of device tables (with full-key verification) and 16 GB of host
    tables: every depth equals the run without tables, the reference's -cpu
    counts at the shallow depths, and the reference's own table build."""
    c = fixture["config5"]
    p = pg.config_position(2, 4)
    assert pg.to_fen(p) == c["fen"]
    tt = _lines(CLI, [c["fen"], "9", "-dtt", "150000", "-htt", "16384"])
    nott = _lines(CLI, [c["fen"], "9", "-nott"])
    assert tt == nott
    # the breadth-first host driver with batched table-mode GPU calls
    assert _lines(CLI, [c["fen"], "9", "-dtt", "150000", "-htt", "16384", "-hd", "2", "-ld", "6"]) == tt
    assert tt[:len(c["counts"])] == c["counts"]
    if os.path.exists(REF):
        assert _lines(REF, [c["fen"], "9", "-dtt", "150000", "-htt", "16384"]) == tt
