"""Pins the CPU oracle to the reference program's own output.

The fixtures in tests/golden/ref_cpu_perft.json were produced by running the
reference's `-cpu -nott` path (built from its sources, tests/golden/
make_golden.py).  The oracle must reproduce every per-depth count, including
the two reference counting conventions (double capture-promotion onto one
square, double en-passant evasion)."""
import pytest


def test_oracle_matches_reference_fixtures(oracle, golden):
    bad = []
    for case in golden:
        for d, want in enumerate(case["counts"], start=1):
            if want > 30_000_000:
                continue  # keeps the CPU suite short; covered on the GPU
            got = oracle.perft(case["fen"], d)
            if got != want:
                bad.append((case["name"], d, got, want))
    assert not bad, bad


def test_oracle_known_counts(oracle):
    # initial array perft 1..5 (the reference prints these for the default run)
    fen = "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1"
    assert [oracle.perft(fen, d) for d in range(1, 6)] == [20, 400, 8902, 197281, 4865609]


def test_oracle_strict_differs_only_on_merged_moves(oracle):
    # two pawns promoting by capture onto c8: the reference counts 17, exact is 21
    fen = "2n4k/1P1P4/8/8/8/8/8/4K3 w - - 0 1"
    assert oracle.count(fen) == 17
    assert oracle.count(fen, strict=True) == 21
    assert len(oracle.moves(fen)) == 21
    # two pawns taking the checking pawn en passant: reference 8, exact 9
    fen = "k7/8/8/3PpP2/5K2/8/8/8 w - e6 0 1"
    assert oracle.count(fen) == 8
    assert oracle.count(fen, strict=True) == 9
    assert len(oracle.moves(fen)) == 9


def test_oracle_strict_count_equals_generation(oracle, golden):
    for case in golden:
        assert oracle.count(case["fen"], strict=True) == len(oracle.moves(case["fen"])), case["name"]


def test_oracle_matches_reference_on_benchmark_workloads(oracle):
    """tests/golden/ref_configs.json holds the reference's counts on the
    benchmark workloads; the oracle reproduces the ones it finishes in
    seconds (configs 1, 2 and 5 to perft 5; config 4's label rows to perft
    3).  The full depths are compared on the GPU."""
    import json
    import os

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_configs.json")
    with open(path) as f:
        cfg = json.load(f)
    for name in ("config1", "config2", "config5"):
        c = cfg[name]
        assert [oracle.perft(c["fen"], d) for d in range(1, 6)] == c["counts"][:5], name
    c = cfg["config4"]
    for fen, want in zip(c["fens"], c["perft1_4"]):
        assert [oracle.perft(fen, d) for d in (1, 2, 3)] == want[:3], fen
