"""Differential runs against the reference's own GPU build (oracle/_ref,
compiled from the reference sources by oracle/Makefile): the same FEN and
depth through both command lines, per-depth counts compared, without and with
transposition tables."""
import os
import subprocess

import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "perft_gpu_ref")
CLI = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")


def _counts(binary, fen, depth, flags):
    out = subprocess.run([binary, fen, str(depth)] + flags, capture_output=True, text=True, timeout=300,
                         check=True).stdout
    return [int(l.split(":")[1].split(",")[0]) for l in out.splitlines() if l.startswith("Perft(")]


def _fens(seed, n):
    ps = [p for p in pg.random_playouts(seed, 2 * n, 4, 40) if pg.count_moves(p, True) > 0]
    return [pg.to_fen(p) for p in ps[:n]]


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build absent (make -C oracle ref)")
def test_cli_matches_reference_gpu_build_without_tables():
    for fen in _fens(4242, 8):
        want = _counts(REF, fen, 6, ["-nott"])
        got = _counts(CLI, fen, 6, ["-nott"])
        assert len(want) == 6 and got == want, fen


@pytest.mark.skipif(not os.path.exists(REF), reason="reference build absent (make -C oracle ref)")
def test_cli_matches_reference_gpu_build_with_tables():
    for fen in _fens(4343, 4):
        want = _counts(REF, fen, 7, ["-dtt", "2000", "-htt", "512"])
        got = _counts(CLI, fen, 7, ["-dtt", "2000", "-htt", "512"])
        assert len(want) == 7 and got == want, fen
