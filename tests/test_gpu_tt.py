"""Transposition-table mode on the GPU: counts with the device and host
tables must equal the no-TT counts (the reference's -nott ground truth) on the
same positions, including when the tables are tiny and constantly overwritten."""
import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu

START = pg.START_FEN
KIWIPETE = "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -"


@pytest.fixture(scope="module")
def tt_engine():
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=4 << 30, device_tt_mb=4096, host_tt_mb=512)
    yield eng
    eng.close()


def test_tt_position_matches_known(tt_engine):
    p = pg.parse_fen(START)
    assert [tt_engine.perft_position(p, d) for d in range(1, 8)] == [
        20, 400, 8902, 197281, 4865609, 119060324, 3195901860]
    # repeat: now served largely from the tables
    assert tt_engine.perft_position(p, 7) == 3195901860


def test_tt_kiwipete_and_bench_position(tt_engine):
    ref = pg.Engine(device=0, use_tt=False, arena_bytes=4 << 30)
    for p, d in [(pg.parse_fen(KIWIPETE), 6), (pg.config_position(4, 1), 7), (pg.config_position(8, 0), 6)]:
        assert tt_engine.perft_position(p, d) == ref.perft_position(p, d)
    ref.close()


def test_tt_matches_fixtures(tt_engine, golden):
    bad = []
    for case in golden:
        p = pg.parse_fen(case["fen"])
        for d, want in enumerate(case["counts"], start=1):
            got = tt_engine.perft_position(p, d)
            if got != want:
                bad.append((case["name"], d, got, want))
    assert not bad, bad


def test_tt_launch_with_host_tables():
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=2 << 30, device_tt_mb=2048, host_tt_mb=256, launch_depth=5)
    res = eng.perft(START, 8)
    assert [r for r, _ in res] == [20, 400, 8902, 197281, 4865609, 119060324, 3195901860, 84998978956]
    eng.close()


def test_tiny_tables_stay_exact():
    # 1 MB budget: the shallow tables cannot be built and the deep ones hold
    # a few hundred slots, so nearly every store overwrites another key
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=1 << 30, device_tt_mb=1, host_tt_mb=1)
    ref = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30)
    for seed in range(6):
        p = pg.config_position(6 + seed, 100 + seed)
        assert eng.perft_position(p, 6) == ref.perft_position(p, 6)
    eng.close()
    ref.close()


def test_tt_strict_mode(oracle):
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=1 << 30, device_tt_mb=1024, strict=True)
    fen = "2n4k/1P1P4/8/8/8/8/8/4K3 w - - 0 1"
    p = pg.parse_fen(fen)
    assert [eng.perft_position(p, d) for d in (3, 4, 5)] == [oracle.perft(fen, d, True) for d in (3, 4, 5)]
    eng.close()


def test_size_priority_buckets_stay_exact():
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=2 << 30, device_tt_mb=2048, host_tt_mb=256)
    eng.set_tuning(tt_replace=2)
    p = pg.parse_fen(START)
    assert [eng.perft_position(p, d) for d in (5, 6, 7)] == [4865609, 119060324, 3195901860]
    ref = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    for q, d in [(pg.parse_fen(KIWIPETE), 6), (pg.config_position(4, 1), 7)]:
        assert eng.perft_position(q, d) == ref.perft_position(q, d)
    ref.close()
    small = pg.Engine(device=0, use_tt=True, arena_bytes=1 << 30, device_tt_mb=1, host_tt_mb=1)
    small.set_tuning(tt_replace=2)
    assert small.perft_position(pg.parse_fen(KIWIPETE), 5) == 193690690
    small.close()
    eng.close()


@pytest.mark.parametrize("use_tt", [True, False])
def test_breadth_first_host_driver_on_the_gpu(use_tt):
    """host_driver 2: the tree above the launch depth expanded ply by ply,
    transpositions merged by key with tables, the launch-depth positions in
    batched GPU calls (table mode: duplicates merged across the batch's
    subtrees too).  Equal to the depth-first driver and the known totals,
    also with an arena so small that batches must be halved."""
    for arena, ld in ((2 << 30, 5), (96 << 20, 4)):
        eng = pg.Engine(device=0, use_tt=use_tt, arena_bytes=arena, device_tt_mb=1024, host_tt_mb=256,
                        launch_depth=ld)
        eng.set_tuning(host_driver=2)
        res = eng.perft(START, 8)
        assert [r for r, _ in res] == [20, 400, 8902, 197281, 4865609, 119060324, 3195901860, 84998978956]
        got, _ = eng.perft_launch(pg.parse_fen(KIWIPETE), 6)
        assert got == 8031647685
        eng.close()
    eng = pg.Engine(device=0, use_tt=use_tt, arena_bytes=2 << 30, device_tt_mb=1024, host_tt_mb=256, launch_depth=4)
    eng.set_tuning(host_driver=2)
    ref = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    for seed in range(4):
        p = pg.config_position(10 + 3 * seed, 500 + seed)
        got, _ = eng.perft_launch(p, 7)
        assert got == ref.perft_position(p, 7)
    ref.close()
    eng.close()


@pytest.mark.parametrize("leaf_kernel", [1, 5])
def test_table_leaf_modes_match_fixtures(golden, leaf_kernel):
    """The table leaf unranked (leaf kernel 1) and ranked with listed pieces
    (5) against the reference fixtures and the bench position."""
    eng = pg.Engine(device=0, use_tt=True, arena_bytes=2 << 30, device_tt_mb=1024, host_tt_mb=256)
    eng.set_tuning(leaf_kernel=leaf_kernel)
    bad = []
    for case in golden:
        p = pg.parse_fen(case["fen"])
        for d, want in enumerate(case["counts"], start=1):
            got = eng.perft_position(p, d)
            if got != want:
                bad.append((case["name"], d, got, want))
    assert not bad, bad
    assert eng.perft_position(pg.config_position(4, 1), 7) == 26402736244
    eng.close()


@pytest.mark.parametrize("leaf_kernel", [4, 5])
def test_persistent_table_leaf_stays_exact(golden, leaf_kernel):
    """tt_leaf 2: CTAs queue their table misses in shared memory and count
    only full CTAs of misses.  Against the fixtures, the bench position at
    perft 7 and the README totals, with tables large (many hits) and tiny
    (nearly all misses, constant overwrites)."""
    for dtt in (2048, 1):
        eng = pg.Engine(device=0, use_tt=True, arena_bytes=2 << 30, device_tt_mb=dtt, host_tt_mb=256)
        eng.set_tuning(leaf_kernel=leaf_kernel, tt_leaf=2)
        bad = []
        for case in golden:
            p = pg.parse_fen(case["fen"])
            for d, want in enumerate(case["counts"], start=1):
                got = eng.perft_position(p, d)
                if got != want:
                    bad.append((case["name"], d, got, want))
        assert not bad, (dtt, bad)
        assert eng.perft_position(pg.config_position(4, 1), 7) == 26402736244
        assert eng.perft_position(pg.parse_fen(START), 8) == 84998978956
        eng.close()
