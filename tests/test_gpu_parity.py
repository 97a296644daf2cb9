"""GPU parity: the CUDA path through the C ABI against the oracle, the
reference-generated fixtures and the reference README's known totals."""
import os
import subprocess

import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu

START = pg.START_FEN
KIWIPETE = "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -"  # README.md:32


def test_scan_matches_torch(gpu_engine):
    import torch

    g = torch.Generator().manual_seed(0)
    for n in (1, 31, 2047, 2048, 2049, 100_003, 5_000_000):
        x = torch.randint(0, 219, (n,), generator=g, dtype=torch.int64)
        d_in = x.to(torch.int32).cuda()
        d_out = torch.empty(n, dtype=torch.int64, device="cuda")
        d_tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        gpu_engine.dev_scan(d_in.data_ptr(), n, d_out.data_ptr(), d_tot.data_ptr())
        torch.cuda.synchronize()
        excl = torch.cumsum(x, 0) - x
        assert torch.equal(d_out.cpu(), excl), n
        assert int(d_tot.item()) == int(x.sum()), n


def test_scan_unaligned_and_many_tiles(gpu_engine):
    """Arrays not on a 32-byte boundary take the scalar path; 40 M counts
    (19,532 tiles) exercise long look-back chains."""
    import torch

    g = torch.Generator().manual_seed(1)
    for n, shift in ((2049, 1), (1_000_001, 3), (40_000_000, 0)):
        x = torch.randint(0, 219, (n,), generator=g, dtype=torch.int64)
        buf_in = torch.empty(n + shift, dtype=torch.int32, device="cuda")
        buf_out = torch.empty(n + shift, dtype=torch.int64, device="cuda")
        d_in, d_out = buf_in[shift:], buf_out[shift:]
        d_in.copy_(x.to(torch.int32))
        d_tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        gpu_engine.dev_scan(d_in.data_ptr(), n, d_out.data_ptr(), d_tot.data_ptr())
        torch.cuda.synchronize()
        excl = torch.cumsum(x, 0) - x
        assert torch.equal(d_out.cpu(), excl), (n, shift)
        assert int(d_tot.item()) == int(x.sum()), (n, shift)


@pytest.mark.parametrize("leaf_kernel", [1, 2, 4, 5, 6])
def test_gpu_matches_reference_fixtures(gpu_engine, golden, leaf_kernel):
    prev = gpu_engine.get_tuning().leaf_kernel
    gpu_engine.set_tuning(leaf_kernel=leaf_kernel)
    bad = []
    for case in golden:
        p = pg.parse_fen(case["fen"])
        for d, want in enumerate(case["counts"], start=1):
            got = gpu_engine.perft_position(p, d)
            if got != want:
                bad.append((case["name"], d, got, want))
    gpu_engine.set_tuning(leaf_kernel=prev)
    assert not bad, bad


@pytest.mark.parametrize("strict", [False, True])
def test_gpu_matches_oracle_on_playouts(oracle, strict):
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30, strict=strict)
    for seed in range(40):
        p, _, _ = pg.random_playout(50_000 + seed, 6 + (seed * 17) % 60)
        if pg.count_moves(p, True) == 0:
            continue
        fen = pg.to_fen(p)
        for d in (3, 4):
            assert eng.perft_position(p, d) == oracle.perft(fen, d, strict), (fen, d)
    eng.close()


def test_strict_mode_counts_merged_moves(oracle):
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30, strict=True)
    fen = "2n4k/1P1P4/8/8/8/8/8/4K3 w - - 0 1"
    p = pg.parse_fen(fen)
    assert eng.perft_position(p, 1) == 21
    assert [eng.perft_position(p, d) for d in (2, 3, 4, 5)] == [oracle.perft(fen, d, True) for d in (2, 3, 4, 5)]
    comp = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30)
    assert comp.perft_position(p, 1) == 17
    eng.close()
    comp.close()


@pytest.mark.parametrize("leaf_kernel", [1, 2, 4, 5, 6])
def test_readme_known_totals(gpu_engine, leaf_kernel):
    # README.md:51-52 and :92 (RTX PRO 6000 / GB10 tables)
    prev = gpu_engine.get_tuning().leaf_kernel
    gpu_engine.set_tuning(leaf_kernel=leaf_kernel)
    assert gpu_engine.perft_position(pg.parse_fen(START), 8) == 84_998_978_956
    assert gpu_engine.perft_position(pg.parse_fen(KIWIPETE), 7) == 374_190_009_323
    gpu_engine.set_tuning(leaf_kernel=prev)


def test_readme_startpos_perft9(gpu_engine):
    # README.md:51: 2,439,530,234,167
    assert gpu_engine.perft_position(pg.parse_fen(START), 9) == 2_439_530_234_167


def test_config1_small_workload(gpu_engine, golden, oracle):
    p = pg.config_position(8, 0)
    want = {c["name"]: c for c in golden}["cfg_8ply_seed0"]["counts"]
    assert [gpu_engine.perft_position(p, d) for d in range(1, 6)] == want
    assert gpu_engine.perft_position(p, 5) == oracle.perft(pg.to_fen(p), 5)


def test_bench_workload_divide_consistency(gpu_engine):
    """perft 7 of the bench position equals the sum of perft 6 over its
    children and the launch-depth split (size-independent properties)."""
    p = pg.config_position(4, 1)
    whole = gpu_engine.perft_position(p, 7)
    parts = sum(gpu_engine.perft_position(pg.make_move(p, m), 6) for m in pg.generate_moves(p))
    assert whole == parts
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30, launch_depth=5)
    split, _ = eng.perft_launch(p, 7)
    eng.close()
    assert whole == split


def test_bench_position_perft6_vs_oracle(gpu_engine, oracle):
    p = pg.config_position(4, 1)
    fen = pg.to_fen(p)
    assert gpu_engine.perft_position(p, 6) == oracle.perft(fen, 6)


def test_small_arena_splits_the_root():
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 20)
    p = pg.parse_fen(START)
    assert eng.perft_position(p, 6) == 119_060_324
    eng.close()


def test_perft_launch_host_recursion():
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30, launch_depth=4)
    res = eng.perft(START, 6)
    assert [r for r, _ in res] == [20, 400, 8902, 197281, 4865609, 119060324]
    eng.close()


def test_batch_matches_oracle(oracle):
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30)
    roots = pg.uneven_roots(48, 6, 40, seed=2)
    got = eng.perft_batch(roots, [4] * len(roots))
    want = [oracle.perft(pg.to_fen(r), 4) for r in roots]
    assert got == want
    eng.close()


def test_stats_and_timing(gpu_engine):
    p = pg.config_position(4, 1)
    gpu_engine.set_timing(True)
    n = gpu_engine.perft_position(p, 6)
    st = gpu_engine.last_stats()
    gpu_engine.set_timing(False)
    assert st.nodes == n
    assert st.leaf_ms > 0 and st.device_ms >= st.leaf_ms
    assert st.leaf_positions > st.leaf_edges > 0
    assert st.kernels == 3 * st.levels + 1


def test_cli_gpu_output():
    cli = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")
    out = subprocess.run([cli, KIWIPETE, "5", "-nott"], capture_output=True, text=True, check=True).stdout
    lines = [l.split(",")[0] for l in out.splitlines() if l.startswith("Perft(")]
    assert lines == ["Perft(01): 48", "Perft(02): 2039", "Perft(03): 97862", "Perft(04): 4085603",
                     "Perft(05): 193690690"]


def test_batch_matches_single_root_runs():
    """Config-3 style roots (uneven playouts, both sides to move): one
    batched pass per depth equals per-root plain runs, bit for bit."""
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=4 << 30)
    roots = pg.uneven_roots(256, 6, 40, seed=2)
    assert {r.color for r in roots} == {0, 1}
    depths = [1 + (i % 5) for i in range(len(roots))]
    got = eng.perft_batch(roots, depths)
    want = [eng.perft_position(r, d) for r, d in zip(roots, depths)]
    assert got == want
    eng.close()


def test_batch_splits_when_arena_is_small():
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=8 << 20)
    roots = pg.uneven_roots(64, 6, 40, seed=7)
    got = eng.perft_batch(roots, [5] * len(roots))
    ref = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30)
    assert got == [ref.perft_position(r, 5) for r in roots]
    eng.close()
    ref.close()


@pytest.mark.parametrize("cfg", [dict(leaf_threads=128), dict(leaf_threads=512), dict(gen_threads=64),
                                 dict(leaf_fuse=1)])
def test_tuned_launch_parameters_keep_counts(cfg, golden):
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    eng.set_tuning(**cfg)
    for case in golden[:30]:
        p = pg.parse_fen(case["fen"])
        for d, want in enumerate(case["counts"], start=1):
            assert eng.perft_position(p, d) == want, (cfg, case["name"], d)
    eng.close()


def test_autotune_picks_a_candidate():
    from perft_gpu_2026_b200 import autotune

    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    res = autotune.tune(eng, depth=5)
    assert res["best"] in autotune.candidates()
    assert eng.get_tuning().as_dict()["leaf_threads"] == res["best"]["leaf_threads"]
    eng.close()


@pytest.mark.parametrize("threads", [128, 256])
def test_deferred_evasion_leaf(golden, threads):
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    eng.set_tuning(leaf_kernel=3, leaf_threads=threads)
    for case in golden:
        p = pg.parse_fen(case["fen"])
        for d, want in enumerate(case["counts"], start=1):
            assert eng.perft_position(p, d) == want, (case["name"], d)
    assert eng.perft_position(pg.parse_fen(KIWIPETE), 6) == 8031647685
    eng.close()


MATED = "rnb1kbnr/pppp1ppp/8/4p3/6Pq/5P2/PPPPP2P/RNBQKBNR w KQkq - 1 3"  # side to move is checkmated
STALEMATE = "7k/5Q2/6K1/8/8/8/8/8 b - - 0 1"  # side to move has no move, not in check


def test_edge_depths_and_terminal_positions(gpu_engine, oracle):
    """perft(0) = 1, terminal roots count 0 at every depth >= 1, on the
    single-root and the batched paths."""
    for fen in (START, MATED, STALEMATE):
        p = pg.parse_fen(fen)
        assert gpu_engine.perft_position(p, 0) == 1
        for d in (1, 2, 3):
            assert gpu_engine.perft_position(p, d) == oracle.perft(fen, d), (fen, d)
    roots = [pg.parse_fen(f) for f in (START, MATED, STALEMATE, START)]
    assert gpu_engine.perft_batch(roots, [0, 3, 2, 1]) == [1, 0, 0, 20]
    # packed roots with one depth for all, and an empty batch
    assert gpu_engine.perft_batch(pg.pack_positions(roots), 2) == [400, 0, 0, 400]
    assert gpu_engine.perft_batch([], []) == []


def test_batched_leaf_ranked_and_unranked_agree():
    """The batched leaf with and without ranking each CTA's children by move
    count, ranked with listed pieces, and balanced across the warps
    (leaf_kernel 4 / 1 / 5 / 6), on uneven roots, both colours to move; also
    the planned batches' grid and queue leaves with kernels 5 and 6."""
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    roots = pg.uneven_roots(192, 6, 40, seed=23)
    depths = [2 + (i % 4) for i in range(len(roots))]
    eng.set_tuning(leaf_kernel=4)
    ranked = eng.perft_batch(roots, depths)
    eng.set_tuning(leaf_kernel=1)
    plain = eng.perft_batch(roots, depths)
    eng.set_tuning(leaf_kernel=5)
    listed = eng.perft_batch(roots, depths)
    eng.set_tuning(leaf_kernel=6)
    balanced = eng.perft_batch(roots, depths)
    assert ranked == plain == listed == balanced
    assert ranked == [eng.perft_position(r, d) for r, d in zip(roots, depths)]
    eng.mlp_init(seed=3, out_bias=[4.5, 9.5, 14.5, 19.0])
    for leaf_kernel in (5, 6):
        for planned_leaf in (1, 2):
            eng.set_tuning(leaf_kernel=leaf_kernel, planned_leaf=planned_leaf)
            got, _ = eng.perft_batch_planned(roots, depths)
            assert list(got) == ranked, (leaf_kernel, planned_leaf)
    # a batch big enough for 1024-thread balanced CTAs (more than 8 per SM)
    big = pg.uneven_roots(2048, 6, 30, seed=29)
    eng.set_tuning(leaf_kernel=6)
    b6 = eng.perft_batch(big, [5] * len(big))
    eng.set_tuning(leaf_kernel=1)
    assert b6 == eng.perft_batch(big, [5] * len(big))
    eng.close()


@pytest.mark.parametrize("leaf_kernel,threads", [(5, 128), (5, 256), (5, 512), (6, 128), (6, 256), (6, 512),
                                                  (6, 1024)])
def test_listed_piece_leaf_on_playouts(threads, leaf_kernel, oracle):
    """Leaf kernel 5 (own-piece squares listed once per child) against the
    oracle on playout positions of every game phase, both colours to move,
    including positions with promoted pieces (more than four of a kind fall
    back to the bitboard count)."""
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    eng.set_tuning(leaf_kernel=leaf_kernel, leaf_threads=threads)
    roots = [p for p in pg.random_playouts(4747, 40, 0, 160) if pg.count_moves(p, True) > 0]
    for p in roots:
        fen = pg.to_fen(p)
        assert eng.perft_position(p, 4) == oracle.perft(fen, 4), fen
    # five queens and five knights: the listed side has more than four of a
    # kind at odd depths (white's pieces are listed) and none at even depths
    many = "7k/8/8/8/8/8/NNNNN3/QQQQQ1K1 w - - 0 1"
    for d in (3, 4, 5):
        assert eng.perft_position(pg.parse_fen(many), d) == oracle.perft(many, d), d
    eng.close()
