"""Host side of the engine (no GPU): the C ABI's chess core, FEN handling and
the workload generator, checked against the oracle and the fixtures."""
import ctypes

import pytest

import perft_gpu_2026_b200 as pg


def test_host_perft_matches_fixtures(golden):
    eng = pg.Engine(device=-1)
    bad = []
    for case in golden:
        p = pg.parse_fen(case["fen"])
        for d, want in enumerate(case["counts"], start=1):
            if want > 30_000_000:
                continue
            got = eng.perft_cpu(p, d)
            if got != want:
                bad.append((case["name"], d, got, want))
    assert not bad, bad


@pytest.mark.parametrize("strict", [False, True])
def test_host_core_matches_oracle_on_playouts(oracle, strict):
    eng = pg.Engine(device=-1, strict=strict)
    for seed in range(120):
        p, _, _ = pg.random_playout(7000 + seed, 4 + (seed * 13) % 70)
        fen = pg.to_fen(p)
        for d in (1, 2, 3):
            assert eng.perft_cpu(p, d) == oracle.perft(fen, d, strict), (fen, d)


def test_generation_matches_strict_count(golden):
    for case in golden:
        p = pg.parse_fen(case["fen"])
        assert len(pg.generate_moves(p)) == pg.count_moves(p, strict=True), case["name"]


def test_generated_moves_match_oracle_as_sets(oracle, golden):
    for case in golden:
        p = pg.parse_fen(case["fen"])
        mine = sorted(pg.move_uci(m) for m in pg.generate_moves(p))
        ref = sorted(pg.move_uci(m) for m in oracle.moves(case["fen"]))
        assert mine == ref, case["name"]


def test_fen_round_trip(golden):
    for case in golden:
        p = pg.parse_fen(case["fen"])
        q = pg.parse_fen(pg.to_fen(p))
        assert p.key() == q.key(), case["name"]


@pytest.mark.parametrize("fen", [
    "8/8/8/8/8/8/8/8 w - - 0 1",            # no kings
    "4k3/8/8/8/8/8/8/4KK2 w - - 0 1",       # two white kings
    "4k3/4K3/8/8/8/8/8/8 w - - 0 1",        # adjacent kings
    "4k3/8/8/8/8/8/8/P3K3 w - - 0 1",       # pawn on the first rank
    "4k3/8/8/8/8/8/8/4R2K w - - 0 1",       # black (not to move) in check
])
def test_fen_rejects_impossible_positions(fen):
    with pytest.raises(pg.PerftError):
        pg.parse_fen(fen)


def test_fen_drops_inconsistent_rights_and_ep():
    p = pg.parse_fen("4k3/8/8/8/8/8/8/4K3 w KQkq e6 0 1")
    assert p.state == 0
    p = pg.parse_fen("4k3/8/8/3Pp3/8/8/8/4K3 w - e6 0 1")
    assert p.state >> 4 == 5


def test_playout_generator_matches_oracle(oracle):
    for seed in range(40):
        plies = 1 + seed % 50
        p, n, st = pg.random_playout(seed, plies)
        ofen, on, ost = oracle.playout_fen(seed, plies)
        assert n == on and st == ost
        q = pg.parse_fen(ofen)
        # the oracle (like the reference -cpu path) records an en-passant file
        # after every double push; the engine only when a capture can follow
        assert p.key()[:4] == q.key()[:4] and p.color == q.color
        assert p.state & 15 == q.state & 15
        if p.state >> 4:
            assert p.state >> 4 == q.state >> 4


def test_config_positions_are_stable(golden):
    byname = {c["name"]: c for c in golden}
    for name in ("cfg_8ply_seed0", "cfg_4ply_seed1", "cfg_2ply_seed4"):
        c = byname[name]
        p = pg.config_position(c["plies"], c["seed"])
        assert pg.to_fen(p) == c["fen"]


def test_uneven_roots_have_moves():
    roots = pg.uneven_roots(64, 6, 40, seed=2)
    assert len(roots) == 64
    assert all(pg.count_moves(r, True) > 0 for r in roots)
    again = pg.uneven_roots(64, 6, 40, seed=2)
    assert [r.key() for r in roots] == [r.key() for r in again]


def test_packed_positions_and_per_root_ints():
    """The batch format of the C ABI: packing a list copies the positions in
    order, a packed array passes through as the same object, and per-root
    ints accept one int for all or one per root (the wrong length is refused)."""
    roots = pg.random_playouts(5, 64, 0, 30)
    packed = pg.random_playouts(5, 64, 0, 30, packed=True)
    assert isinstance(packed, ctypes.Array) and len(packed) == 64
    assert [p.key() for p in packed] == [p.key() for p in roots]
    again = pg.pack_positions(roots)
    assert [p.key() for p in again] == [p.key() for p in roots]
    assert pg.pack_positions(packed) is packed
    view = pg.pack_slice(packed, 10, 20)
    assert [p.key() for p in view] == [p.key() for p in roots[10:20]]
    assert ctypes.addressof(view) == ctypes.addressof(packed) + 10 * ctypes.sizeof(pg.Pos)  # no copy
    assert len(pg.pack_slice(packed, 60, 80)) == 4
    assert [p.key() for p in pg.pack_slice(roots, 10, 20)] == [p.key() for p in roots[10:20]]
    assert pg._c_ints(5, 3).tolist() == [5, 5, 5]
    assert pg._c_ints([1, 2, 3], 3).tolist() == [1, 2, 3]
    with pytest.raises(ValueError):
        pg._c_ints([1, 2], 3)
    # a batch call without a GPU reaches the library with the packed arrays
    eng = pg.Engine(device=-1)
    with pytest.raises(pg.PerftError):
        eng.perft_batch(packed, 3)


def test_cpu_cli_output_format():
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")
    out = subprocess.run([cli, pg.START_FEN, "4", "-cpu"], capture_output=True, text=True, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("Perft(")]
    assert [l.split(",")[0] for l in lines] == ["Perft(01): 20", "Perft(02): 400", "Perft(03): 8902",
                                                 "Perft(04): 197281"]
    assert all(" seconds" in l for l in lines)


def test_cli_batch_file_and_json(tmp_path):
    import json
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")
    f = tmp_path / "pos.epd"
    f.write_text("# comment\n"
                 "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1 ;D1 20 ;D2 400 ;D3 8902\n"
                 "2n4k/1P1P4/8/8/8/8/8/4K3 w - - 0 1 ;D1 17 ;D2 93\n")
    out = subprocess.run([cli, "-batch", str(f), "-cpu", "-json"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    js = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert [j["nodes"] for j in js] == ["37", "493", "10523"]
    assert "0 mismatches" in out.stdout
    f.write_text("2n4k/1P1P4/8/8/8/8/8/4K3 w - - 0 1 ;D1 21\n")  # the exact count, not the reference's
    out = subprocess.run([cli, "-batch", str(f), "-cpu"], capture_output=True, text=True)
    assert out.returncode == 2 and "MISMATCH" in out.stdout
    out = subprocess.run([cli, "-batch", str(f), "-cpu", "-strict"], capture_output=True, text=True)
    assert out.returncode == 0


def test_host_edge_depths_and_terminal_positions(oracle):
    eng = pg.Engine(device=-1)
    mated = "rnb1kbnr/pppp1ppp/8/4p3/6Pq/5P2/PPPPP2P/RNBQKBNR w KQkq - 1 3"
    stalemate = "7k/5Q2/6K1/8/8/8/8/8 b - - 0 1"
    for fen in (pg.START_FEN, mated, stalemate):
        p = pg.parse_fen(fen)
        assert eng.perft_cpu(p, 0) == 1
        for d in (1, 2, 3):
            assert eng.perft_cpu(p, d) == oracle.perft(fen, d), (fen, d)
    assert pg.count_moves(pg.parse_fen(mated)) == 0
    assert pg.count_moves(pg.parse_fen(stalemate)) == 0


def test_cli_flags_anywhere_and_positional_launch_depth():
    """The reference's argument handling: flags may come before, between or
    after the positional arguments, and a third positional is the launch
    depth; every form counts the same."""
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")
    kiwi = "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -"
    want = ["Perft(01): 48", "Perft(02): 2039", "Perft(03): 97862"]
    for argv in ([kiwi, "3", "-cpu", "-nott"], ["-cpu", kiwi, "-nott", "3"], ["-nott", "-cpu", kiwi, "3", "2"],
                 [kiwi, "-ld", "2", "3", "-cpu"]):
        out = subprocess.run([cli] + argv, capture_output=True, text=True, check=True).stdout
        got = [l.split(",")[0] for l in out.splitlines() if l.startswith("Perft(")]
        assert got == want, argv


def test_incremental_hash_equals_full_hash_along_playouts():
    """The key after every move, updated from the parent's key, equals the key
    computed from scratch - over playouts long enough to meet castling, en
    passant, promotions and captures - and different move orders reaching the
    same position give the same key."""
    seen_flags = set()
    st = 8080
    for game in range(300):
        p = pg.parse_fen(pg.START_FEN)
        key = pg.position_hash(p)
        for ply in range(160):
            moves = pg.generate_moves(p)
            if not moves:
                break
            r, st = pg.splitmix64(st)
            m = moves[r % len(moves)]
            seen_flags.add(m >> 12)
            key = pg.hash_after_move(key, p, m)
            p = pg.make_move(p, m)
            assert key == pg.position_hash(p), (game, ply, pg.to_fen(p))
    assert {1, 2, 3, 5}.issubset(seen_flags) and any(f & 8 for f in seen_flags), seen_flags
    # transposition: 1.Nf3 Nf6 2.Nc3 Nc6 and 1.Nc3 Nc6 2.Nf3 Nf6
    def play(ucis):
        p = pg.parse_fen(pg.START_FEN)
        key = pg.position_hash(p)
        for u in ucis:
            m = next(m for m in pg.generate_moves(p) if pg.move_uci(m) == u)
            key = pg.hash_after_move(key, p, m)
            p = pg.make_move(p, m)
        return key, p.key()
    a, pa = play(["g1f3", "g8f6", "b1c3", "b8c6"])
    b, pb = play(["b1c3", "b8c6", "g1f3", "g8f6"])
    assert pa == pb and a == b
    c, _ = play(["g1f3", "g8f6", "b1c3", "b8a6"])
    assert c != a


def test_cli_journal_resumes_a_partial_run(tmp_path):
    """-journal: a run records every root move's subtree at the final depth;
    a rerun after losing part of the file recomputes only the missing moves
    and prints the same totals."""
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(pg.__file__), "perft_gpu")
    kiwi = "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -"
    j = tmp_path / "run.journal"

    def run():
        out = subprocess.run([cli, kiwi, "4", "-cpu", "-journal", str(j)], capture_output=True, text=True,
                             check=True).stdout
        lines = [l.split(",")[0] for l in out.splitlines() if l.startswith("Perft(")]
        return lines, out

    want = ["Perft(01): 48", "Perft(02): 2039", "Perft(03): 97862", "Perft(04): 4085603"]
    lines, out = run()
    assert lines == want and "read back" not in out
    rec = j.read_text().splitlines()
    assert len(rec) == 48 and all(r.startswith("4 ") and r.endswith(kiwi) for r in rec)
    j.write_text("\n".join(rec[:20] + ["3 a2a3 999 " + kiwi]) + "\n")  # an interrupted run (+ another depth)
    lines, out = run()
    assert lines == want and "journal: 20 root moves read back" in out
    assert len([r for r in j.read_text().splitlines() if r.startswith("4 ")]) == 48


def test_u128_accumulation_and_text_across_2_64():
    """128-bit counts (uint128.h:46-108): the library's accumulation, the one
    the host recursion applies to every subtree count, carries into the high
    word, and the printed text is the exact decimal value.  The reference's
    start position perft 14 total (README.md:63) is the known value past 2^64."""
    import random

    two64 = 1 << 64
    rng = random.Random(5)
    # subtree counts near 2^63..2^64: the running sum crosses 2^64 many times
    vals = [rng.randrange(two64 // 2, two64) for _ in range(200)] + [two64 - 1, 1, 0, two64 - 1]
    acc = 0
    for v in vals:
        acc = pg.u128_add(acc, v)
    assert acc == sum(vals) and acc >> 64 > 1
    assert pg.u128_add(two64 - 1, 1) == two64  # carry out of the low word
    perft14 = 61885021521585529237
    assert perft14 > two64
    for v in (0, 1, 999_999_999, 1_000_000_000, two64 - 1, two64, two64 + 1, perft14, acc,
              10 ** 27, 10 ** 27 - 1, (1 << 128) - 1):
        assert pg.u128_text(v) == str(v), v
    # the sum of the perft 14 total split into u64-sized parts
    parts = [perft14 // 7] * 6 + [perft14 - 6 * (perft14 // 7)]
    acc = 0
    for v in parts:
        acc = pg.u128_add(acc, v)
    assert pg.u128_text(acc) == "61885021521585529237"


def test_listed_piece_counts_equal_bitboard_counts(golden):
    """The listed-piece counter of leaf kernel 5 (the side's knight and slider
    squares listed once per parent position) against the bitboard counter on
    every child of playout positions and of the fixture positions (pins,
    captures of listed pieces, checks, promotions, castling, en passant)."""
    positions = [pg.parse_fen(c["fen"]) for c in golden]
    positions += pg.random_playouts(31337, 6000, 0, 120)
    # grandchildren of the fixtures as parents too: more pinned and captured pieces
    for c in golden[:20]:
        p = pg.parse_fen(c["fen"])
        positions += [pg.make_move(p, m) for m in pg.generate_moves(p)]
    checked, bad = pg.selftest_listed_counts(positions)
    assert bad == 0
    assert checked > 100_000


@pytest.mark.parametrize("use_tt", [False, True])
def test_breadth_first_host_driver(use_tt, golden):
    """host_driver 2: the tree above the launch depth expanded ply by ply
    (transpositions merged by key, each with its path count, when tables are
    on) must give the depth-first driver's counts (perft_cpu_recurse order)
    on a host-only context, and the known totals."""
    kiwi = "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq -"
    cases = [(pg.START_FEN, 5, 4_865_609), (kiwi, 4, 4_085_603)]
    cases += [(c["fen"], len(c["counts"]), c["counts"][-1]) for c in golden[:12] if c["counts"][-1] < 3_000_000]
    for ld in (1, 2, 3):
        bf = pg.Engine(device=-1, use_tt=use_tt, launch_depth=ld, host_tt_mb=64)
        bf.set_tuning(host_driver=2)
        df = pg.Engine(device=-1, use_tt=use_tt, launch_depth=ld, host_tt_mb=64)
        for fen, depth, want in cases:
            p = pg.parse_fen(fen)
            got, _ = bf.perft_launch(p, depth)
            ref, _ = df.perft_launch(p, depth)
            assert got == ref == want, (fen, depth, ld, got, ref)
        bf.close()
        df.close()
