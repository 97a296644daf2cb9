"""Learned batch planner: predicted level sizes, bin-packing, root splitting
and graph-captured batches must give exactly the counts of the plain batched
path - also when the plan is wrong (overflow -> exact rerun)."""
import numpy as np
import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu


def _train(eng, n=3072, seed=90_000):
    pos = [pg.random_playout(seed + i, i % 60)[0] for i in range(n)]
    pos = [p for p in pos if pg.count_moves(p, True) > 0]
    counts = np.array([eng.perft_batch(pos, [d] * len(pos)) for d in (1, 2, 3, 4)], dtype=np.float64).T
    t = np.log2(1.0 + counts)
    eng.mlp_init(seed=5, out_bias=list(t.mean(0)))
    eng.mlp_train(pos, t, epochs=20, batch=256, lr=2e-3)


def test_planned_batch_matches_exact_counts():
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=4 << 30)
    _train(eng)
    roots = pg.uneven_roots(200, 6, 40, seed=31)
    depths = [2 + (i % 4) for i in range(len(roots))]
    got, st = eng.perft_batch_planned(roots, depths)
    assert got == eng.perft_batch(roots, depths)
    assert st.graph_batches >= 1
    # the packed form with one depth for all, an empty batch, terminal roots
    packed = pg.pack_positions(roots)
    assert eng.perft_batch_planned(packed, 4)[0] == eng.perft_batch(packed, 4)
    empty, st0 = eng.perft_batch_planned([], [])
    assert empty == [] and st0.batches == 0
    mated = pg.parse_fen("rnb1kbnr/pppp1ppp/8/4p3/6Pq/5P2/PPPPP2P/RNBQKBNR w KQkq - 1 3")
    assert eng.perft_batch_planned([mated, roots[0]], [5, 1])[0] == [0, pg.count_moves(roots[0])]
    eng.close()


def test_wrong_plan_reruns_exactly():
    # an untrained network predicting ~0 for every level: every batch
    # overflows its plan and is rerun with exact sizing
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    eng.mlp_init(seed=9, out_bias=[0.0, 0.0, 0.0, 0.0])
    params = eng.mlp_params()
    params[:] = 0.0
    eng.mlp_set_params(params)
    roots = pg.uneven_roots(64, 6, 40, seed=32)
    got, st = eng.perft_batch_planned(roots, [5] * len(roots))
    assert got == eng.perft_batch(roots, [5] * len(roots))
    assert st.retries >= 1
    eng.close()


def test_large_roots_are_split():
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=64 << 20)
    _train(eng, n=1024, seed=91_000)
    roots = [pg.config_position(4, 1), pg.parse_fen(pg.START_FEN)]
    got, st = eng.perft_batch_planned(roots, [7, 7])
    ref = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30)
    assert got == [ref.perft_position(r, 7) for r in roots]
    assert st.split_roots >= 1
    ref.close()
    eng.close()


def test_trained_network_plans_a_tight_arena_better_than_a_constant_guess():
    """What the network gains over planning without it: the same planner fed a
    constant size guess (every root predicted at the training mean of log2
    perft(k)) against the trained network, on 64 uneven roots at perft 6 in a
    512 MB arena.  The constant guess underestimates the large roots, so a
    batch outgrows its plan and is rerun exactly (measured: 1 rerun); the
    trained network plans the same batches with none.  Counts are equal in
    both cases; the prediction error is clearly lower when trained."""
    from perft_gpu_2026_b200 import scheduler

    big = pg.Engine(device=0, use_tt=False, arena_bytes=8 << 30)
    pos, y, _ = scheduler.make_training_set(big, 1 << 16)
    held = pg.uneven_roots(64, 10, 30, seed=11)
    depths = [6] * len(held)
    want = big.perft_batch(held, depths)
    truth = np.log2(1.0 + scheduler.label(big, held))
    big.close()

    eng = pg.Engine(device=0, use_tt=False, arena_bytes=512 << 20)
    res = {}
    for name in ("constant", "trained"):
        eng.mlp_init(seed=1, out_bias=list(y.mean(0)))
        if name == "constant":
            p = eng.mlp_params()
            p[:] = 0
            p[-4:] = list(y.mean(0))  # output bias only: the same guess for every root
            eng.mlp_set_params(p)
        else:
            eng.mlp_train(pos, y, epochs=12, batch=4096, lr=2e-3)
        mae = float(np.abs(eng.mlp_predict(held) - truth).mean())
        got, st = eng.perft_batch_planned(held, depths)
        assert got == want, name
        res[name] = (mae, st.retries)
    eng.close()
    # a strict gain: the constant guess must rerun at least one batch, the
    # trained network none
    assert res["trained"][1] == 0, res
    assert res["constant"][1] > res["trained"][1], res
    assert res["trained"][0] < 0.8 * res["constant"][0], res


def test_planned_batch_strict_mode_matches_strict_per_root():
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30, strict=True)
    _train(eng, n=1024)
    roots = pg.uneven_roots(96, 6, 40, seed=21)
    depths = [3 + (i % 3) for i in range(len(roots))]
    got, _ = eng.perft_batch_planned(roots, depths)
    assert got == [eng.perft_position(r, d) for r, d in zip(roots, depths)]
    eng.close()
