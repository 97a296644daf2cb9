"""The scheduler network's hand-written kernels (embedding-bag layer 1, BF16
tensor-core GEMMs, Adam) against the FP32 numpy restatement: forward values,
loss and every parameter gradient."""
import numpy as np
import pytest

import perft_gpu_2026_b200 as pg
from perft_gpu_2026_b200 import mlp_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = pg.Engine(device=0, use_tt=False, arena_bytes=1 << 30)
    e.mlp_init(seed=11, out_bias=[4.0, 9.0, 14.0, 19.0])
    yield e
    e.close()


def _batch(n, seed):
    pos = [pg.random_playout(seed + i, (i * 7) % 50)[0] for i in range(n)]
    rng = np.random.default_rng(seed)
    t = rng.uniform(0, 20, size=(n, 4)).astype(np.float32)
    return pos, t


def test_gradients_match_numpy_reference(eng):
    pos, t = _batch(128, 500)
    g, loss = eng.mlp_gradients(pos, t)
    params = eng.mlp_params()
    _, ref_loss, ref_g = mlp_ref.forward_backward(params, mlp_ref.features(pos), t)
    # BF16 operands, FP32 accumulation: 2 % relative tolerance per tensor
    assert abs(loss - ref_loss) <= 1e-3 * max(1.0, ref_loss)
    sl = [(mlp_ref.OFF_W1, mlp_ref.OFF_B1), (mlp_ref.OFF_B1, mlp_ref.OFF_W2), (mlp_ref.OFF_W2, mlp_ref.OFF_B2),
          (mlp_ref.OFF_B2, mlp_ref.OFF_W3), (mlp_ref.OFF_W3, mlp_ref.OFF_B3), (mlp_ref.OFF_B3, mlp_ref.N_PARAMS)]
    for a, b in sl:
        d = np.linalg.norm(g[a:b] - ref_g[a:b])
        r = np.linalg.norm(ref_g[a:b])
        assert d <= 2e-2 * r + 1e-6, (a, b, d, r)


def test_prediction_matches_numpy_forward(eng):
    pos, t = _batch(100, 900)  # not a multiple of 64: the library pads
    y = eng.mlp_predict(pos)
    ref_y, _, _ = mlp_ref.forward_backward(eng.mlp_params(), mlp_ref.features(pos), t)
    assert np.allclose(y, ref_y, rtol=1e-2, atol=2e-2)


def test_training_learns_perft_sizes():
    e = pg.Engine(device=0, use_tt=False, arena_bytes=2 << 30)
    pos = [pg.random_playout(70_000 + i, i % 60)[0] for i in range(4096)]
    pos = [p for p in pos if pg.count_moves(p, True) > 0][:3968]
    counts = np.array([e.perft_batch(pos, [d] * len(pos)) for d in (1, 2, 3, 4)], dtype=np.float64).T
    t = np.log2(1.0 + counts)
    e.mlp_init(seed=3, out_bias=list(t.mean(0)))
    base = float(((t - t.mean(0)) ** 2).mean())
    loss = e.mlp_train(pos, t, epochs=30, batch=256, lr=2e-3)
    assert loss < 0.3 * base, (loss, base)
    e.close()
