"""The scheduler network's hand-written kernels (embedding-bag layer 1, BF16
tcgen05 tensor-core GEMMs, Adam) against the FP32 numpy restatement: the GEMM
alone, forward values, loss and every parameter gradient."""
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


def _bf16(x):
    """float32 -> (BF16 bit patterns, the float32 values they hold); round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    bits = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return bits, (bits.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("ta,tb,m,n,k", [(0, 0, 192, 256, 256), (1, 0, 256, 256, 448), (0, 1, 200, 256, 256),
                                         (1, 1, 8, 128, 64), (0, 0, 4096, 256, 256), (1, 0, 256, 256, 4096),
                                         (1, 0, 136, 256, 1088), (0, 0, 128, 128, 640)])
def test_tensor_core_gemm_matches_numpy(eng, ta, tb, m, n, k):
    """k_gemm_tc against a float64 product of the same BF16 values: partial
    row tiles (M = 192, 200, 136, 8), an odd number of K chunks (448 = 7 x
    64), K split over CTAs (the weight-gradient shape 256 x 256 x 4096: 16
    splits of 4 chunks; 1088 = 17 chunks in 4 uneven splits; 640 = 10 chunks
    in 2), every transpose combination the network uses and one it does not."""
    rng = np.random.default_rng(m * 7 + k + 3 * ta + tb)
    a = rng.uniform(-1, 1, size=(m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, size=(k, n)).astype(np.float32)
    a_bits, a_val = _bf16(a.T.copy() if ta else a)
    b_bits, b_val = _bf16(b.T.copy() if tb else b)
    a_ref = (a_val.T if ta else a_val).astype(np.float64)
    b_ref = (b_val.T if tb else b_val).astype(np.float64)
    c = eng.selftest_gemm(a_bits, b_bits, bool(ta), bool(tb), m, n, k)
    want = a_ref @ b_ref
    # exact BF16 products, FP32 accumulation over k terms
    assert np.abs(c - want).max() <= 1e-5 * k + 1e-4, np.abs(c - want).max()


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
