"""Unit tests of the BFS level kernels against the host chess core, through
the C ABI on caller-owned device buffers: the make+count kernel must give
bit-identical child boards and states and exact move counts, and the staged
generation kernel the host generator's moves in the host generator's order,
each tagged with its parent (also when a CTA's moves overflow its
shared-memory staging)."""
import numpy as np
import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu


def _parents(color, n=1000):
    ps = [p for p in pg.random_playouts(6060 + color, 4 * n, 0, 80) if p.color == color and pg.count_moves(p, True)]
    return ps[:n]


def _max_moves(golden):
    fen = {c["name"]: c for c in golden}["max_moves_218"]["fen"]
    return pg.parse_fen(fen)


def _device_positions(ps):
    import torch

    bb = np.array([[p.bb[k] for k in range(4)] for p in ps], dtype=np.uint64)
    st = np.array([p.state for p in ps], dtype=np.uint8)
    return torch.from_numpy(bb.view(np.int64)).cuda(), torch.from_numpy(st).cuda()


@pytest.mark.parametrize("color", [0, 1])
def test_expand_kernel_matches_host_make_and_count(gpu_engine, color):
    import torch

    ps = _parents(color)
    pidx, mvs, children = [], [], []
    for j, p in enumerate(ps):
        for m in pg.generate_moves(p):
            pidx.append(j)
            mvs.append(m)
            children.append(pg.make_move(p, m))
    n = len(mvs)
    d_b, d_s = _device_positions(ps)
    d_pi = torch.tensor(pidx, dtype=torch.int32, device="cuda")
    d_mv = torch.from_numpy(np.array(mvs, dtype=np.uint16).view(np.int16)).cuda()
    c_b = torch.zeros((n, 4), dtype=torch.int64, device="cuda")
    c_s = torch.zeros(n, dtype=torch.uint8, device="cuda")
    c_n = torch.zeros(n, dtype=torch.int32, device="cuda")
    gpu_engine.dev_expand(d_b.data_ptr(), d_s.data_ptr(), color, d_pi.data_ptr(), d_mv.data_ptr(), n, len(ps),
                          c_b.data_ptr(), c_s.data_ptr(), c_n.data_ptr())
    got_b = c_b.cpu().numpy().view(np.uint64)
    got_s = c_s.cpu().numpy()
    got_n = c_n.cpu().numpy()
    want_b = np.array([[c.bb[k] for k in range(4)] for c in children], dtype=np.uint64)
    assert np.array_equal(got_b, want_b)
    assert np.array_equal(got_s, np.array([c.state for c in children], dtype=np.uint8))
    assert np.array_equal(got_n, np.array([pg.count_moves(c, True) for c in children], dtype=np.int32))


@pytest.mark.parametrize("color", [0, 1])
def test_generate_kernel_matches_host_order(gpu_engine, golden, color):
    import torch

    ps = _parents(color)
    if color == 0:
        ps = ps[:300] + [_max_moves(golden)] * 200 + ps[300:]  # 200 x 218 moves: overflows the staging
    counts = np.array([pg.count_moves(p, True) for p in ps], dtype=np.int64)
    offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    total = int(counts.sum())
    d_b, d_s = _device_positions(ps)
    d_offs = torch.from_numpy(offs).cuda()
    d_total = torch.tensor([total], dtype=torch.int64, device="cuda")
    o_mv = torch.zeros(total, dtype=torch.int16, device="cuda")
    o_pi = torch.zeros(total, dtype=torch.int32, device="cuda")
    gpu_engine.dev_generate(d_b.data_ptr(), d_s.data_ptr(), color, d_offs.data_ptr(), d_total.data_ptr(), len(ps),
                            o_mv.data_ptr(), o_pi.data_ptr())
    mv = o_mv.cpu().numpy().view(np.uint16)
    pi = o_pi.cpu().numpy()
    want_mv = np.concatenate([np.array(pg.generate_moves(p), dtype=np.uint16) for p in ps])
    want_pi = np.repeat(np.arange(len(ps), dtype=np.int32), counts)
    assert np.array_equal(mv, want_mv)
    assert np.array_equal(pi, want_pi)
