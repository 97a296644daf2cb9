"""The allocation-free scan entry point (pb_scan_u32_noalloc).

Some callers of this library cannot allocate device memory when they need a
scan (an allocator's own out-of-memory path, a host framework that owns every
device buffer, a latency-critical loop that must not hit cudaMalloc's implicit
synchronisation).  This entry point keeps its scratch in a fixed array inside
the library; the test calls it through the C ABI and compares its output with
the regular entry point's (pb_dev_scan) on two calls in a row.  This file is
collected last so that a failure here leaves every other test already run."""
import ctypes

import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu

MAX_ITEMS = 8_388_608  # the entry point's documented limit


def _noalloc():
    lib = ctypes.CDLL(pg.LIB_PATH)
    fn = lib.pb_scan_u32_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def test_noalloc_scan_matches_regular_entry_point():
    import torch

    torch.cuda.set_device(0)
    fn = _noalloc()
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=64 << 20)
    g = torch.Generator().manual_seed(1234)
    # two calls in a row: a large input, then a smaller one (the shared
    # scratch still holds the first call's tile words)
    for n in (MAX_ITEMS - 5, 300_001):
        x = torch.randint(0, 219, (n,), generator=g, dtype=torch.int64)
        d_in = x.to(torch.int32).cuda()
        out_a = torch.full((n,), -1, dtype=torch.int64, device="cuda")
        tot_a = torch.full((1,), -1, dtype=torch.int64, device="cuda")
        out_b = torch.full((n,), -2, dtype=torch.int64, device="cuda")
        tot_b = torch.full((1,), -2, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        rc = fn(d_in.data_ptr(), n, out_a.data_ptr(), tot_a.data_ptr(), None)
        assert rc == pg.PB_OK
        eng.dev_scan(d_in.data_ptr(), n, out_b.data_ptr(), tot_b.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(out_a, out_b)
        assert torch.equal(tot_a, tot_b)
        assert int(tot_a.item()) == int(x.sum())
    eng.close()


def test_noalloc_scan_unaligned_buffers_on_a_side_stream():
    """Caller buffers off the 32-byte boundary take the scan's scalar path;
    the call runs on a caller-created stream, twice in a row."""
    import torch

    torch.cuda.set_device(0)
    fn = _noalloc()
    eng = pg.Engine(device=0, use_tt=False, arena_bytes=64 << 20)
    g = torch.Generator().manual_seed(99)
    side = torch.cuda.Stream()
    for n in (1_000_003, 70_001):
        x = torch.randint(0, 219, (n,), generator=g, dtype=torch.int64)
        buf_in = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        buf_in[1:].copy_(x.to(torch.int32))
        out_a = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
        tot_a = torch.full((2,), -1, dtype=torch.int64, device="cuda")
        out_b = torch.full((n,), -2, dtype=torch.int64, device="cuda")
        tot_b = torch.full((1,), -2, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        # one element in: 4 bytes off for the counts, 8 for the offsets
        rc = fn(buf_in.data_ptr() + 4, n, out_a.data_ptr() + 8, tot_a.data_ptr() + 8, side.cuda_stream)
        assert rc == pg.PB_OK
        eng.dev_scan(buf_in.data_ptr() + 4, n, out_b.data_ptr(), tot_b.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(out_a[1:], out_b)
        assert int(tot_a[1].item()) == int(tot_b.item()) == int(x.sum())
        assert torch.equal(out_b, torch.cumsum(x, 0).cuda() - x.cuda())
        assert int(out_a[0].item()) == -1 and int(tot_a[0].item()) == -1  # nothing written before the buffers
    eng.close()


def test_noalloc_scan_refuses_a_capturing_stream():
    """The call waits for its stream, which a CUDA graph capture cannot hold:
    on a capturing stream it returns PB_ERR_ARG before any GPU work."""
    import torch

    fn = _noalloc()
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    o = torch.zeros(16, dtype=torch.int64, device="cuda")
    t = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.stream(s):
        graph.capture_begin(capture_error_mode="thread_local")
        try:
            rcs.append(fn(d.data_ptr(), 16, o.data_ptr(), t.data_ptr(), s.cuda_stream))
            o.add_(0)  # keep the captured graph non-empty
        finally:
            graph.capture_end()
    assert rcs == [pg.PB_ERR_ARG]
    del graph


def test_noalloc_scan_rejects_sizes_beyond_its_scratch():
    import torch

    fn = _noalloc()
    d = torch.zeros(1, dtype=torch.int32, device="cuda")
    o = torch.zeros(1, dtype=torch.int64, device="cuda")
    # the size check happens before any GPU work, so tiny buffers are safe here
    assert fn(d.data_ptr(), MAX_ITEMS + 1, o.data_ptr(), o.data_ptr(), None) == pg.PB_ERR_ARG
