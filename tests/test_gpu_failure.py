"""Device-side failure detection without a GPU fault: a wait that can never
be satisfied gives up after its bound, the kernel returns an error status the
host reads, and the context keeps working."""
import pytest

import perft_gpu_2026_b200 as pg

pytestmark = pytest.mark.gpu

DEVERR_SCAN_TIMEOUT = 1


def test_scan_wait_gives_up_and_reports(gpu_engine):
    err, secs = gpu_engine.selftest_wait_timeout()
    assert err == DEVERR_SCAN_TIMEOUT
    assert 0.0 < secs < 30.0
    # the same context and its stream are still usable
    assert gpu_engine.perft_position(pg.parse_fen(pg.START_FEN), 5) == 4_865_609
    err2, _ = gpu_engine.selftest_wait_timeout()
    assert err2 == DEVERR_SCAN_TIMEOUT
