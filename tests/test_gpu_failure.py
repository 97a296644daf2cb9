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


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_device_table_races_never_return_a_foreign_count(gpu_engine, mode):
    """Stores and probes of colliding keys from every thread at once: a probe
    either misses or returns its own key's count (the XOR lock and the full
    key check reject torn and foreign entries).  Mode 2 runs the 16-byte
    format at the size the engine actually builds (2^24 slots), with the
    keys packed into 8 slots so they still collide."""
    bad, hits = gpu_engine.selftest_tt_race(mode)
    assert hits > 1000
    assert bad == 0
