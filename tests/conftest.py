import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def oracle():
    import _oracle

    return _oracle.load()


@pytest.fixture(scope="session")
def golden():
    import json

    with open(os.path.join(TESTS, "golden", "ref_cpu_perft.json")) as f:
        return json.load(f)["cases"]


@pytest.fixture(scope="session")
def gpu_engine():
    import perft_gpu_2026_b200 as pg

    eng = pg.Engine(device=0, use_tt=False, arena_bytes=4 << 30)
    yield eng
    eng.close()
