"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls that need a GPU)."""
import ctypes
import glob
import os
import re

import perft_gpu_2026_b200 as pg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(pb_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("pb_create", "pb_destroy", "pb_perft", "pb_perft_position", "pb_perft_launch",
                 "pb_perft_batch", "pb_perft_cpu", "pb_parse_fen", "pb_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(pg.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_host_context():
    assert pg.version().startswith("perft-b200")
    eng = pg.Engine(device=-1)
    assert eng.perft_cpu(pg.parse_fen(pg.START_FEN), 3) == 8902
    eng.close()


def test_gpu_entry_points_refuse_host_context():
    eng = pg.Engine(device=-1)
    try:
        eng.perft_position(pg.parse_fen(pg.START_FEN), 3)
        raised = False
    except pg.PerftError as e:
        raised = e.code == pg.PB_ERR_NODEVICE
    assert raised
