"""ctypes loader for the CPU oracle (oracle/liboracle.so), the checker of the
test suite.  Builds it with make if it is missing."""
import ctypes
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "liboracle.so")


class OPos(ctypes.Structure):
    _fields_ = [("bb", ctypes.c_uint64 * 4), ("state", ctypes.c_uint8), ("color", ctypes.c_uint8),
                ("pad", ctypes.c_uint8 * 6)]


class Oracle:
    def __init__(self, lib):
        self.lib = lib
        lib.or_perft.restype = ctypes.c_uint64
        lib.or_perft_strict.restype = ctypes.c_uint64
        lib.or_count_moves.restype = ctypes.c_uint32
        lib.or_count_moves_strict.restype = ctypes.c_uint32
        lib.or_generate_moves.restype = ctypes.c_uint32
        lib.or_splitmix64.restype = ctypes.c_uint64

    def pos(self, fen):
        p = OPos()
        if self.lib.or_parse_fen(fen.encode(), ctypes.byref(p)) != 0:
            raise ValueError(fen)
        return p

    def perft(self, fen, depth, strict=False):
        p = self.pos(fen)
        f = self.lib.or_perft_strict if strict else self.lib.or_perft
        return f(ctypes.byref(p), depth)

    def count(self, fen, strict=False):
        p = self.pos(fen)
        f = self.lib.or_count_moves_strict if strict else self.lib.or_count_moves
        return f(ctypes.byref(p))

    def moves(self, fen):
        p = self.pos(fen)
        buf = (ctypes.c_uint16 * 256)()
        n = self.lib.or_generate_moves(ctypes.byref(p), buf)
        return list(buf[:n])

    def playout_fen(self, seed, plies):
        st = ctypes.c_uint64(seed)
        p = OPos()
        n = self.lib.or_random_playout(ctypes.byref(st), plies, ctypes.byref(p))
        buf = ctypes.create_string_buffer(128)
        self.lib.or_to_fen(ctypes.byref(p), buf)
        return buf.value.decode(), n, st.value


def load() -> Oracle:
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True)
    return Oracle(ctypes.CDLL(LIB))
