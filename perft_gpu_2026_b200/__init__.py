"""perft_gpu_2026_b200 - Python binding of the B200 perft engine.

The engine is the native library ``libperftb200.so`` (CUDA kernels for sm_100a
plus a C++ host driver) behind the C ABI declared in ``include/perft_b200.h``.
This module loads it with ctypes and mirrors the reference's operator set:

    perft_gpu <fen> <depth> [-nott] [-dtt MB] [-htt MB] [-ld N] [-cpu]   (perft.cu:13-186)

``Engine.perft`` is the per-depth loop, ``Engine.perft_position`` the single
GPU breadth-first call (perft_gpu_host_bfs, perft_kernels.cu:620-990) and
``Engine.perft_cpu`` the host path (perft_cpu_dispatch, launcher.cu:807-816).
There is no Python fallback: if the library is missing the import fails.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PERFT_B200_LIB") or os.path.join(_HERE, "libperftb200.so")

START_FEN = "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1"

PB_OK = 0
PB_ERR_ARG = -1
PB_ERR_FEN = -2
PB_ERR_CUDA = -3
PB_ERR_NOMEM = -4
PB_ERR_DEVICE = -5
PB_ERR_NODEVICE = -6


class Pos(ctypes.Structure):
    """pb_pos: quad bitboard + state byte + side to move (40 bytes)."""

    _fields_ = [
        ("bb", ctypes.c_uint64 * 4),
        ("state", ctypes.c_uint8),
        ("color", ctypes.c_uint8),
        ("pad", ctypes.c_uint8 * 6),
    ]

    def key(self) -> Tuple[int, int, int, int, int, int]:
        return (self.bb[0], self.bb[1], self.bb[2], self.bb[3], self.state, self.color)


class U128(ctypes.Structure):
    _fields_ = [("lo", ctypes.c_uint64), ("hi", ctypes.c_uint64)]

    def value(self) -> int:
        return (self.hi << 64) | self.lo


class Opts(ctypes.Structure):
    _fields_ = [
        ("arena_bytes", ctypes.c_size_t),
        ("use_tt", ctypes.c_int),
        ("device_tt_mb", ctypes.c_int),
        ("host_tt_mb", ctypes.c_int),
        ("launch_depth", ctypes.c_int),
        ("strict", ctypes.c_int),
        ("verbose", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    """pb_stats: per-call statistics (CUDA-event device times, sizes, launches)."""

    _fields_ = [
        ("device_ms", ctypes.c_double),
        ("leaf_ms", ctypes.c_double),
        ("leaf_edges", ctypes.c_uint64),
        ("leaf_positions", ctypes.c_uint64),
        ("nodes", ctypes.c_uint64),
        ("kernels", ctypes.c_uint32),
        ("levels", ctypes.c_uint32),
        ("level_sizes", ctypes.c_uint64 * 16),
        ("h2d_bytes", ctypes.c_uint64),
        ("d2h_bytes", ctypes.c_uint64),
    ]


class Tuning(ctypes.Structure):
    """pb_tuning: launch parameters (zero = keep current)."""

    _fields_ = [("leaf_kernel", ctypes.c_int), ("leaf_blocks_per_sm", ctypes.c_int),
                ("leaf_threads", ctypes.c_int), ("gen_threads", ctypes.c_int), ("leaf_fuse", ctypes.c_int),
                ("tt_replace", ctypes.c_int), ("planned_leaf", ctypes.c_int), ("host_driver", ctypes.c_int),
                ("tt_leaf", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k in ("leaf_kernel", "leaf_blocks_per_sm", "leaf_threads", "gen_threads",
                                              "leaf_fuse", "tt_replace", "planned_leaf", "host_driver", "tt_leaf")}


class PlanStats(ctypes.Structure):
    _fields_ = [("batches", ctypes.c_uint32), ("graph_batches", ctypes.c_uint32), ("retries", ctypes.c_uint32),
                ("split_roots", ctypes.c_uint32)]


class PerftError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"perft engine error {code}: {msg}")
        self.code = code


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m perft_gpu_2026_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    sig = {
        "pb_version": (ctypes.c_char_p, []),
        "pb_default_opts": (None, [P(Opts)]),
        "pb_create": (ctypes.c_int, [ctypes.c_int, P(Opts), P(ctypes.c_void_p)]),
        "pb_destroy": (None, [ctypes.c_void_p]),
        "pb_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
        "pb_parse_fen": (ctypes.c_int, [ctypes.c_char_p, P(Pos)]),
        "pb_to_fen": (ctypes.c_int, [P(Pos), ctypes.c_char_p, ctypes.c_size_t]),
        "pb_perft_position": (ctypes.c_int, [ctypes.c_void_p, P(Pos), ctypes.c_int, P(ctypes.c_uint64)]),
        "pb_perft_launch": (ctypes.c_int, [ctypes.c_void_p, P(Pos), ctypes.c_int, P(U128), P(ctypes.c_double)]),
        "pb_perft": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, P(U128), P(ctypes.c_double)]),
        "pb_perft_cpu": (ctypes.c_int, [ctypes.c_void_p, P(Pos), ctypes.c_int, P(ctypes.c_uint64)]),
        "pb_perft_batch": (ctypes.c_int, [ctypes.c_void_p, P(Pos), P(ctypes.c_int), ctypes.c_int, P(ctypes.c_uint64)]),
        "pb_count_moves": (ctypes.c_int, [P(Pos), ctypes.c_int]),
        "pb_generate_moves": (ctypes.c_int, [P(Pos), P(ctypes.c_uint16)]),
        "pb_make_move": (ctypes.c_int, [P(Pos), ctypes.c_uint16]),
        "pb_position_hash": (ctypes.c_int, [P(Pos), P(U128)]),
        "pb_hash_after_move": (ctypes.c_int, [P(U128), P(Pos), ctypes.c_uint16, P(U128)]),
        "pb_random_playout": (ctypes.c_int, [P(ctypes.c_uint64), ctypes.c_int, P(Pos)]),
        "pb_random_playouts": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int, P(Pos),
                                               P(ctypes.c_int)]),
        "pb_selftest_listed_counts": (ctypes.c_int, [P(Pos), ctypes.c_int, P(ctypes.c_uint64), P(ctypes.c_uint64)]),
        "pb_u128_add": (None, [P(U128), P(U128)]),
        "pb_u128_text": (ctypes.c_int, [P(U128), ctypes.c_char_p, ctypes.c_size_t]),
        "pb_device_count": (ctypes.c_int, []),
        "pb_choose_launch_depth": (ctypes.c_int, [ctypes.c_void_p, P(Pos)]),
        "pb_prepare": (ctypes.c_int, [ctypes.c_void_p, P(Pos), ctypes.c_int]),
        "pb_set_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
        "pb_set_tuning": (ctypes.c_int, [ctypes.c_void_p, P(Tuning)]),
        "pb_get_tuning": (ctypes.c_int, [ctypes.c_void_p, P(Tuning)]),
        "pb_last_stats": (ctypes.c_int, [ctypes.c_void_p, P(Stats)]),
        "pb_mlp_param_count": (ctypes.c_size_t, []),
        "pb_mlp_init": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, P(ctypes.c_float)]),
        "pb_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, P(ctypes.c_float), ctypes.c_size_t]),
        "pb_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, P(ctypes.c_float), ctypes.c_size_t]),
        "pb_mlp_gradients": (ctypes.c_int, [ctypes.c_void_p, P(Pos), P(ctypes.c_float), ctypes.c_int,
                                             P(ctypes.c_float), P(ctypes.c_float)]),
        "pb_mlp_train": (ctypes.c_int, [ctypes.c_void_p, P(Pos), P(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_float, ctypes.c_uint64, P(ctypes.c_float)]),
        "pb_mlp_predict": (ctypes.c_int, [ctypes.c_void_p, P(Pos), ctypes.c_int, P(ctypes.c_float)]),
        "pb_perft_batch_planned": (ctypes.c_int, [ctypes.c_void_p, P(Pos), P(ctypes.c_int), ctypes.c_int,
                                                   P(ctypes.c_uint64), P(PlanStats)]),
        "pb_dev_scan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]),
        "pb_selftest_wait_timeout": (ctypes.c_int, [ctypes.c_void_p, P(ctypes.c_uint32), P(ctypes.c_double)]),
        "pb_selftest_tt_race": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_uint64), P(ctypes.c_uint64)]),
        "pb_selftest_gemm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, P(ctypes.c_uint16), P(ctypes.c_uint16), P(ctypes.c_float),
                                            ctypes.c_int, P(ctypes.c_double)]),
        "pb_dev_expand": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p]),
        "pb_dev_generate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                           ctypes.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


class _LazyLib:
    """Loads libperftb200.so on first use; raises ImportError if it is not built."""

    def __getattr__(self, name):
        global _LIB
        if _LIB is None:
            _LIB = _load()
        return getattr(_LIB, name)


lib = _LazyLib()


def device_count() -> int:
    return lib.pb_device_count()


def version() -> str:
    return lib.pb_version().decode()


def parse_fen(fen: str) -> Pos:
    p = Pos()
    rc = lib.pb_parse_fen(fen.encode(), ctypes.byref(p))
    if rc != PB_OK:
        raise PerftError(rc, f"invalid FEN: {fen!r}")
    return p


def to_fen(p: Pos) -> str:
    buf = ctypes.create_string_buffer(128)
    lib.pb_to_fen(ctypes.byref(p), buf, 128)
    return buf.value.decode()


def count_moves(p: Pos, strict: bool = False) -> int:
    return lib.pb_count_moves(ctypes.byref(p), int(strict))


def generate_moves(p: Pos) -> List[int]:
    buf = (ctypes.c_uint16 * 256)()
    n = lib.pb_generate_moves(ctypes.byref(p), buf)
    return list(buf[:n])


def make_move(p: Pos, move: int) -> Pos:
    q = Pos()
    ctypes.memmove(ctypes.byref(q), ctypes.byref(p), ctypes.sizeof(Pos))
    lib.pb_make_move(ctypes.byref(q), move)
    return q


def position_hash(p: Pos) -> int:
    """128-bit Zobrist key of the position (as one Python int)."""
    out = U128()
    lib.pb_position_hash(ctypes.byref(p), ctypes.byref(out))
    return out.value()


def hash_after_move(key: int, p: Pos, move: int) -> int:
    """Key after `move`, updated incrementally from `key` (the key of p)."""
    k = U128(key & ((1 << 64) - 1), key >> 64)
    out = U128()
    lib.pb_hash_after_move(ctypes.byref(k), ctypes.byref(p), move, ctypes.byref(out))
    return out.value()


def selftest_listed_counts(positions: Sequence[Pos]) -> Tuple[int, int]:
    """(children compared, mismatches) of the listed-piece move count against
    the bitboard count, on the host, over every child of each position."""
    arr = (Pos * len(positions))(*positions)
    checked, bad = ctypes.c_uint64(0), ctypes.c_uint64(0)
    rc = lib.pb_selftest_listed_counts(arr, len(positions), ctypes.byref(checked), ctypes.byref(bad))
    if rc != PB_OK:
        raise PerftError(rc, "listed-count self-test")
    return checked.value, bad.value


def u128_add(acc: int, v: int) -> int:
    """acc + v through the library's 128-bit accumulation (the one the host
    recursion applies to subtree counts), wrapping at 2^128 like the C type."""
    a = U128(acc & ((1 << 64) - 1), (acc >> 64) & ((1 << 64) - 1))
    b = U128(v & ((1 << 64) - 1), (v >> 64) & ((1 << 64) - 1))
    lib.pb_u128_add(ctypes.byref(a), ctypes.byref(b))
    return a.value()


def u128_text(v: int) -> str:
    """Decimal text of a 128-bit count as the command line prints it."""
    x = U128(v & ((1 << 64) - 1), (v >> 64) & ((1 << 64) - 1))
    buf = ctypes.create_string_buffer(48)
    n = lib.pb_u128_text(ctypes.byref(x), buf, 48)
    if n < 0:
        raise PerftError(n, "u128 text")
    return buf.value.decode()


def move_uci(m: int) -> str:
    f, t, fl = m & 63, (m >> 6) & 63, m >> 12
    s = "abcdefgh"[f & 7] + str(1 + (f >> 3)) + "abcdefgh"[t & 7] + str(1 + (t >> 3))
    if fl & 8:
        s += "nbrq"[fl & 3]
    return s


def random_playout(seed_state: int, plies: int) -> Tuple[Pos, int, int]:
    """Returns (position, plies played, advanced generator state)."""
    st = ctypes.c_uint64(seed_state)
    p = Pos()
    n = lib.pb_random_playout(ctypes.byref(st), plies, ctypes.byref(p))
    return p, n, st.value


def random_playouts(seed: int, n: int, min_plies: int, max_plies: int, packed: bool = False):
    """n playouts (threaded in the library); position i's generator state is
    the i-th splitmix64 draw of `seed`, its length uniform in [min, max].
    A list of Pos, or with packed=True the packed array (pack_positions)."""
    arr = (Pos * n)()
    rc = lib.pb_random_playouts(seed, n, min_plies, max_plies, arr, None)
    if rc != PB_OK:
        raise PerftError(rc, "pb_random_playouts failed")
    return arr if packed else list(arr)


def pack_positions(roots) -> ctypes.Array:
    """Positions as one contiguous pb_pos array, the batch format of the C
    ABI (pb_perft_batch, pb_perft_batch_planned, pb_mlp_predict).  A packed
    array is returned as it is; a sequence of Pos is copied once.  The batch
    methods accept either; passing the packed array spares the copy (about
    0.3 us per position in CPython) on every call."""
    if isinstance(roots, ctypes.Array) and roots._type_ is Pos:
        return roots
    return (Pos * len(roots))(*roots)


def pack_slice(roots, a: int, b: int) -> ctypes.Array:
    """Positions a..b-1 as a packed array: a view sharing the memory of a
    packed array (no copy), or a copy of that part of a sequence of Pos."""
    if isinstance(roots, ctypes.Array) and roots._type_ is Pos:
        b = min(b, len(roots))
        return (Pos * max(b - a, 0)).from_buffer(roots, a * ctypes.sizeof(Pos))
    return pack_positions(roots[a:b])


def _c_ints(values, n: int):
    """Per-position ints (or one int for all) as a contiguous C int array."""
    import numpy as np

    a = np.full(n, values, dtype=np.intc) if np.ndim(values) == 0 else np.ascontiguousarray(values, dtype=np.intc)
    if a.shape != (n,):
        raise ValueError(f"expected {n} values, got shape {a.shape}")
    return a


def splitmix64(state: int) -> Tuple[int, int]:
    """One splitmix64 step in Python: returns (value, new state)."""
    m = (1 << 64) - 1
    state = (state + 0x9E3779B97F4A7C15) & m
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
    return z ^ (z >> 31), state


@dataclass
class Workload:
    """A named set of root positions with their perft depths."""

    name: str
    roots: List[Pos]
    depths: List[int]


def config_position(plies: int, seed: int) -> Pos:
    """A position reached by `plies` random legal moves from the initial array."""
    p, _, _ = random_playout(seed, plies)
    return p


def uneven_roots(n: int, lo: int, hi: int, seed: int) -> List[Pos]:
    """n roots from playouts of U[lo, hi] plies, drawn from one splitmix64
    stream (length draw, then the moves), keeping roots with a legal move."""
    out: List[Pos] = []
    st = seed
    span = hi - lo + 1
    while len(out) < n:
        r, st = splitmix64(st)
        plies = lo + ((r * span) >> 64)
        c = ctypes.c_uint64(st)
        p = Pos()
        lib.pb_random_playout(ctypes.byref(c), plies, ctypes.byref(p))
        st = c.value
        if lib.pb_count_moves(ctypes.byref(p), 1) > 0:
            out.append(p)
    return out


class Engine:
    """A perft context on one device (device < 0: host only, the -cpu mode)."""

    def __init__(self, device: int = 0, use_tt: bool = False, arena_bytes: int = 0, strict: bool = False,
                 launch_depth: int = 0, device_tt_mb: int = 0, host_tt_mb: int = 0, verbose: bool = False):
        o = Opts()
        lib.pb_default_opts(ctypes.byref(o))
        o.use_tt = int(use_tt)
        o.arena_bytes = arena_bytes
        o.strict = int(strict)
        o.launch_depth = launch_depth
        o.device_tt_mb = device_tt_mb
        o.host_tt_mb = host_tt_mb
        o.verbose = int(verbose)
        h = ctypes.c_void_p()
        rc = lib.pb_create(device, ctypes.byref(o), ctypes.byref(h))
        if rc != PB_OK:
            raise PerftError(rc, "pb_create failed")
        self._h = h
        self.device = device

    def close(self) -> None:
        if self._h:
            lib.pb_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> None:
        if rc != PB_OK:
            raise PerftError(rc, lib.pb_last_error(self._h).decode())

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def perft_position(self, p: Pos, depth: int) -> int:
        out = ctypes.c_uint64()
        self._check(lib.pb_perft_position(self._h, ctypes.byref(p), depth, ctypes.byref(out)))
        return out.value

    def perft_launch(self, p: Pos, depth: int) -> Tuple[int, float]:
        out = U128()
        secs = ctypes.c_double()
        self._check(lib.pb_perft_launch(self._h, ctypes.byref(p), depth, ctypes.byref(out), ctypes.byref(secs)))
        return out.value(), secs.value

    def perft(self, fen: str, max_depth: int) -> List[Tuple[int, float]]:
        res = (U128 * max_depth)()
        secs = (ctypes.c_double * max_depth)()
        self._check(lib.pb_perft(self._h, fen.encode(), max_depth, res, secs))
        return [(res[i].value(), secs[i]) for i in range(max_depth)]

    def perft_cpu(self, p: Pos, depth: int) -> int:
        out = ctypes.c_uint64()
        self._check(lib.pb_perft_cpu(self._h, ctypes.byref(p), depth, ctypes.byref(out)))
        return out.value

    def perft_batch_planned(self, roots, depths):
        """Learned-planner batch: returns (counts, PlanStats).  roots: a
        sequence of Pos or a packed array (pack_positions); depths: one int
        per root, or one int for all."""
        import numpy as np

        arr = pack_positions(roots)
        n = len(arr)
        d = _c_ints(depths, n)
        out = np.zeros(n, dtype=np.uint64)
        st = PlanStats()
        self._check(lib.pb_perft_batch_planned(self._h, arr, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n,
                                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                               ctypes.byref(st)))
        return out.tolist(), st

    def perft_batch(self, roots, depths) -> List[int]:
        """Count-then-allocate batch (pb_perft_batch): one count per root.
        roots: a sequence of Pos or a packed array (pack_positions); depths:
        one int per root, or one int for all."""
        import numpy as np

        arr = pack_positions(roots)
        n = len(arr)
        d = _c_ints(depths, n)
        out = np.zeros(n, dtype=np.uint64)
        self._check(lib.pb_perft_batch(self._h, arr, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out.tolist()

    def set_timing(self, enable: bool = True) -> None:
        self._check(lib.pb_set_timing(self._h, int(enable)))

    def set_tuning(self, leaf_kernel: int = 0, leaf_blocks_per_sm: int = 0, leaf_threads: int = 0,
                   gen_threads: int = 0, leaf_fuse: int = 0, tt_replace: int = 0, planned_leaf: int = 0,
                   host_driver: int = 0, tt_leaf: int = 0) -> None:
        """Launch parameters (pb_set_tuning); 0 keeps the current value.
        leaf_kernel 1 = one edge per thread, 2 = cooperative, 3 = in-check
        children deferred, 4 = children ranked by move count,
        5 = ranked with each child's own-piece squares listed once,
        6 = as 5 with four children per thread balanced across the warps
        (default); leaf_threads 128/256/512, or 1024 with leaf kernel 6
        (default); gen_threads 64/128; leaf_fuse 1/2;
        tt_replace 1 = always overwrite, 2 = two-slot size priority;
        planned_leaf 1 = grid over the planned capacity (default),
        2 = persistent work-queue leaf; host_driver 1 = depth-first tree
        above the launch depth (default), 2 = breadth first with batched
        GPU calls; tt_leaf 1 = one edge per thread, 2 = persistent table leaf
        that counts only full CTAs of table misses."""
        t = Tuning()
        t.tt_replace = tt_replace
        t.planned_leaf = planned_leaf
        t.host_driver = host_driver
        t.tt_leaf = tt_leaf
        t.leaf_kernel = leaf_kernel
        t.leaf_blocks_per_sm = leaf_blocks_per_sm
        t.leaf_threads = leaf_threads
        t.gen_threads = gen_threads
        t.leaf_fuse = leaf_fuse
        self._check(lib.pb_set_tuning(self._h, ctypes.byref(t)))

    def get_tuning(self) -> Tuning:
        t = Tuning()
        self._check(lib.pb_get_tuning(self._h, ctypes.byref(t)))
        return t

    def last_stats(self) -> Stats:
        st = Stats()
        self._check(lib.pb_last_stats(self._h, ctypes.byref(st)))
        return st

    def prepare(self, p: Pos, max_depth: int) -> int:
        return lib.pb_prepare(self._h, ctypes.byref(p), max_depth)

    def choose_launch_depth(self, p: Pos) -> int:
        return lib.pb_choose_launch_depth(self._h, ctypes.byref(p))

    # ---- learned scheduler network
    def mlp_init(self, seed: int = 1, out_bias=None) -> None:
        ob = (ctypes.c_float * 4)(*out_bias) if out_bias is not None else None
        self._check(lib.pb_mlp_init(self._h, seed, ob))

    def mlp_params(self):
        import numpy as np

        n = lib.pb_mlp_param_count()
        buf = np.empty(n, dtype=np.float32)
        self._check(lib.pb_mlp_get_params(self._h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n))
        return buf

    def mlp_set_params(self, params) -> None:
        import numpy as np

        buf = np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib.pb_mlp_set_params(self._h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), buf.size))

    def mlp_gradients(self, positions: Sequence[Pos], targets):
        import numpy as np

        n = len(positions)
        arr = (Pos * n)(*positions)
        t = np.ascontiguousarray(targets, dtype=np.float32).reshape(n, 4)
        g = np.empty(lib.pb_mlp_param_count(), dtype=np.float32)
        loss = ctypes.c_float()
        FP = ctypes.POINTER(ctypes.c_float)
        self._check(lib.pb_mlp_gradients(self._h, arr, t.ctypes.data_as(FP), n, g.ctypes.data_as(FP),
                                         ctypes.byref(loss)))
        return g, loss.value

    def mlp_train(self, positions: Sequence[Pos], targets, epochs: int, batch: int = 4096, lr: float = 1e-3,
                  seed: int = 7) -> float:
        import numpy as np

        arr = pack_positions(positions)
        n = len(arr)
        t = np.ascontiguousarray(targets, dtype=np.float32).reshape(n, 4)
        loss = ctypes.c_float()
        self._check(lib.pb_mlp_train(self._h, arr, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n, epochs,
                                     batch, lr, seed, ctypes.byref(loss)))
        return loss.value

    def mlp_predict(self, positions: Sequence[Pos]):
        import numpy as np

        arr = pack_positions(positions)
        n = len(arr)
        out = np.empty((n, 4), dtype=np.float32)
        self._check(lib.pb_mlp_predict(self._h, arr, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def dev_expand(self, d_boards: int, d_states: int, color: int, d_pidx: int, d_moves: int, n: int, nparents: int,
                   d_child_boards: int, d_child_states: int, d_counts: int) -> None:
        """The make+count level kernel on caller-owned device buffers (tests)."""
        self._check(lib.pb_dev_expand(self._h, d_boards, d_states, color, d_pidx, d_moves, n, nparents, d_child_boards,
                                      d_child_states, d_counts))

    def dev_generate(self, d_boards: int, d_states: int, color: int, d_offs: int, d_total: int, n: int, d_moves: int,
                     d_pidx: int) -> None:
        """The staged generation kernel on caller-owned device buffers (tests)."""
        self._check(lib.pb_dev_generate(self._h, d_boards, d_states, color, d_offs, d_total, n, d_moves, d_pidx))

    def selftest_tt_race(self, mode: int):
        """(wrong hits, hits) of the device-table race self-test: mode 0 =
        1024-slot 16-byte table, 1 = 1024-slot 32-byte table, 2 = 2^24-slot
        16-byte table with the keys packed into 8 slots."""
        bad = ctypes.c_uint64()
        hits = ctypes.c_uint64()
        self._check(lib.pb_selftest_tt_race(self._h, int(mode), ctypes.byref(bad), ctypes.byref(hits)))
        return bad.value, hits.value

    def selftest_gemm(self, a_bits, b_bits, ta: bool, tb: bool, m: int, n: int, k: int, reps: int = 0):
        """The network's tensor-core GEMM on BF16 bit patterns (uint16 arrays in
        the layouts pb_selftest_gemm names); returns C as an (m, n) float32
        array, or with reps > 0 (C, mean CUDA-event ms of reps more launches)."""
        import numpy as np

        a = np.ascontiguousarray(a_bits, dtype=np.uint16)
        b = np.ascontiguousarray(b_bits, dtype=np.uint16)
        if a.size != m * k or b.size != k * n:
            raise ValueError("operand sizes do not match m, n, k")
        c = np.empty((m, n), dtype=np.float32)
        u16 = ctypes.POINTER(ctypes.c_uint16)
        ms = ctypes.c_double()
        self._check(lib.pb_selftest_gemm(self._h, int(ta), int(tb), m, n, k, a.ctypes.data_as(u16),
                                         b.ctypes.data_as(u16), c.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                         int(reps), ctypes.byref(ms)))
        return (c, ms.value) if reps > 0 else c

    def selftest_wait_timeout(self):
        """(device error word, seconds) of a scan tile whose predecessor never
        publishes: the bounded wait gives up and reports 1."""
        err = ctypes.c_uint32()
        secs = ctypes.c_double()
        self._check(lib.pb_selftest_wait_timeout(self._h, ctypes.byref(err), ctypes.byref(secs)))
        return err.value, secs.value

    def dev_scan(self, d_in: int, n: int, d_out: int, d_total: int) -> None:
        self._check(lib.pb_dev_scan(self._h, ctypes.c_void_p(d_in), n, ctypes.c_void_p(d_out), ctypes.c_void_p(d_total)))
