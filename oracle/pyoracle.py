"""TEST/BENCH INFRASTRUCTURE ONLY: ctypes access to oracle/liboracle.so.

The scalar oracle (hyoracle.c) checks the CUDA backend in tests/ and __graft_entry__.smoke(); the
AVX2 restatement (avx2_port.cpp) is the CPU baseline bench.py times. The shipped package never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


class Hit(C.Structure):
    _fields_ = [("score", C.c_int32), ("db_index", C.c_uint64), ("query_end", C.c_int64),
                ("target_end", C.c_int64)]


class Alignment(C.Structure):
    _fields_ = [("score", C.c_int32), ("query_start", C.c_uint64), ("query_end", C.c_uint64),
                ("target_start", C.c_uint64), ("target_end", C.c_uint64), ("n_ops", C.c_uint64)]


_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)


def _load():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    sig = {
        "hyo_scoring_validate": (C.c_int, [C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, _i64p, _i64p, _i64p]),
        "hyo_magnitude_bound": (C.c_int64, [C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_uint64]),
        "hyo_required_width": (C.c_int, [C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_uint64, _i64p]),
        "hyo_align_core": (None, [_u8p, C.c_uint64, _u8p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, _i32p, _i64p, _i64p]),
        "hyo_scan": (None, [_u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, C.c_int, _u8p, C.c_uint64, C.POINTER(Hit)]),
        "hyo_scan_all_mt": (None, [_u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, C.c_int, _u8p, C.c_uint64, C.POINTER(Hit), C.c_int]),
        "hyo_scan_scores_mt": (None, [_u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, _u8p, C.c_uint64, _i32p, C.c_int]),
        "hyo_align_pairs": (C.c_int, [_u8p, _u64p, _u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, C.c_int, C.POINTER(Hit), C.c_int, _i64p, _i64p]),
        "hyo_traceback": (None, [_u8p, C.c_uint64, _u8p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, C.POINTER(Alignment), _u8p]),
        "hyo_align": (C.c_int, [_u8p, C.c_uint64, _u8p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, C.c_uint64, C.POINTER(Alignment), _u8p, _i64p, _i64p]),
        "hyo_scan_all_aligned_mt": (None, [_u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, _u8p, C.c_uint64, C.POINTER(Alignment), _u8p, C.c_int]),
        "hyo_position_max": (C.c_int32, [_u8p, C.c_uint64, _u8p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, _i32p, _i64p]),
        "hyo_position_max_mt": (None, [_u8p, _u64p, _u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, _i32p, _i32p, C.c_int]),
        "hyo_score2": (C.c_int, [_i32p, C.c_uint64, C.c_int32, C.c_uint64, C.c_int32, C.c_int32, _i32p, _u64p]),
        "hyo_traceback_needed": (C.c_uint64, [C.c_uint64, C.c_uint64, C.c_uint64]),
        "hyo_traceback_min_bytes_for_database": (C.c_uint64, [C.c_uint64, C.c_uint64]),
        "hyo_brute": (C.c_int32, [C.c_int, _u8p, C.c_uint64, _u8p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32]),
        "hyb_db_create": (C.c_void_p, [_u8p, _u64p, C.c_uint64, _i32p, C.c_uint64, C.c_int32, C.c_int32, C.c_int, C.c_int, C.c_uint64, C.c_int]),
        "hyb_db_destroy": (None, [C.c_void_p]),
        "hyb_scratch_create": (C.c_void_p, []),
        "hyb_scratch_destroy": (None, [C.c_void_p]),
        "hyb_scan": (None, [C.c_void_p, C.c_void_p, _u8p, C.c_uint64, C.POINTER(Hit)]),
        "hyb_scan_scores": (None, [C.c_void_p, C.c_void_p, _u8p, C.c_uint64, _i32p]),
        "hyb_scan_many": (None, [C.c_void_p, _u8p, _u64p, C.c_uint64, C.POINTER(Hit), C.c_int]),
        "hyb_scan_stream": (None, [C.POINTER(C.c_void_p), _u64p, C.c_uint64, _u8p, _u64p, C.c_uint64,
                                   C.POINTER(Hit), C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _u8(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a if a.size else np.zeros(1, np.uint8)


def _p(a, t):
    return a.ctypes.data_as(t)


def as_hit(h):
    """(score, db_index, query_end or None, target_end or None)."""
    return (int(h.score), int(h.db_index), None if h.query_end < 0 else int(h.query_end),
            None if h.target_end < 0 else int(h.target_end))


def _mat(matrix):
    return np.ascontiguousarray(np.asarray(matrix, dtype=np.int64).astype(np.int32))


def concat(seqs):
    parts = [np.asarray(list(s) if not isinstance(s, np.ndarray) else s, dtype=np.int64).astype(np.uint8)
             for s in seqs]
    off = np.zeros(len(parts) + 1, np.uint64)
    if parts:
        off[1:] = np.cumsum([len(p) for p in parts])
    res = np.concatenate(parts) if parts and off[-1] else np.zeros(1, np.uint8)
    return _u8(res), off


def required_width(mode, min_e, max_e, go, ge, m, n):
    b = C.c_int64()
    w = lib.hyo_required_width(int(mode), min_e, max_e, go, ge, m, n, C.byref(b))
    return w, int(b.value)


def magnitude_bound(mode, min_e, max_e, go, ge, m, n):
    return int(lib.hyo_magnitude_bound(int(mode), min_e, max_e, go, ge, m, n))


def align_pair(q, t, matrix, al, go, ge, mode, search_type=1):
    """(score, query_end, target_end) of one pair (align_core); ends None for Score."""
    qa = np.asarray(list(q), dtype=np.int64).astype(np.uint8)
    ta = np.asarray(list(t), dtype=np.int64).astype(np.uint8)
    qb, tb, mat = _u8(qa), _u8(ta), _mat(matrix)
    s, qe, te = C.c_int32(), C.c_int64(), C.c_int64()
    lib.hyo_align_core(_p(qb, _u8p), len(qa), _p(tb, _u8p), len(ta), _p(mat, _i32p), al, go, ge,
                       int(mode), C.byref(s), C.byref(qe), C.byref(te))
    if search_type == 0:
        return int(s.value), None, None
    return (int(s.value), None if qe.value < 0 else int(qe.value),
            None if te.value < 0 else int(te.value))


class OracleDb:
    """The scalar oracle's view of a database: scan / scan_all / scan_scores semantics."""

    def __init__(self, seqs_or_concat, matrix, al, go, ge, mode, search_type):
        if isinstance(seqs_or_concat, tuple):
            self.res, self.off = _u8(seqs_or_concat[0]), np.ascontiguousarray(seqs_or_concat[1], dtype=np.uint64)
        else:
            self.res, self.off = concat(seqs_or_concat)
        self.n = len(self.off) - 1
        self.mat = _mat(matrix)
        self.al, self.go, self.ge, self.mode, self.st = al, go, ge, int(mode), int(search_type)

    def _args(self):
        return (_p(self.res, _u8p), _p(self.off, _u64p), self.n, _p(self.mat, _i32p), self.al,
                self.go, self.ge, self.mode)

    def scan(self, query):
        q = _u8(np.asarray(list(query), dtype=np.int64).astype(np.uint8) if not isinstance(query, np.ndarray) else query)
        ql = len(query)
        h = Hit()
        lib.hyo_scan(*self._args(), self.st, _p(q, _u8p), ql, C.byref(h))
        return as_hit(h)

    def scan_all(self, query, threads=8):
        q = _u8(np.asarray(list(query), dtype=np.int64).astype(np.uint8) if not isinstance(query, np.ndarray) else query)
        out = (Hit * max(self.n, 1))()
        lib.hyo_scan_all_mt(*self._args(), self.st, _p(q, _u8p), len(query), out, threads)
        return [as_hit(out[k]) for k in range(self.n)]

    def seq(self, k):
        return self.res[int(self.off[k]): int(self.off[k + 1])]

    def scan_all_aligned(self, query):
        """Database::scan_all_aligned (src/database.rs:540-549): every sequence traced back."""
        return [traceback(query, self.seq(k), self.mat, self.al, self.go, self.ge, self.mode)
                for k in range(self.n)]

    def scan_all_aligned_mt(self, query, threads=8):
        """scan_all_aligned over `threads` threads: list of alignment tuples."""
        q = _seq(query)
        out = (Alignment * max(self.n, 1))()
        cap = self.n * len(query) + int(self.off[-1] - self.off[0]) + 1
        ops = np.zeros(cap, np.uint8)
        lib.hyo_scan_all_aligned_mt(*self._args(), _p(q, _u8p), len(query), out, _p(ops, _u8p), threads)
        res = []
        for k in range(self.n):
            base = k * len(query) + int(self.off[k] - self.off[0])
            res.append(as_alignment(out[k], ops[base: base + int(out[k].n_ops)]))
        return res

    def scan_aligned(self, query):
        """Database::scan_aligned (src/database.rs:527-536): (db_index, alignment) of the winner."""
        k = self.scan(query)[1]
        return k, traceback(query, self.seq(k), self.mat, self.al, self.go, self.ge, self.mode)

    def scan_scores(self, query, threads=8):
        q = _u8(np.asarray(list(query), dtype=np.int64).astype(np.uint8) if not isinstance(query, np.ndarray) else query)
        out = np.empty(max(self.n, 1), np.int32)
        lib.hyo_scan_scores_mt(*self._args(), _p(q, _u8p), len(query), _p(out, _i32p), threads)
        return out[: self.n]


def align_pairs(pairs_q, pairs_t, matrix, al, go, ge, mode, search_type, threads=8):
    """Returns (status, failed_index, hits list)."""
    qr, qo = concat(pairs_q)
    tr, to = concat(pairs_t)
    mat = _mat(matrix)
    n = len(qo) - 1
    out = (Hit * max(n, 1))()
    d1, d2 = C.c_int64(), C.c_int64()
    st = lib.hyo_align_pairs(_p(qr, _u8p), _p(qo, _u64p), _p(tr, _u8p), _p(to, _u64p), n, _p(mat, _i32p),
                             al, go, ge, int(mode), int(search_type), out, threads, C.byref(d1), C.byref(d2))
    return st, [as_hit(out[k]) for k in range(n)], (int(d1.value), int(d2.value))


U64_MAX = (1 << 64) - 1
OPS = "MXID"  # AlignOp codes 0 Match, 1 Mismatch, 2 Ins, 3 Del (src/align.rs:47-56)


def _seq(x):
    return _u8(np.asarray(list(x) if not isinstance(x, np.ndarray) else x, dtype=np.int64).astype(np.uint8))


def as_alignment(a, ops):
    """(score, query_start, query_end, target_start, target_end, ops bytes)."""
    return (int(a.score), int(a.query_start), int(a.query_end), int(a.target_start),
            int(a.target_end), bytes(ops[: int(a.n_ops)]))


def traceback(q, t, matrix, al, go, ge, mode):
    """traceback_full + walk (src/align.rs:345-545) on validated input."""
    qb, tb, mat = _seq(q), _seq(t), _mat(matrix)
    a = Alignment()
    ops = np.zeros(len(q) + len(t) + 1, np.uint8)
    lib.hyo_traceback(_p(qb, _u8p), len(q), _p(tb, _u8p), len(t), _p(mat, _i32p), al, go, ge,
                      int(mode), C.byref(a), _p(ops, _u8p))
    return as_alignment(a, ops)


def align(q, t, matrix, al, go, ge, mode, max_bytes=U64_MAX):
    """align (src/align.rs:169-222): (status, alignment or None, (d1, d2))."""
    qb, tb, mat = _seq(q), _seq(t), _mat(matrix)
    a = Alignment()
    ops = np.zeros(len(q) + len(t) + 1, np.uint8)
    d1, d2 = C.c_int64(), C.c_int64()
    st = lib.hyo_align(_p(qb, _u8p), len(q), _p(tb, _u8p), len(t), _p(mat, _i32p), al, go, ge,
                       int(mode), max_bytes, C.byref(a), _p(ops, _u8p), C.byref(d1), C.byref(d2))
    return st, (as_alignment(a, ops) if st == 0 else None), (int(d1.value), int(d2.value))


def position_max(q, t, matrix, al, go, ge):
    """(column maxima list, score, target_end or None) of align_pair_position_max."""
    qb, tb, mat = _seq(q), _seq(t), _mat(matrix)
    out = np.zeros(max(1, len(t)), np.int32)
    te = C.c_int64()
    s = lib.hyo_position_max(_p(qb, _u8p), len(q), _p(tb, _u8p), len(t), _p(mat, _i32p), al, go, ge,
                             _p(out, _i32p), C.byref(te))
    return [int(v) for v in out[: len(t)]], int(s), (None if te.value < 0 else int(te.value))


def position_max_many(q_res, q_off, t_res, t_off, matrix, al, go, ge, threads=8):
    """(column maxima aligned with t_res, scores) of many pairs over `threads` threads."""
    q_res, t_res = _u8(q_res), _u8(t_res)
    q_off = np.ascontiguousarray(q_off, dtype=np.uint64)
    t_off = np.ascontiguousarray(t_off, dtype=np.uint64)
    n = len(q_off) - 1
    out = np.zeros(max(1, int(t_off[-1] - t_off[0])), np.int32)
    scores = np.zeros(max(n, 1), np.int32)
    mat = _mat(matrix)
    lib.hyo_position_max_mt(_p(q_res, _u8p), _p(q_off, _u64p), _p(t_res, _u8p), _p(t_off, _u64p), n,
                            _p(mat, _i32p), al, go, ge, _p(out, _i32p), _p(scores, _i32p), threads)
    return out, scores[:n]


def score2(colmax, best_score, best_target_end, matrix_max, min_score):
    cm = np.ascontiguousarray(np.asarray(colmax, dtype=np.int64).astype(np.int32))
    cm1 = cm if cm.size else np.zeros(1, np.int32)
    sc, pos = C.c_int32(), C.c_uint64()
    ok = lib.hyo_score2(_p(cm1, _i32p), len(cm), best_score, best_target_end, matrix_max, min_score,
                        C.byref(sc), C.byref(pos))
    return (int(sc.value), int(pos.value)) if ok else None


def traceback_needed(m, n, max_bytes):
    return int(lib.hyo_traceback_needed(m, n, max_bytes))


def traceback_min_bytes_for_database(max_m, max_n):
    return int(lib.hyo_traceback_min_bytes_for_database(max_m, max_n))


def cigar(ops, extended=False):
    """Alignment::cigar / cigar_extended (src/align.rs:96-130): run-length of the op letters."""
    letters = ("=X" if extended else "MM") + "ID"
    out, prev, run = [], None, 0
    for o in ops:
        c = letters[o]
        if c == prev:
            run += 1
        else:
            if prev is not None:
                out.append(f"{run}{prev}")
            prev, run = c, 1
    if prev is not None:
        out.append(f"{run}{prev}")
    return "".join(out)


def brute(mode, q, t, matrix, al, go, ge):
    qa = _u8(np.asarray(list(q), dtype=np.int64).astype(np.uint8))
    ta = _u8(np.asarray(list(t), dtype=np.int64).astype(np.uint8))
    mat = _mat(matrix)
    return int(lib.hyo_brute(int(mode), _p(qa, _u8p), len(q), _p(ta, _u8p), len(t), _p(mat, _i32p), al, go, ge))


class Avx2Db:
    """The AVX2 baseline restatement (db-order batches, Precomputed, width groups)."""

    def __init__(self, res, off, matrix, al, go, ge, mode, search_type, max_query_len, gathered_i8=False):
        self.res, self.off = _u8(res), np.ascontiguousarray(off, dtype=np.uint64)
        self.mat = _mat(matrix)
        self.h = lib.hyb_db_create(_p(self.res, _u8p), _p(self.off, _u64p), len(self.off) - 1,
                                   _p(self.mat, _i32p), al, go, ge, int(mode), int(search_type),
                                   max_query_len, 1 if gathered_i8 else 0)
        if not self.h:
            raise ValueError("width proof failed")
        self.n = len(self.off) - 1

    def __del__(self):
        if getattr(self, "h", None):
            lib.hyb_db_destroy(self.h)
            self.h = None

    def scan_many(self, queries, threads):
        qr, qo = concat(queries)
        out = (Hit * max(len(queries), 1))()
        lib.hyb_scan_many(self.h, _p(qr, _u8p), _p(qo, _u64p), len(queries), out, threads)
        return [as_hit(out[k]) for k in range(len(queries))]

    def scan_scores(self, query):
        q = _u8(np.asarray(list(query), dtype=np.int64).astype(np.uint8))
        sc = lib.hyb_scratch_create()
        out = np.empty(max(self.n, 1), np.int32)
        lib.hyb_scan_scores(self.h, sc, _p(q, _u8p), len(query), _p(out, _i32p))
        lib.hyb_scratch_destroy(sc)
        return out[: self.n]


class Avx2SlicedDb:
    """The AVX2 baseline over one database held as consecutive slices of about equal residues, so
    that a query stream can be spread over every host thread in (query, slice) units
    (hyb_scan_stream): the same hits as Avx2Db.scan_many, with no thread idle on a long query."""

    def __init__(self, res, off, matrix, al, go, ge, mode, search_type, max_query_len, n_slices):
        off = np.ascontiguousarray(off, dtype=np.uint64)
        n = len(off) - 1
        total = int(off[-1] - off[0])
        cuts = [0]
        for s in range(1, n_slices):
            k = int(np.searchsorted(off, off[0] + total * s // n_slices))
            if cuts[-1] < k < n:
                cuts.append(k)
        cuts.append(n)
        self.slices = []
        for a, b in zip(cuts[:-1], cuts[1:]):
            sub_off = off[a:b + 1] - off[a]
            self.slices.append(Avx2Db(np.asarray(res)[int(off[a]):int(off[b])], sub_off, matrix, al, go, ge, mode,
                                      search_type, max_query_len))
        self.base = np.ascontiguousarray(cuts[:-1], dtype=np.uint64)
        self.n = n

    def scan_stream(self, queries, threads):
        qr, qo = concat(queries)
        out = (Hit * max(len(queries), 1))()
        hs = (C.c_void_p * len(self.slices))(*[d.h for d in self.slices])
        lib.hyb_scan_stream(hs, _p(self.base, _u64p), len(self.slices), _p(qr, _u8p), _p(qo, _u64p),
                            len(queries), out, threads)
        return [as_hit(out[k]) for k in range(len(queries))]
