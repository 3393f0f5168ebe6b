"""hyalite_b200 -- the B200 `cuda` backend of hyalite's inter-sequence database scan.

A Python mirror of hyalite's public API for this path (src/lib.rs:54-67): ``Scoring``, ``Mode``,
``SearchType``, ``BestHit``, ``Backend`` / ``BackendChoice`` / ``BACKEND_ENV_VAR``, ``Layout`` /
``LayoutChoice``, ``ScoreWidth``, ``Database`` / ``DatabaseBuilder`` / ``Scratch``,
``align_pairs`` and the traceback (``align``, ``Alignment``, ``AlignOp``, ``AlignedHit``,
``Database.scan_aligned`` / ``scan_all_aligned``), with the same names, argument meanings and error behaviour, over the C ABI of
include/hyalite_cuda.h. All compute runs in the in-tree CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import enum
import os
import weakref
from dataclasses import dataclass
from typing import Iterable, List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import lib

BACKEND_ENV_VAR = "HYALITE_BACKEND"


# ---- errors (src/error.rs:16-96) -----------------------------------------------------------------

class Error(Exception):
    """A hyalite error. ``kind`` is the variant name of src/error.rs (or a C-ABI-only condition such
    as ``QueryTooLong`` / ``Cuda``); ``fields`` holds the variant's fields."""

    _FIELDS = {
        "MatrixShape": ("alphabet_len", "expected", "got"),
        "NegativeGapPenalty": ("gap_open", "gap_ext"),
        "GapOpenLessThanExtend": ("gap_open", "gap_ext"),
        "ScoreRangeTooWide": ("bound",),
        "SymbolOutOfRange": ("symbol", "alphabet_len"),
        "BackendUnavailable": ("backend",),
        "QueryTooLong": ("len", "max"),
        "TracebackBudgetExceeded": ("needed_bytes", "budget_bytes"),
        "Cuda": ("code",),
    }

    def __init__(self, kind: str, **fields):
        self.kind = kind
        self.fields = fields
        super().__init__(f"{kind}{fields if fields else ''}")

    def __eq__(self, other):
        return isinstance(other, Error) and (self.kind, self.fields) == (other.kind, other.fields)

    def __hash__(self):
        return hash((self.kind, tuple(sorted(self.fields.items()))))

    @classmethod
    def from_status(cls, status: int) -> "Error":
        kind = _abi.STATUS_NAMES.get(status, f"Status{status}")
        d = _abi.last_detail()
        names = cls._FIELDS.get(kind, ())
        fields = {n: int(d[i]) for i, n in enumerate(names)}
        if kind == "TracebackBudgetExceeded":  # u64 / usize fields carried in int64
            fields = {n: v & (2**64 - 1) for n, v in fields.items()}
        if kind == "BackendUnavailable":
            fields["backend"] = Backend(fields["backend"])
        return cls(kind, **fields)


def _check(status: int) -> None:
    if status != _abi.OK:
        raise Error.from_status(status)


# ---- enums ----------------------------------------------------------------------------------------

class Mode(enum.IntEnum):
    """Alignment mode (src/mode.rs:11-27)."""
    Sw = 0
    Nw = 1
    Hw = 2
    Ov = 3
    Shw = 4

    def is_local(self) -> bool:
        return self is Mode.Sw

    def code(self) -> str:
        return {0: "SW", 1: "NW", 2: "HW", 3: "OV", 4: "SHW"}[int(self)]

    def __str__(self) -> str:
        return self.code()


ALL_MODES = (Mode.Sw, Mode.Nw, Mode.Hw, Mode.Ov, Mode.Shw)


USIZE_MAX = 2**64 - 1


class SearchType(enum.IntEnum):
    """What a search returns (src/search.rs:13-27). ``Alignment`` carries a traceback budget:
    ``SearchType.alignment(max_bytes)``; the bare member means ``max_bytes = usize::MAX``."""
    Score = 0
    ScoreEnd = 1
    Alignment = 2

    def tracks_end(self) -> bool:
        return self is not SearchType.Score

    @staticmethod
    def alignment(max_bytes: int) -> "AlignmentSearch":
        return AlignmentSearch(int(max_bytes))


@dataclass(frozen=True)
class AlignmentSearch:
    """SearchType::Alignment { max_bytes } (src/search.rs:20-26)."""
    max_bytes: int

    def tracks_end(self) -> bool:
        return True

    def __int__(self) -> int:
        return int(SearchType.Alignment)

    def __str__(self) -> str:
        return f"Alignment {{ max_bytes: {self.max_bytes} }}"


class ScoreWidth(enum.IntEnum):
    """src/width.rs:26-34."""
    I8 = 0
    I16 = 1
    I32 = 2

    def max_abs(self) -> int:
        return {0: 127, 1: 32767, 2: 536870911}[int(self)]

    def bytes(self) -> int:
        return {0: 1, 1: 2, 2: 4}[int(self)]


class Backend(enum.IntEnum):
    """src/backend.rs:25-36, plus ``Cuda`` (the enum is non-exhaustive upstream)."""
    Scalar = 0
    Sse41 = 1
    Avx2 = 2
    Neon = 3
    Cuda = 4

    def name_str(self) -> str:
        return lib.hy_backend_name(int(self)).decode()

    def is_available(self) -> bool:
        return bool(lib.hy_backend_is_available(int(self)))

    def __str__(self) -> str:
        return self.name_str()


@dataclass(frozen=True)
class BackendChoice:
    """``Auto`` or ``Force(backend)`` (src/backend.rs:123-133)."""
    forced: Optional[Backend] = None

    @staticmethod
    def Auto() -> "BackendChoice":
        return BackendChoice(None)

    @staticmethod
    def Force(b: Backend) -> "BackendChoice":
        return BackendChoice(Backend(b))

    @staticmethod
    def parse(s: str) -> "BackendChoice":
        """BackendChoice::parse (src/backend.rs:143-155), plus ``"cuda"``."""
        out = C.c_int()
        st = lib.hy_backend_parse(s.encode(), C.byref(out))
        if st != _abi.OK:
            raise Error("InvalidBackendName", name=s)
        return BackendChoice.Auto() if out.value == _abi.CHOICE_AUTO else BackendChoice.Force(Backend(out.value))

    def _code(self) -> int:
        return _abi.CHOICE_AUTO if self.forced is None else int(self.forced)


class Layout(enum.IntEnum):
    """src/inter.rs:317-330. On the device: Gathered adds two per-letter query-profile words per
    cell pair; Precomputed stores each pair column as one code and loads one pair-table word (Auto
    picks it for alphabets of at most 6 symbols). Results never depend on the layout."""
    Gathered = 0
    Precomputed = 1


@dataclass(frozen=True)
class LayoutChoice:
    forced: Optional[Layout] = None

    @staticmethod
    def Auto() -> "LayoutChoice":
        return LayoutChoice(None)

    @staticmethod
    def Force(layout: Layout) -> "LayoutChoice":
        return LayoutChoice(Layout(layout))

    def _code(self) -> int:
        return _abi.LAYOUT_AUTO if self.forced is None else int(self.forced)


@dataclass(frozen=True)
class BestHit:
    """src/hit.rs:16-25: 0-based ends, ``None`` when nothing aligned or for ``Score`` searches."""
    score: int
    db_index: int
    query_end: Optional[int]
    target_end: Optional[int]

    @staticmethod
    def _from(h: _abi.HyHit) -> "BestHit":
        return BestHit(int(h.score), int(h.db_index), None if h.query_end < 0 else int(h.query_end),
                       None if h.target_end < 0 else int(h.target_end))


# ---- traceback results (src/align.rs:40-150) ------------------------------------------------------

class AlignOp(enum.IntEnum):
    """src/align.rs:47-56: Match / Mismatch by symbol equality; Ins consumes a query symbol, Del a
    target symbol (the target is the reference)."""
    Match = 0
    Mismatch = 1
    Ins = 2
    Del = 3


def _cigar(ops: bytes, extended: bool) -> str:
    """Alignment::encode (src/align.rs:108-150): run-length of the op letters."""
    letters = ("=", "X", "I", "D") if extended else ("M", "M", "I", "D")
    out = []
    prev, run = None, 0
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


class Alignment:
    """src/align.rs:57-83: score, half-open spans and the operations (kept as one byte each,
    ``AlignOp`` codes; ``ops`` gives them as ``AlignOp`` values)."""
    __slots__ = ("score", "query_start", "query_end", "target_start", "target_end", "ops_bytes")

    def __init__(self, score, query_start, query_end, target_start, target_end, ops_bytes: bytes):
        self.score = int(score)
        self.query_start = int(query_start)
        self.query_end = int(query_end)
        self.target_start = int(target_start)
        self.target_end = int(target_end)
        self.ops_bytes = bytes(ops_bytes)

    @property
    def ops(self) -> List[AlignOp]:
        return [AlignOp(o) for o in self.ops_bytes]

    def cigar(self) -> str:
        return _cigar(self.ops_bytes, False)

    def cigar_extended(self) -> str:
        return _cigar(self.ops_bytes, True)

    def as_tuple(self):
        return (self.score, self.query_start, self.query_end, self.target_start, self.target_end,
                self.ops_bytes)

    def __eq__(self, other):
        return isinstance(other, Alignment) and self.as_tuple() == other.as_tuple()

    def __hash__(self):
        return hash(self.as_tuple())

    def __repr__(self):
        return (f"Alignment(score={self.score}, query={self.query_start}..{self.query_end}, "
                f"target={self.target_start}..{self.target_end}, cigar={self.cigar_extended()!r})")

    @staticmethod
    def _from(a: _abi.HyAlignment, ops) -> "Alignment":
        o, n = int(a.ops_offset), int(a.n_ops)
        return Alignment(a.score, a.query_start, a.query_end, a.target_start, a.target_end,
                         C.string_at(C.addressof(ops.contents) + o, n) if n else b"")


@dataclass(frozen=True)
class AlignedHit:
    """src/align.rs:85-92: a database index with the alignment against that sequence."""
    db_index: int
    alignment: Alignment


# ---- scoring (src/scoring.rs) ----------------------------------------------------------------------

def _i32_array(values) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=np.int64)).astype(np.int32)


class Scoring:
    """A validated substitution matrix plus affine gaps (src/scoring.rs:41-100): a gap of length n
    costs ``gap_open + (n - 1) * gap_ext``."""

    def __init__(self, alphabet_len: int, matrix: Sequence[int], gap_open: int, gap_ext: int):
        mat = _i32_array(matrix) if len(matrix) else np.zeros(0, dtype=np.int32)
        _check(lib.hy_scoring_validate(alphabet_len, mat.ctypes.data_as(_abi._i32p), len(mat),
                                       gap_open, gap_ext))
        self._al = int(alphabet_len)
        self._matrix = mat
        self._go = int(gap_open)
        self._ge = int(gap_ext)

    @staticmethod
    def new(alphabet_len, matrix, gap_open, gap_ext) -> "Scoring":
        return Scoring(alphabet_len, matrix, gap_open, gap_ext)

    def alphabet_len(self) -> int:
        return self._al

    def gap_open(self) -> int:
        return self._go

    def gap_ext(self) -> int:
        return self._ge

    def matrix(self) -> np.ndarray:
        return self._matrix

    def entry_bounds(self):
        return int(self._matrix.min()), int(self._matrix.max())

    def score(self, q: int, t: int) -> int:
        if not (0 <= q < self._al and 0 <= t < self._al):
            raise IndexError(f"symbol index out of range: q={q}, t={t}, alphabet_len={self._al}")
        return int(self._matrix[q * self._al + t])

    def required_width(self, mode: Mode, max_query_len: int, max_target_len: int) -> ScoreWidth:
        lo, hi = self.entry_bounds()
        return required_width(mode, lo, hi, self._go, self._ge, max_query_len, max_target_len)

    def __eq__(self, other):
        return (isinstance(other, Scoring) and self._al == other._al and self._go == other._go
                and self._ge == other._ge and np.array_equal(self._matrix, other._matrix))


def required_width(mode, min_entry, max_entry, gap_open, gap_ext, max_query_len, max_target_len):
    """width::required_width (src/width.rs:145-169)."""
    w = C.c_int()
    b = C.c_int64()
    _check(lib.hy_required_width(int(mode), min_entry, max_entry, gap_open, gap_ext,
                                 min(int(max_query_len), 2**64 - 1), min(int(max_target_len), 2**64 - 1),
                                 C.byref(w), C.byref(b)))
    return ScoreWidth(w.value)


# ---- sequences ---------------------------------------------------------------------------------------

def _as_u8(seq) -> np.ndarray:
    if isinstance(seq, np.ndarray):
        return np.ascontiguousarray(seq, dtype=np.uint8)
    if isinstance(seq, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(seq), dtype=np.uint8)
    return np.asarray(list(seq), dtype=np.int64).astype(np.uint8) if len(seq) else np.zeros(0, np.uint8)


def concat(seqs: Iterable) -> tuple:
    """Concatenate sequences into (residues uint8, offsets uint64 of len n+1)."""
    parts = [_as_u8(s) for s in seqs]
    offsets = np.zeros(len(parts) + 1, dtype=np.uint64)
    if parts:
        offsets[1:] = np.cumsum([len(p) for p in parts], dtype=np.uint64)
    residues = np.concatenate(parts) if parts and offsets[-1] > 0 else np.zeros(1, np.uint8)
    return np.ascontiguousarray(residues, dtype=np.uint8), offsets


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


# ---- database (src/database.rs) ------------------------------------------------------------------------

class Database:
    """An immutable, device-resident database (src/database.rs:47-63). Shareable across threads;
    each thread scans with its own ``Scratch``."""

    def __init__(self, handle, n_seqs):
        self._h = C.c_void_p(handle)
        self._n = n_seqs

    def __del__(self, _lib=lib):
        # _lib keeps the library reachable when the module is torn down at interpreter exit.
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.hy_db_destroy(h)
            self._h = C.c_void_p(None)

    @staticmethod
    def builder() -> "DatabaseBuilder":
        return DatabaseBuilder()

    # -- scans --
    def scan(self, scratch: "Scratch", query) -> BestHit:
        q = _as_u8(query)
        out = _abi.HyHit()
        _check(lib.hy_scan(self._h, scratch._h, _ptr(q, _abi._u8p), len(q), C.byref(out)))
        return BestHit._from(out)

    def scan_all(self, scratch: "Scratch", query, out: list) -> None:
        arr = self.scan_all_array(scratch, query)
        out.clear()
        for h in arr:
            out.append(BestHit._from(h))

    def scan_all_array(self, scratch: "Scratch", query):
        q = _as_u8(query)
        arr = (_abi.HyHit * self._n)()
        _check(lib.hy_scan_all(self._h, scratch._h, _ptr(q, _abi._u8p), len(q), arr))
        return arr

    def scan_scores(self, scratch: "Scratch", query, out: list) -> None:
        res = self.scan_scores_array(scratch, query)
        out.clear()
        out.extend(int(x) for x in res)

    def scan_scores_array(self, scratch: "Scratch", query) -> np.ndarray:
        q = _as_u8(query)
        res = np.empty(self._n, dtype=np.int32)
        _check(lib.hy_scan_scores(self._h, scratch._h, _ptr(q, _abi._u8p), len(q), _ptr(res, _abi._i32p)))
        return res

    # -- traceback (src/database.rs:517-565) --
    def scan_aligned(self, scratch: "Scratch", query) -> AlignedHit:
        """The winner of ``scan`` (same tie-break) with its full alignment."""
        q = _as_u8(query)
        out = _abi.HyAlignment()
        idx = C.c_uint64()
        ops = _abi._u8p()
        _check(lib.hy_scan_aligned(self._h, scratch._h, _ptr(q, _abi._u8p), len(q), C.byref(idx),
                                   C.byref(out), C.byref(ops)))
        return AlignedHit(int(idx.value), Alignment._from(out, ops))

    def scan_all_aligned_arrays(self, scratch: "Scratch", query):
        """The raw form of ``scan_all_aligned``: a numpy structured view of the per-sequence
        records (score, spans, n_ops, ops_offset) and the concatenated operations (uint8)."""
        q = _as_u8(query)
        arr = (_abi.HyAlignment * self._n)()
        ops = _abi._u8p()
        _check(lib.hy_scan_all_aligned(self._h, scratch._h, _ptr(q, _abi._u8p), len(q), arr, C.byref(ops)))
        total = 0
        if self._n:
            last = arr[self._n - 1]
            total = int(last.ops_offset) + int(last.n_ops)
        buf = np.frombuffer(C.string_at(ops, total), dtype=np.uint8) if total else np.zeros(0, np.uint8)
        return arr, buf

    def scan_all_aligned(self, scratch: "Scratch", query, out: list) -> None:
        """One ``Alignment`` per database sequence, in database order."""
        arr, buf = self.scan_all_aligned_arrays(scratch, query)
        raw = buf.tobytes()
        out.clear()
        for a in arr:
            o = int(a.ops_offset)
            out.append(Alignment(a.score, a.query_start, a.query_end, a.target_start, a.target_end,
                                 raw[o: o + int(a.n_ops)]))

    # -- accessors (src/database.rs:570-638) --
    def traceback_max_bytes(self) -> int:
        return int(lib.hy_db_traceback_max_bytes(self._h))

    def sequence_count(self) -> int:
        return self._n

    def mode(self) -> Mode:
        return Mode(lib.hy_db_mode(self._h))

    def search_type(self):
        st = SearchType(lib.hy_db_search_type(self._h))
        return AlignmentSearch(self.traceback_max_bytes()) if st is SearchType.Alignment else st

    def score_width(self) -> ScoreWidth:
        return ScoreWidth(lib.hy_db_score_width(self._h))

    def backend(self) -> Backend:
        return Backend(lib.hy_db_backend(self._h))

    def layout(self) -> Optional[Layout]:
        return Layout(lib.hy_db_layout(self._h))

    def max_query_len(self) -> int:
        return int(lib.hy_db_max_query_len(self._h))

    def max_target_len(self) -> int:
        return int(lib.hy_db_max_target_len(self._h))

    def device_bytes(self) -> int:
        return int(lib.hy_db_device_bytes(self._h))

    def scratch_bytes(self) -> int:
        return int(lib.hy_db_scratch_bytes(self._h))

    def partition(self):
        a, b = C.c_uint64(), C.c_uint64()
        lib.hy_db_partition(self._h, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)


class DatabaseBuilder:
    """DatabaseBuilder (src/database.rs:657-877). Required: sequences, scoring, mode,
    max_query_len; search_type defaults to Score."""

    def __init__(self):
        self._seqs = None
        self._scoring = None
        self._mode = None
        self._st = None
        self._mql = None
        self._backend = None
        self._layout = None

    def sequences(self, seqs) -> "DatabaseBuilder":
        self._seqs = concat(seqs)
        return self

    def sequences_concat(self, residues: np.ndarray, offsets: np.ndarray) -> "DatabaseBuilder":
        """The same database given already concatenated: sequence k is
        residues[offsets[k]:offsets[k+1]]."""
        res = np.ascontiguousarray(residues, dtype=np.uint8)
        if res.size == 0:
            res = np.zeros(1, np.uint8)
        self._seqs = (res, np.ascontiguousarray(offsets, dtype=np.uint64))
        return self

    def scoring(self, scoring: Scoring) -> "DatabaseBuilder":
        self._scoring = scoring
        return self

    def mode(self, mode: Mode) -> "DatabaseBuilder":
        self._mode = Mode(mode)
        return self

    def search_type(self, st) -> "DatabaseBuilder":
        self._st = st if isinstance(st, AlignmentSearch) else SearchType(st)
        return self

    def max_query_len(self, n: int) -> "DatabaseBuilder":
        self._mql = int(n)
        return self

    def backend(self, choice: BackendChoice) -> "DatabaseBuilder":
        self._backend = choice
        return self

    def layout(self, choice: LayoutChoice) -> "DatabaseBuilder":
        self._layout = choice
        return self

    def build(self) -> Database:
        for name, val in (("sequences", self._seqs), ("scoring", self._scoring),
                          ("mode", self._mode), ("max_query_len", self._mql)):
            if val is None:
                raise Error("IncompleteBuilder", field=name)
        res, off = self._seqs
        n = len(off) - 1
        sc = self._scoring
        st = self._st if self._st is not None else SearchType.Score
        tb_budget = st.max_bytes if isinstance(st, AlignmentSearch) else USIZE_MAX
        choice = _abi.CHOICE_UNSET if self._backend is None else self._backend._code()
        layout = _abi.LAYOUT_AUTO if self._layout is None else self._layout._code()
        h = C.c_void_p()
        status = lib.hy_db_create(_ptr(res, _abi._u8p), _ptr(off, _abi._u64p), n,
                                  _ptr(sc._matrix, _abi._i32p), sc._al, sc._go, sc._ge, int(self._mode),
                                  int(st), tb_budget, self._mql, choice, layout, C.byref(h))
        if status == 10:  # InvalidBackendName from HYALITE_BACKEND
            raise Error("InvalidBackendName", name=os.environ.get(BACKEND_ENV_VAR, ""))
        _check(status)
        return Database(h.value, n)


class Scratch:
    """Per-thread working memory (src/database.rs:954-998): one CUDA stream plus device buffers."""

    def __init__(self, db: Database):
        h = C.c_void_p()
        _check(lib.hy_scratch_create(db._h, C.byref(h)))
        self._h = h
        self._db = db  # keep the database alive while the scratch exists

    def __del__(self, _lib=lib):
        # _lib keeps the library reachable when the module is torn down at interpreter exit.
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.hy_scratch_destroy(h)
            self._h = C.c_void_p(None)

    @staticmethod
    def new(db: Database) -> "Scratch":
        return Scratch(db)

    def stream_ptr(self) -> int:
        return int(lib.hy_scratch_stream(self._h) or 0)


# ---- batched scan (no reference counterpart) ---------------------------------------------------------------

class Batch:
    """Many queries per call, each against one of a fixed list of databases (any modes): the same
    BestHit per query as ``Database.scan``, computed by persistent kernels under a CUDA graph
    (hy_scan_batch). With ``autotune`` the first call of each batch shape tunes the launch shapes."""

    def __init__(self, dbs: Sequence[Database], max_queries: int, autotune: bool = True):
        dbs = list(dbs)
        arr = (C.c_void_p * len(dbs))(*[d._h.value for d in dbs])
        h = C.c_void_p()
        _check(lib.hy_batch_create(arr, len(dbs), int(max_queries), 1 if autotune else 0, C.byref(h)))
        self._h = h
        self._dbs = dbs  # keep the databases alive while the batch exists
        self.max_queries = int(max_queries)

    def __del__(self, _lib=lib):
        # _lib keeps the library reachable when the module is torn down at interpreter exit.
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.hy_batch_destroy(h)
            self._h = C.c_void_p(None)

    @staticmethod
    def _pack(queries, db_of_query):
        qs = [_as_u8(q) for q in queries]
        off = np.zeros(len(qs) + 1, dtype=np.uint64)
        off[1:] = np.cumsum([len(q) for q in qs]) if qs else []
        res = np.concatenate(qs) if qs and off[-1] > 0 else np.zeros(1, np.uint8)
        dbq = np.zeros(len(qs), np.uint32) if db_of_query is None else np.ascontiguousarray(db_of_query, np.uint32)
        if len(dbq) != len(qs):
            raise ValueError("db_of_query must name one database per query")
        return res, off, dbq

    def scan_arrays(self, q_res, q_off, db_of_query):
        """Hits (a ctypes array of hy_hit) for concatenated queries; raises the first query's error
        with ``failed_query`` set on the exception."""
        q_res = np.ascontiguousarray(q_res, dtype=np.uint8)
        q_res = q_res if q_res.size else np.zeros(1, np.uint8)
        q_off = np.ascontiguousarray(q_off, dtype=np.uint64)
        dbq = np.ascontiguousarray(db_of_query, dtype=np.uint32)
        n = len(q_off) - 1
        out = (_abi.HyHit * max(n, 1))()
        failed = C.c_uint32(0)
        st = lib.hy_scan_batch(self._h, n, _ptr(dbq, _abi._u32p), _ptr(q_res, _abi._u8p),
                               _ptr(q_off, _abi._u64p), out, C.byref(failed))
        if st != _abi.OK:
            err = Error.from_status(st)
            err.failed_query = int(failed.value)
            raise err
        return out

    def scan(self, queries, db_of_query=None) -> List[BestHit]:
        res, off, dbq = self._pack(queries, db_of_query)
        arr = self.scan_arrays(res, off, dbq)
        return [BestHit._from(arr[i]) for i in range(len(off) - 1)]

    def tune(self, queries, db_of_query=None, stride: int = 0) -> float:
        """Runs the autotuner on this batch now; returns the chosen configuration's sampled ms."""
        res, off, dbq = self._pack(queries, db_of_query)
        ms = C.c_double()
        _check(lib.hy_batch_tune(self._h, len(off) - 1, _ptr(dbq, _abi._u32p), _ptr(res, _abi._u8p),
                                 _ptr(off, _abi._u64p), int(stride), C.byref(ms)))
        return float(ms.value)

    def config(self):
        """(max query length with 8 rows per lane, with 16 rows, long-pair width split)."""
        c = (C.c_int32 * 3)()
        _check(lib.hy_batch_get_config(self._h, c))
        return tuple(int(x) for x in c)

    def set_config(self, rows8_max: int, rows16_max: int, long_w: int) -> None:
        c = (C.c_int32 * 3)(rows8_max, rows16_max, long_w)
        _check(lib.hy_batch_set_config(self._h, c))

    def device_bytes(self) -> int:
        return int(lib.hy_batch_device_bytes(self._h))

    def stream_ptr(self) -> int:
        return int(lib.hy_batch_stream(self._h) or 0)


# ---- served scan (no reference counterpart) -----------------------------------------------------------------

class ServerRequest:
    """A submitted request: its id and, for a scores request, the array the scores land in."""

    def __init__(self, rid: int, db: int, scores: Optional[np.ndarray]):
        self.id = rid
        self.db = db
        self.scores = scores
        self.latency_ms: Optional[float] = None  # submit to result ready, once waited for


class Server:
    """A request loop over a fixed list of databases (hy_server): requests are admitted by memory
    into device batches, several batches run at once, and each result equals the plain call's."""

    def __init__(self, dbs: Sequence[Database], max_batch: int = 64, in_flight: int = 2,
                 max_pending: int = 4096, profile_budget: int = 0, scores_budget: int = 0,
                 launch_config=None):
        dbs = list(dbs)
        arr = (C.c_void_p * len(dbs))(*[d._h.value for d in dbs])
        cfg = _abi.HyServerConfig()
        cfg.max_batch, cfg.in_flight, cfg.max_pending = max_batch, in_flight, max_pending
        cfg.profile_budget, cfg.scores_budget = profile_budget, scores_budget
        if launch_config is not None:
            for i, v in enumerate(launch_config):
                cfg.launch_config[i] = int(v)
        h = C.c_void_p()
        _check(lib.hy_server_create(arr, len(dbs), C.byref(cfg), C.byref(h)))
        self._h = h
        self._dbs = dbs
        # Requests not yet waited for: the server writes their score arrays at completion, so the
        # arrays stay referenced here until wait() or close().
        self._live = {}

    def close(self, _lib=lib) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.hy_server_destroy(h)
            self._h = C.c_void_p(None)
        self._live = {}

    def __del__(self):
        self.close()

    def submit(self, query, db: int = 0, want_scores: bool = False) -> ServerRequest:
        q = _as_u8(query)
        qb = q if q.size else np.zeros(1, np.uint8)
        scores = np.empty(self._dbs[db].sequence_count(), dtype=np.int32) if want_scores else None
        sp = _ptr(scores, _abi._i32p) if want_scores else None
        rid = C.c_uint64()
        _check(lib.hy_server_submit(self._h, int(db), _ptr(qb, _abi._u8p), len(q), 1 if want_scores else 0,
                                    sp, C.byref(rid)))
        req = ServerRequest(int(rid.value), int(db), scores)
        self._live[req.id] = req
        return req

    def request_bytes(self, qlen: int, db: int = 0, want_scores: bool = False):
        """(query-profile bytes, score-output bytes) a request takes from its batch's budgets."""
        sb = C.c_uint64()
        pb = lib.hy_server_request_bytes(self._h, int(db), int(qlen), 1 if want_scores else 0, C.byref(sb))
        return int(pb), int(sb.value)

    def poll(self, req: ServerRequest) -> bool:
        done = C.c_int()
        _check(lib.hy_server_poll(self._h, req.id, C.byref(done)))
        return bool(done.value)

    def wait(self, req: ServerRequest, timeout: float = 600.0) -> BestHit:
        """The request's BestHit (for a scores request, its scores are then in ``req.scores``);
        ``req.latency_ms`` receives its latency, submit to result ready."""
        out = _abi.HyHit()
        lat = C.c_double()
        st = lib.hy_server_wait_timed(self._h, req.id, float(timeout), C.byref(out), C.byref(lat))
        if st != _abi.TIMEOUT:
            self._live.pop(req.id, None)
        _check(st)
        req.latency_ms = float(lat.value)
        return BestHit._from(out)

    def stats(self, reset: bool = False) -> dict:
        s = _abi.HyServerStats()
        _check(lib.hy_server_stats_read(self._h, 1 if reset else 0, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}


# ---- pairwise batch (src/kernel.rs:429-452) -------------------------------------------------------------

def align_pairs_arrays(q_res, q_off, t_res, t_off, scoring: Scoring, mode: Mode, search_type: SearchType):
    """align_pairs over concatenated queries and targets; returns (hits ctypes array, error or None).
    On an error, hits[:failed] are valid."""
    q_res = np.ascontiguousarray(q_res, dtype=np.uint8)
    t_res = np.ascontiguousarray(t_res, dtype=np.uint8)
    q_res = q_res if q_res.size else np.zeros(1, np.uint8)
    t_res = t_res if t_res.size else np.zeros(1, np.uint8)
    q_off = np.ascontiguousarray(q_off, dtype=np.uint64)
    t_off = np.ascontiguousarray(t_off, dtype=np.uint64)
    n = len(q_off) - 1
    out = (_abi.HyHit * max(n, 1))()
    failed = C.c_uint64()
    st = lib.hy_align_pairs(_ptr(q_res, _abi._u8p), _ptr(q_off, _abi._u64p), _ptr(t_res, _abi._u8p),
                            _ptr(t_off, _abi._u64p), n, _ptr(scoring._matrix, _abi._i32p), scoring._al,
                            scoring._go, scoring._ge, int(mode), int(search_type), out, C.byref(failed))
    err = None if st == _abi.OK else Error.from_status(st)
    return out, (err, int(failed.value))


def align(query, target, scoring: Scoring, mode: Mode, max_bytes: int) -> Alignment:
    """align (src/align.rs:169-222): the full alignment of one pair, traced back on the device.
    ``max_bytes`` is the reference's traceback budget (``USIZE_MAX`` for usize::MAX)."""
    q, t = _as_u8(query), _as_u8(target)
    out = _abi.HyAlignment()
    ops = np.zeros(max(1, len(q) + len(t)), np.uint8)
    _check(lib.hy_align(_ptr(q, _abi._u8p), len(q), _ptr(t, _abi._u8p), len(t),
                        _ptr(scoring._matrix, _abi._i32p), scoring._al, scoring._go, scoring._ge,
                        int(Mode(mode)), int(max_bytes), C.byref(out), _ptr(ops, _abi._u8p)))
    return Alignment(out.score, out.query_start, out.query_end, out.target_start, out.target_end,
                     ops[: int(out.n_ops)].tobytes())


def traceback_timing(scratch: Optional["Scratch"] = None) -> dict:
    """Timing of the last traceback call of ``scratch`` (None: this thread's ``align``): device ms
    of the fill and of the walk + compaction kernels, the device span (first fill to the end of
    compaction; walks overlap the next chunk's fill), the whole call's ms, and the cells traced."""
    out = (C.c_double * 5)()
    _check(lib.hy_traceback_timing(None if scratch is None else scratch._h, out))
    return {"fill_ms": out[0], "walk_ms": out[1], "device_ms": out[2], "call_ms": out[3], "cells": out[4]}


def traceback_min_bytes_for_database(max_m: int, max_n: int) -> int:
    """src/align.rs:245-250."""
    return int(lib.hy_traceback_min_bytes_for_database(max_m, max_n))


def align_pairs_timing():
    """(device ms of the call's kernels: packing, pair and stripe kernels; whole call ms) of this
    thread's last align_pairs call."""
    k, c = C.c_double(), C.c_double()
    _check(lib.hy_align_pairs_timing(C.byref(k), C.byref(c)))
    return float(k.value), float(c.value)


def pinned_empty(n: int, dtype=np.uint8) -> np.ndarray:
    """An uninitialised numpy array of n elements in page-locked host memory (hy_host_alloc), freed
    when the last view of it goes. align_pairs / align_pairs_position_max copy such residues and
    column-maxima arrays from and to where they are, without staging copies."""
    dt = np.dtype(dtype)
    nbytes = max(1, int(n) * dt.itemsize)
    ptr = C.c_void_p()
    _check(lib.hy_host_alloc(nbytes, C.byref(ptr)))
    buf = (C.c_uint8 * nbytes).from_address(ptr.value)
    weakref.finalize(buf, lib.hy_host_free, ptr.value)
    return np.frombuffer(buf, dtype=dt, count=int(n))


def align_pairs_phases():
    """Phases (ms) of this thread's last align_pairs call: the host lengths pass and routing; host
    sort and item packing, and waits for the staging copies (which run on their own threads beside
    the next chunk's sort), each summed over the chunks; the chunk pipeline
    (wall time to the device's end, overlapping the two before); results; host waits for a staging
    slot; host copies of the column maxima (align_pairs_position_max, whose last call it also
    reports)."""
    out = (C.c_double * 7)()
    _check(lib.hy_align_pairs_phases(out, 7))
    return {"lengths": out[0], "sort_pack": out[1], "staging": out[2], "pipeline": out[3], "results": out[4],
            "slot_wait": out[5], "colmax_copy": out[6]}


def align_pairs_position_max_arrays(q_res, q_off, t_res, t_off, scoring: Scoring, min_score: Optional[int] = None,
                                    colmax_out: Optional[np.ndarray] = None):
    """align_pair_position_max over many pairs (src/kernel.rs:474-553) on the device: returns
    (hits ctypes array, column maxima int32 array aligned with t_res, score2 int32 array of
    (score, position) per pair or None, (error or None, failed index)). ``min_score`` set: each pair's
    score2 (src/kernel.rs:741-792) with its best score, its target end (0 when None) and the
    matrix's largest entry; position -1 means None. ``colmax_out``: a contiguous int32 array of at
    least t_off[-1] - t_off[0] entries refilled in place and returned (the reference's ``out``
    vector is likewise the caller's, cleared and refilled), instead of a new array a call."""
    q_res = np.ascontiguousarray(q_res, dtype=np.uint8)
    t_res = np.ascontiguousarray(t_res, dtype=np.uint8)
    q_res = q_res if q_res.size else np.zeros(1, np.uint8)
    t_res = t_res if t_res.size else np.zeros(1, np.uint8)
    q_off = np.ascontiguousarray(q_off, dtype=np.uint64)
    t_off = np.ascontiguousarray(t_off, dtype=np.uint64)
    n = len(q_off) - 1
    out = (_abi.HyHit * max(n, 1))()
    need = max(1, int(t_off[-1] - t_off[0])) if n else 1
    if colmax_out is not None:
        if colmax_out.dtype != np.int32 or not colmax_out.flags.c_contiguous or colmax_out.size < need:
            raise ValueError("colmax_out must be a contiguous int32 array of t_off[-1] - t_off[0] entries")
        cm = colmax_out
    else:
        cm = np.zeros(need, np.int32)
    s2 = np.zeros(2 * max(n, 1), np.int32) if min_score is not None else None
    failed = C.c_uint64()
    st = lib.hy_align_pairs_position_max(
        _ptr(q_res, _abi._u8p), _ptr(q_off, _abi._u64p), _ptr(t_res, _abi._u8p), _ptr(t_off, _abi._u64p), n,
        _ptr(scoring._matrix, _abi._i32p), scoring._al, scoring._go, scoring._ge, _ptr(cm, _abi._i32p), out,
        0 if min_score is None else int(min_score), None if s2 is None else _ptr(s2, _abi._i32p), C.byref(failed))
    err = None if st == _abi.OK else Error.from_status(st)
    return out, cm, s2, (err, int(failed.value))


def position_max_timing() -> dict:
    """This thread's last position-max call: device ms of its kernels, whole call ms, cells."""
    out = (C.c_double * 3)()
    _check(lib.hy_position_max_timing(out))
    return {"kernel_ms": out[0], "call_ms": out[1], "cells": out[2]}


def align_pair_position_max(query, target, scoring: Scoring, out: list) -> BestHit:
    """align_pair_position_max (src/kernel.rs:474-553): ``out`` is cleared and refilled with the
    best SW score ending at each target position; returns the BestHit (query_end None)."""
    q, t = _as_u8(query), _as_u8(target)
    qo = np.array([0, len(q)], np.uint64)
    to = np.array([0, len(t)], np.uint64)
    hits, cm, _, (err, _) = align_pairs_position_max_arrays(q, qo, t, to, scoring)
    out.clear()
    if err is not None:
        raise err
    out.extend(int(v) for v in cm[: len(t)])
    return BestHit._from(hits[0])


def score2(colmax, best_score: int, best_target_end: int, matrix_max: int, min_score: int):
    """score2 (src/kernel.rs:741-792): bwa's second-best peak outside the best hit's window, as
    (score, position), or None."""
    cm = np.ascontiguousarray(np.asarray(colmax, dtype=np.int64).astype(np.int32))
    sc, pos = C.c_int32(), C.c_uint64()
    ok = lib.hy_score2(_ptr(cm if cm.size else np.zeros(1, np.int32), _abi._i32p), len(cm), int(best_score),
                       int(best_target_end), int(matrix_max), int(min_score), C.byref(sc), C.byref(pos))
    return (int(sc.value), int(pos.value)) if ok else None


def align_pair(query, target, scoring: Scoring, mode: Mode, search_type) -> BestHit:
    """align_pair (src/kernel.rs:331-352): one pair's BestHit (db_index 0). A long pair (a query of
    256 residues or more and at least 1 Mi cells) runs on the stripe kernel, every 128 query rows
    on their own warp."""
    out: list = []
    align_pairs([(query, target)], scoring, mode, search_type, out)
    return out[0]


def align_pairs(pairs, scoring: Scoring, mode: Mode, search_type: SearchType, out: list) -> None:
    """Align independent (query, target) pairs; one BestHit per pair in input order with
    db_index = pair index. Raises the first failing pair's error; ``out`` then holds the hits of
    the pairs before it (src/kernel.rs:429-452)."""
    qs, ts = zip(*pairs) if pairs else ((), ())
    q_res, q_off = concat(qs)
    t_res, t_off = concat(ts)
    hits, (err, failed) = align_pairs_arrays(q_res, q_off, t_res, t_off, scoring, mode, search_type)
    out.clear()
    upto = len(pairs) if err is None else failed
    for k in range(upto):
        out.append(BestHit._from(hits[k]))
    if err is not None:
        raise err


__all__ = [
    "BACKEND_ENV_VAR", "Backend", "BackendChoice", "BestHit", "Database", "DatabaseBuilder", "Error",
    "Batch", "Layout", "LayoutChoice", "Mode", "ALL_MODES", "ScoreWidth", "Scoring", "Scratch", "SearchType",
    "Server", "ServerRequest", "AlignOp", "Alignment", "AlignedHit", "AlignmentSearch", "USIZE_MAX",
    "align", "align_pair", "align_pairs", "align_pairs_arrays", "required_width", "concat",
    "traceback_min_bytes_for_database", "traceback_timing", "align_pair_position_max",
    "align_pairs_position_max_arrays", "score2", "position_max_timing",
]
