"""Helpers for the GPU parity tests: build the same database in the cuda backend and in the CPU
oracle and compare scan / scan_all / scan_scores bit for bit."""
import numpy as np

import pyoracle as o

import hyalite_b200 as hy

# The standard BLOSUM62 matrix (Henikoff & Henikoff 1992; public domain), order ARNDCQEGHILKMFPSTWYV.
BLOSUM62 = [
    4, -1, -2, -2, 0, -1, -1, 0, -2, -1, -1, -1, -1, -2, -1, 1, 0, -3, -2, 0,
    -1, 5, 0, -2, -3, 1, 0, -2, 0, -3, -2, 2, -1, -3, -2, -1, -1, -3, -2, -3,
    -2, 0, 6, 1, -3, 0, 0, 0, 1, -3, -3, 0, -2, -3, -2, 1, 0, -4, -2, -3,
    -2, -2, 1, 6, -3, 0, 2, -1, -1, -3, -4, -1, -3, -3, -1, 0, -1, -4, -3, -3,
    0, -3, -3, -3, 9, -3, -4, -3, -3, -1, -1, -3, -1, -2, -3, -1, -1, -2, -2, -1,
    -1, 1, 0, 0, -3, 5, 2, -2, 0, -3, -2, 1, 0, -3, -1, 0, -1, -2, -1, -2,
    -1, 0, 0, 2, -4, 2, 5, -2, 0, -3, -3, 1, -2, -3, -1, 0, -1, -3, -2, -2,
    0, -2, 0, -1, -3, -2, -2, 6, -2, -4, -4, -2, -3, -3, -2, 0, -2, -2, -3, -3,
    -2, 0, 1, -1, -3, 0, 0, -2, 8, -3, -3, -1, -2, -1, -2, -1, -2, -2, 2, -3,
    -1, -3, -3, -3, -1, -3, -3, -4, -3, 4, 2, -3, 1, 0, -3, -2, -1, -3, -1, 3,
    -1, -2, -3, -4, -1, -2, -3, -4, -3, 2, 4, -2, 2, 0, -3, -2, -1, -2, -1, 1,
    -1, 2, 0, -1, -3, 1, 1, -2, -1, -3, -2, 5, -1, -3, -1, 0, -1, -3, -2, -2,
    -1, -1, -2, -3, -1, 0, -2, -3, -2, 1, 2, -1, 5, 0, -2, -1, -1, -1, -1, 1,
    -2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0, -3, 0, 6, -4, -2, -2, 1, 3, -1,
    -1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2,
    1, -1, 1, 0, -1, 0, 0, 0, -1, -2, -2, 0, -1, -2, -1, 4, 1, -3, -2, -2,
    0, -1, 0, -1, -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1, 5, -2, -2, 0,
    -3, -3, -4, -4, -2, -2, -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2, -3,
    -2, -2, -2, -3, -2, -1, -2, -3, 2, -1, -1, -2, -1, 3, -3, -2, -2, 2, 7, -2,
    0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1, -2, 1, -1, -2, -2, 0, -3, -2, 4,
]
AMINO = "ARNDCQEGHILKMFPSTWYV"


def hit_tuple(h):
    return (h.score, h.db_index, h.query_end, h.target_end)


def build(seqs, matrix, al, go, ge, mode, st, mql):
    return (hy.Database.builder().sequences(seqs).scoring(hy.Scoring(al, matrix, go, ge))
            .mode(hy.Mode(mode)).search_type(hy.SearchType(st)).max_query_len(mql).build())


def check(seqs, matrix, al, go, ge, mode, st, queries, mql=None, all_too=True):
    """Every query: cuda scan == oracle scan; scan_all / scan_scores == oracle per target. One
    Scratch is reused across all queries (catches stale device buffers, tests/sweeps.rs:56-116)."""
    if mql is None:
        mql = max([len(q) for q in queries] + [1])
    db = build(seqs, matrix, al, go, ge, mode, st, mql)
    ref = o.OracleDb(seqs, matrix, al, go, ge, mode, st)
    sc = hy.Scratch(db)
    for q in queries:
        want = ref.scan(q)
        got = hit_tuple(db.scan(sc, q))
        assert got == want, f"scan mode={mode} st={st} q={list(q)[:20]} n={len(seqs)} got={got} want={want}"
        if all_too:
            arr = db.scan_all_array(sc, q)
            got_all = [(h.score, h.db_index, None if h.query_end < 0 else h.query_end,
                        None if h.target_end < 0 else h.target_end) for h in arr]
            want_all = ref.scan_all(q)
            if got_all != want_all:
                bad = [k for k in range(len(want_all)) if got_all[k] != want_all[k]][:5]
                raise AssertionError(f"scan_all mode={mode} st={st}: first diffs "
                                     f"{[(k, got_all[k], want_all[k], len(seqs[k])) for k in bad]}")
            got_sc = db.scan_scores_array(sc, q)
            want_sc = ref.scan_scores(q)
            assert np.array_equal(got_sc, want_sc), f"scan_scores mode={mode}"
    return db


def rand_seqs(rng, n, al, lo, hi):
    return [list(rng.integers(0, al, int(rng.integers(lo, hi + 1)))) for _ in range(n)]
